#!/usr/bin/env python
"""bench.py -- sigma-build throughput of the determinant-CI hot path.

Workload (default): FCI(12e,12o), 924 x 924 = 853 776 determinants, the
3-root configuration, seeded synthetic integrals (rank 12, seed 102) -- the
largest named configuration the metric is quoted on that fits one GPU run of
a few seconds.  A step is one sigma = H c build for a block of 3 vectors (one
per root) in FP64 with every input resident in HBM; the L2 (126 MB) is
flushed by writing a 256 MiB buffer before every step because the vectors
and tables would otherwise stay L2-resident.

value  = determinants x vectors / sigma time  (Gdet/s, all ranks)
e2e    = the same through the public C ABI (jci_sigma) from pinned host
         buffers, host->device copy of the 3 input vectors and device->host
         copy of the 3 sigma vectors inside every timed step
Extra fields report the FP32 sigma rate and full Davidson solves (plain
FP64 reference schedule vs mixed FP32->FP64 block Davidson, energies
compared) measured outside the timed region.

--impl reference times the reference's own CPU code (oracle/_ref, the
reference's mpi_source compiled unchanged against a single-process GA/MPI
stand-in) on the same workload: each step runs the reference's sigma
kernel compute_cblock_Hfastest with all host threads over a fixed sample of
rows spread evenly across the determinant list and extrapolates to the full
sigma.  Multi-GPU runs (torchrun) are replicas: every rank builds the same
workload independently (weak scaling); no data-path collective exists.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (&general electrons, orbitals, nfrozen), roots, alpha singles s, doubles d
    "fci12_12": ((12, 12, 0), 3, 36, 225),
    "cas10_10": ((10, 10, 0), 1, 25, 100),
    "fci14_14_fc2": ((18, 16, 2), 4, 49, 441),
    "fci16_16": ((16, 16, 0), 1, 64, 784),
}
METRIC = json.load(open(os.path.join(ROOT, "BASELINE.json")))["metric"] \
    if os.path.exists(os.path.join(ROOT, "BASELINE.json")) else "sigma-build Gdet/s"


def env_int(k, d):
    return int(os.environ.get(k, d))


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def committed_traffic(workload):
    """Per-launch DRAM bytes of the sigma kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", f"sigma_{workload}_traffic.json")
    if os.path.exists(p):
        try:
            return json.load(open(p)).get("dram_bytes_per_launch")
        except Exception:
            return None
    return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None

    def stop(self):
        if not self.p:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        out, _ = self.p.communicate(timeout=10)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_sample_plan(ndets, chunks=8, frac=0.25):
    rows = max(1, int(ndets * frac / chunks))
    starts = [int((i + 0.5) * ndets / chunks - rows / 2) for i in range(chunks)]
    return [(max(0, min(ndets - rows - 1, s)), rows) for s in starts]


def reference_sigma_sample(name, nvec, frac=0.25):
    """Time the reference's own sigma kernel on an even row sample; returns
    (extrapolated seconds for a full sigma of nvec vectors, sample string)."""
    import ctypes

    import numpy as np

    from jayci_b200.synth import workload_integrals
    from oracle.oracle import RefSpace, _ptr, ref_available
    if not ref_available():
        return None, "reference build absent"
    (e, o, nfc), _, _, _ = WORKLOADS[name]
    ints = workload_integrals(name)
    m1, m2 = ints.packed()
    ref = RefSpace(e, o, nfc)
    L = ref.lib()
    L.ref_sigma_rows_timed.restype = ctypes.c_double
    V = np.random.default_rng(0).standard_normal((nvec, ref.ndets))
    L.ref_sigma_prepare(_ptr(m1), _ptr(m2), nvec, _ptr(V))
    plan = cpu_sample_plan(ref.ndets, frac=frac)
    t = sum(L.ref_sigma_rows_timed(r0, nr) for r0, nr in plan)
    rows = sum(nr for _, nr in plan)
    L.ref_sigma_release()
    return t * ref.ndets / rows, f"{len(plan)} evenly spaced row blocks, {rows} of {ref.ndets} rows"


def run_reference(a):
    rank = env_int("RANK", 0)
    if rank != 0:
        return 0
    (geo, nroots, s, d) = WORKLOADS[a.workload]
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    os.environ.setdefault("OMP_SCHEDULE", "dynamic,64")
    from jayci_b200.synth import WORKLOADS as W
    w = W[a.workload]
    ndets = 1
    import math
    ndets = math.comb(w["n"], w["k"]) ** 2
    vals = []
    sample = ""
    for i in range(a.warmup + a.steps):
        full_s, sample = reference_sigma_sample(a.workload, nroots, frac=a.ref_step_frac)
        if full_s is None:
            print(json.dumps({"impl": "reference", "unavailable": sample}))
            return 0
        if i >= a.warmup:
            vals.append(full_s)
    t = statistics.mean(vals)
    value = ndets * nroots / t / 1e9
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Gdet/s",
           "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
           "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded integrals)",
           "config": {"workload": a.workload, "ndets": ndets, "vectors_per_step": nroots,
                      "sample": sample},
           "cpu_baseline": {"value": value, "unit": "Gdet/s", "cores": threads,
                            "kind": "reference", "sample": sample},
           "e2e": {"value": value, "unit": "Gdet/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def run_gpu(a):
    import numpy as np
    import torch

    import jayci_b200 as jb
    from jayci_b200.synth import workload_integrals

    rank, world, local = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    (geo, nroots, s_exc, d_exc) = WORKLOADS[a.workload]
    ints = workload_integrals(a.workload)
    m1, m2 = ints.packed()
    sp = jb.Space(*geo)
    sp.set_integrals(m1, m2, ints.e_nuc, ints.e_fc)
    N, nvec = sp.ndets, nroots
    stream = torch.cuda.Stream()
    gen = torch.Generator(device="cuda").manual_seed(1234 + rank)
    with torch.cuda.stream(stream):
        V = torch.randn(nvec, N, dtype=torch.float64, device="cuda", generator=gen)
        S = torch.empty_like(V)
        V32 = V.float()
        S32 = torch.empty_like(V32)
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    sh = stream.cuda_stream

    def step(events, prec=jb.FP64, v=V, o=S):
        flush.fill_(1.0)
        for k in range(nvec):
            if events is not None:
                events[k][0].record(stream)
            sp.sigma_device(v[k].data_ptr(), o[k].data_ptr(), 1, N, prec, sh)
            if events is not None:
                events[k][1].record(stream)

    def timed(K, prec, v, o):
        ev = [[[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(nvec)]
              for _ in range(K)]
        with torch.cuda.stream(stream):
            for i in range(K):
                step(ev[i], prec, v, o)
        torch.cuda.synchronize()
        launches = [e[0].elapsed_time(e[1]) for row in ev for e in row]
        return sum(launches), launches

    with torch.cuda.stream(stream):
        for _ in range(a.warmup):
            step(None)
            step(None, jb.FP32, V32, S32)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    tot_ms, launches = timed(a.steps, jb.FP64, V, S)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    tot32_ms, launches32 = timed(a.steps, jb.FP32, V32, S32)
    if dist:
        t = torch.tensor([tot_ms, tot32_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot_ms, tot32_ms = float(t[0]), float(t[1])
    value = world * N * nvec * a.steps / (tot_ms / 1e3) / 1e9
    value32 = world * N * nvec * a.steps / (tot32_ms / 1e3) / 1e9

    # end to end through the C ABI from pinned host memory
    hv = torch.randn(nvec, N, dtype=torch.float64, generator=torch.Generator().manual_seed(7))
    hv = hv.pin_memory()
    hs = torch.empty_like(hv).pin_memory()
    hvn, hsn = hv.numpy(), hs.numpy()
    for _ in range(2):
        jb.lib().jci_sigma(sp.h, nvec, hvn.ctypes.data, hsn.ctypes.data, jb.FP64)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        rc = jb.lib().jci_sigma(sp.h, nvec, hvn.ctypes.data, hsn.ctypes.data, jb.FP64)
        if rc:
            raise jb.JciError(rc, "jci_sigma")
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t[0])
    e2e = world * N * nvec * a.steps / e2e_s / 1e9

    # roofline of the sigma kernel (row-stream algorithmic bytes per vector)
    w = 8
    bytes_per_launch = w * N * (2 + s_exc + d_exc)
    avg_launch_s = statistics.mean(launches) / 1e3
    peak, peak_kind = measured_peaks()
    achieved = bytes_per_launch / avg_launch_s / 1e9
    traffic = committed_traffic(a.workload)
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic,
            "algorithmic_bytes_per_launch": bytes_per_launch, "peak_source": peak_kind,
            "kernel_ms_per_launch": avg_launch_s * 1e3}

    # full solves (outside the timed region): reference schedule FP64 vs mixed block
    solves = {}
    if not a.no_solves:
        kw = dict(maxiter=2000, krymin=6, krymax=24, nroots=nroots, refdim=12, restol=1e-8)
        r64 = sp.davidson(**kw)
        rmx = sp.davidson(precision=jb.MIXED, block=True, **kw)
        solves = {"fp64_solve_s": r64.stats.total_seconds, "fp64_converged": r64.converged,
                  "mixed_solve_s": rmx.stats.total_seconds, "mixed_converged": rmx.converged,
                  "fp64_solves_per_s": world / r64.stats.total_seconds,
                  "mixed_solves_per_s": world / rmx.stats.total_seconds,
                  "mixed_vs_fp64_max_abs_dE": float(np.abs(rmx.energies - r64.energies).max()),
                  "energies_fp64": [float(x) for x in r64.energies],
                  "mixed_speedup": r64.stats.total_seconds / rmx.stats.total_seconds}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        full_s, sample = reference_sigma_sample(a.workload, nvec, frac=a.ref_frac)
        if full_s is not None:
            cpu = {"value": N * nvec / full_s / 1e9, "unit": "Gdet/s",
                   "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"reference sigma (compute_cblock_Hfastest), {nvec} vectors, "
                             f"{sample}, OMP_SCHEDULE=dynamic,64"}
    mode, nt, R, B, _ = sp.sigma_tuning(jb.FP64)
    out = {"metric": METRIC, "value": value, "unit": "Gdet/s", "n_gpus": world,
           "steps": a.steps, "warmup": a.warmup, "ms_per_step": tot_ms / a.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded integrals, random CI vectors)",
           "config": {"workload": a.workload, "ndets": N, "vectors_per_step": nvec,
                      "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                      "l2": "flushed (256 MiB write) before every step",
                      "sigma_plan": {"mode": ["staged rows", "dense product, global panel",
                                              "dense product, shared-memory panel"][mode],
                                     "row_kernel_threads": nt,
                                     ("staged_rows" if mode == 0 else "product_ctas_per_sm"): R,
                                     "rows_per_cta": B}},
           "roofline": roof, "cpu_baseline": cpu,
           "e2e": {"value": e2e, "unit": "Gdet/s", "h2d_bytes_per_step": nvec * N * 8,
                   "d2h_bytes_per_step": nvec * N * 8},
           "gpu_launches": a.steps * nvec * (2 if mode >= 1 else 1),
           "clocks": clk,
           "fp32_sigma_gdet_s": value32,
           "solves": solves}
    if rank == 0:
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="jci", choices=["jci", "reference"])
    ap.add_argument("--workload", default="fci12_12", choices=sorted(WORKLOADS))
    ap.add_argument("--no-solves", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--ref-frac", type=float, default=0.25,
                    help="fraction of rows in the CPU-baseline sample (about 10 s)")
    ap.add_argument("--ref-step-frac", type=float, default=0.02,
                    help="fraction of rows per step of --impl reference")
    a = ap.parse_args()
    if a.warmup < 3:
        a.warmup = 3
    if a.impl == "reference":
        return run_reference(a)
    return run_gpu(a)


if __name__ == "__main__":
    sys.exit(main())
