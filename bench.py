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
FP64 reference schedule vs the mixed FP32->FP64 two-phase schedule,
energies compared) measured outside the timed region.

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
# &dalginfo per workload: krymin, krymax, refdim, maxiter (restol 1e-8)
DALGINFO = {"cas10_10": (4, 12, 8, 500), "fci12_12": (6, 24, 12, 500),
            "fci14_14_fc2": (8, 48, 16, 2000), "fci16_16": (4, 12, 8, 500)}
METRIC = json.load(open(os.path.join(ROOT, "BASELINE.json")))["metric"] \
    if os.path.exists(os.path.join(ROOT, "BASELINE.json")) else "sigma-build Gdet/s"


def env_int(k, d):
    return int(os.environ.get(k, d))


# kernels per sigma vector of each plan (jci_sigma_tuning modes)
SIGMA_KERNELS = {0: 1, 1: 2, 2: 2, 3: 5, 4: 5, 5: 2, 6: 6, 7: 6}
PLAN_NAMES = {0: "staged rows", 1: "row kernel, dense product through a global panel",
              2: "row kernel, dense product from shared-memory chunks",
              3: "row streams on C and C^T, dense product through a global panel",
              4: "row streams on C and C^T, fused product and gather",
              5: "row kernel, fused product and gather",
              6: "string-group doubles, beta-singles stream, dense product through a "
                 "global panel",
              7: "string-group doubles, beta-singles stream, fused product and gather"}


def sigma_plan_desc(mode, nt, R, B):
    streams, groups = mode in (3, 4), mode in (6, 7)
    d = {"mode": mode, "name": PLAN_NAMES[mode],
         ("alpha_pass_threads" if streams else "beta_singles_threads" if groups
          else "row_kernel_threads"): nt,
         ("staged_rows" if mode == 0 else
          "product_column_threads" if mode in (4, 5, 7) else "product_ctas_per_sm"): R}
    if groups:
        d["group_kernel"] = (f"{B} column(s) per thread" if B <= 2 else
                             f"targets split over 4 warps, {5 - B} column(s) per lane")
    else:
        d["beta_pass_threads" if streams else "rows_per_cta"] = B
    return d


def max_over_ranks(dist, values, device):
    """Each value's maximum over all ranks (the slowest replica's time); the
    values themselves when running alone (dist is None)."""
    if dist is None:
        return list(values)
    import torch
    t = torch.tensor(list(values), device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def replica_rate(world, units_per_rank, seconds):
    """Whole-job throughput of independent replicas: the units every rank
    processed over the slowest rank's time (weak scaling), in units/s."""
    return world * units_per_rank / seconds


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def committed_traffic(workload, mode, B):
    """Per-launch DRAM bytes of sigma plan `mode` on `workload` from the
    committed ncu summary, or None when that plan was not captured.  Entries
    are keyed by mode, and for the string-group plans (6, 7) by mode and
    group kernel variant ("7:3")."""
    key = f"{mode}:{B}" if mode in (6, 7) else str(mode)
    p = os.path.join(ROOT, "profiles", f"sigma_{workload}_traffic.json")
    if os.path.exists(p):
        try:
            plan = json.load(open(p)).get("plans", {}).get(key)
            return plan.get("dram_bytes_per_launch") if plan else None
        except Exception:
            return None
    return None


def committed_tensor_pipe(workload):
    """Tensor-pipe utilisation of the kernels that use the tensor cores on
    `workload`, from the committed ncu captures, or None when there is none.
    ncu cannot run inside a timed bench, so these figures are quoted from
    the captures, each with the summary that holds its command."""
    p = os.path.join(ROOT, "profiles", f"tensor_pipe_{workload}.json")
    if os.path.exists(p):
        try:
            d = json.load(open(p))
            return {"source": d["note"],
                    "kernels": [{k: e[k] for k in ("kernel", "use", "pipe", "active_pct",
                                                   "useful_fraction_of_tile", "summary")
                                 if k in e}
                                for e in d["kernels"]]}
        except Exception:
            return None
    return None


class ClockSampler:
    """SM clock and throttle-reason sampling during the timed region: NVML
    (the library nvidia-smi reads) polled from a thread every 2 ms, so short
    timed regions still get samples.  Read-only: no setting is changed."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40,
               "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}

    def __init__(self, dev):
        self.dev = dev
        self.samples, self.mask, self.mx = [], 0, None
        self.t = None
        self.stop_flag = False

    def start(self):
        try:
            import threading

            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByIndex(self.dev)
            self.mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)

            def run():
                while not self.stop_flag:
                    try:
                        self.samples.append(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                        self.mask |= nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    except Exception:
                        pass
                    time.sleep(0.002)
            self.t = threading.Thread(target=run, daemon=True)
            self.t.start()
        except Exception:
            self.t = None

    def stop(self):
        if self.t is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"]}
        self.stop_flag = True
        self.t.join(timeout=5)
        reasons = [n for n, b in self.REASONS.items() if self.mask & b]
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.mx, "reasons": sorted(reasons),
                "samples": len(self.samples)}


def cpu_sample_plan(ndets, chunks=2, frac=0.25):
    """Row blocks of the CPU sample.  Each call of the reference's kernel has a
    fixed cost (about 50 ms here), which small blocks would charge to the
    reference many times over; two blocks of 12.5% keep it under a few percent
    of the timed work."""
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
    tot_ms, tot32_ms = max_over_ranks(dist, [tot_ms, tot32_ms], "cuda")
    value = replica_rate(world, N * nvec * a.steps, tot_ms / 1e3) / 1e9
    value32 = replica_rate(world, N * nvec * a.steps, tot32_ms / 1e3) / 1e9

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
    e2e_s, = max_over_ranks(dist, [e2e_s], "cuda")
    e2e = replica_rate(world, N * nvec * a.steps, e2e_s) / 1e9

    # roofline of the sigma kernel (row-stream algorithmic bytes per vector)
    w = 8
    bytes_per_launch = w * N * (2 + s_exc + d_exc)
    avg_launch_s = statistics.mean(launches) / 1e3
    peak, peak_kind = measured_peaks()
    achieved = bytes_per_launch / avg_launch_s / 1e9
    mode, nt, R, B, _ = sp.sigma_tuning(jb.FP64)
    traffic = committed_traffic(a.workload, mode, B)
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic,
            "algorithmic_bytes_per_launch": bytes_per_launch, "peak_source": peak_kind,
            "kernel_ms_per_launch": avg_launch_s * 1e3}

    # full solves (outside the timed region): reference schedule FP64 vs mixed block
    solves = {}
    if not a.no_solves:
        kmin, kmax, refdim, maxiter = DALGINFO[a.workload]
        kw = dict(maxiter=maxiter, krymin=kmin, krymax=kmax, nroots=nroots, refdim=refdim,
                  restol=1e-8)
        r64 = sp.davidson(**kw)
        rmx = sp.davidson(precision=jb.MIXED, **kw)
        solves = {"fp64_solve_s": r64.stats.total_seconds, "fp64_converged": r64.converged,
                  "mixed_solve_s": rmx.stats.total_seconds, "mixed_converged": rmx.converged,
                  "fp64_sigma_vectors": r64.stats.sigma_vectors,
                  "mixed_sigma_vectors": [rmx.stats.fp32_sigma_vectors,
                                          rmx.stats.sigma_vectors - rmx.stats.fp32_sigma_vectors],
                  "davidson": dict(krymin=kmin, krymax=kmax, refdim=refdim, maxiter=maxiter),
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
    out = {"metric": METRIC, "value": value, "unit": "Gdet/s", "n_gpus": world,
           "steps": a.steps, "warmup": a.warmup, "ms_per_step": tot_ms / a.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded integrals, random CI vectors)",
           "config": {"workload": a.workload, "ndets": N, "vectors_per_step": nvec,
                      "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                      "l2": "flushed (256 MiB write) before every step",
                      "sigma_plan": sigma_plan_desc(mode, nt, R, B)},
           "roofline": roof, "cpu_baseline": cpu,
           "e2e": {"value": e2e, "unit": "Gdet/s", "h2d_bytes_per_step": nvec * N * 8,
                   "d2h_bytes_per_step": nvec * N * 8},
           "gpu_launches": a.steps * nvec * SIGMA_KERNELS[mode],
           "clocks": clk,
           "fp32_sigma_gdet_s": value32,
           "solves": solves}
    tp = committed_tensor_pipe(a.workload)
    if tp:
        out["tensor_pipe"] = tp
    if rank == 0:
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def serve_subspace(nroots):
    """&dalginfo krymin, krymax of a serving request: a basis of 4 to 16 for
    one or two roots, 8 to 24 for three or four.  Collapsing to only the
    roots' own Ritz vectors (krymin = nroots) loses the thick restart: a
    4-root CAS(12,12) solve takes 2289 iterations at 4 / 16 and 767 at
    8 / 24."""
    return (4, 16) if nroots <= 2 else (8, 24)


def run_serve(a):
    """Serving stream: CAS(m,m) solves, m uniform in {6, 8, 10, 12}, 1-4 roots,
    chained in 32-step geometry scans (base integrals seed 105 + scan, each
    step adds N(0, 1e-3) perturbations, seed 105000 + request), each step
    warm-started from the previous one of its scan.  Three arms:
      plain    -- each request solved alone through the single-solve API
                  (FP64, reference Davidson schedule, cold start; string
                  spaces built once per size), on the first --serve-sample
                  steps of every scan;
      one_slot -- the server with one slot: requests back to back, warm
                  starts, cached spaces, the chosen precision;
      batched  -- the server with --slots slots, Poisson arrivals at 1.5x
                  the one_slot rate."""
    import numpy as np

    import jayci_b200 as jb
    from jayci_b200.synth import make_integrals, perturb

    rng = np.random.default_rng(105)
    nscan = max(1, a.serve // 32)
    sizes = rng.choice([6, 8, 10, 12], size=nscan)
    scans = []
    for sc in range(nscan):
        m = int(sizes[sc])
        ints = make_integrals(m, m, 105 + sc)
        steps = []
        for st in range(32):
            if st:
                ints = perturb(ints, 105000 + sc * 32 + st)
            m1, m2 = ints.packed()
            steps.append(dict(scan=sc, step=st, m=m, nroots=int(rng.integers(1, 5)),
                              m1=m1, m2=m2, e_nuc=ints.e_nuc))
        scans.append(steps)
    # arrival order: a random interleaving that keeps each scan's step order
    pos = [0] * nscan
    seq = []
    while len(seq) < nscan * 32:
        sc = int(rng.choice([s for s in range(nscan) if pos[s] < 32]))
        seq.append(scans[sc][pos[sc]])
        pos[sc] += 1
    N = len(seq)
    prec = jb.MIXED if a.serve_mixed else jb.FP64
    kw = dict(refdim=8, restol=1e-8, maxiter=5000, precision=prec)

    def submit(srv, r, warm):
        kmin, kmax = serve_subspace(r["nroots"])
        return srv.submit((r["m"], r["m"], 0, 0, r["m"], 0, 0), r["m1"], r["m2"], r["e_nuc"],
                          0.0, nroots=r["nroots"], warm_from=warm, krymin=kmin, krymax=kmax,
                          **kw)

    def by_size(rows):
        out = {}
        for m in sorted(set(x[0] for x in rows)):
            sel = [x for x in rows if x[0] == m]
            out[f"cas{m}"] = dict(n=len(sel),
                                  solve_ms=float(np.mean([x[1] for x in sel]) * 1e3),
                                  iterations=float(np.mean([x[2] for x in sel])),
                                  sigma_ms=float(np.mean([x[3] for x in sel]) * 1e3))
        return out

    # warm-up: one solve per size class (autotuning, table build)
    srv = jb.Server(slots=1)
    for m in sorted(set(int(x) for x in sizes)):
        r = next(x for x in seq if x["m"] == m)
        srv.wait(submit(srv, r, -1))
    srv.close()

    # plain single solves on a bounded sample of scan steps
    spaces = {}
    sample = [x for x in seq if x["step"] < a.serve_sample]
    rows = []
    t0 = time.perf_counter()
    for r in sample:
        m = r["m"]
        if m not in spaces:
            spaces[m] = jb.Space(m, m)
        sp = spaces[m]
        ts = time.perf_counter()
        sp.set_integrals(r["m1"], r["m2"], r["e_nuc"], 0.0)
        kmin, kmax = serve_subspace(r["nroots"])
        res = sp.davidson(maxiter=5000, krymin=kmin, krymax=kmax, nroots=r["nroots"], refdim=8,
                          restol=1e-8, want_vectors=False)
        rows.append((m, time.perf_counter() - ts, res.stats.iterations,
                     res.stats.sigma_seconds))
    t1 = time.perf_counter()
    for sp in spaces.values():
        sp.close()
    plain = dict(solves_per_s=len(sample) / (t1 - t0), requests=len(sample),
                 sample=f"steps < {a.serve_sample} of every scan",
                 p50_ms=float(np.percentile([x[1] for x in rows], 50) * 1e3),
                 p99_ms=float(np.percentile([x[1] for x in rows], 99) * 1e3),
                 by_size=by_size(rows))

    def play(slots, rate):
        srv = jb.Server(slots=slots)
        last = {}
        tickets = []
        t0 = time.perf_counter()
        t_next = t0
        arr = np.random.default_rng(7)
        for r in seq:
            if rate:
                t_next += arr.exponential(1.0 / rate)
                d = t_next - time.perf_counter()
                if d > 0:
                    time.sleep(d)
            t = submit(srv, r, last.get(r["scan"], -1))
            last[r["scan"]] = t
            tickets.append(t)
            if not rate:
                srv.wait(t)
        res = [srv.wait(t) for t in tickets]
        t1 = time.perf_counter()
        srv.close()
        lat = np.array([x.queue_seconds + x.solve_seconds for x in res])
        ok = all(x.status == 0 and x.converged for x in res)
        rows = [(r["m"], x.solve_seconds, x.iterations, x.sigma_seconds)
                for r, x in zip(seq, res)]
        failed = [dict(scan=r["scan"], step=r["step"], cas=r["m"], nroots=r["nroots"],
                       iterations=x.iterations, status=x.status, warm=x.warm_started)
                  for r, x in zip(seq, res) if not (x.status == 0 and x.converged)]
        return dict(solves_per_s=N / (t1 - t0), wall_s=t1 - t0,
                    p50_ms=float(np.percentile(lat, 50) * 1e3),
                    p99_ms=float(np.percentile(lat, 99) * 1e3),
                    warm_started=int(sum(x.warm_started for x in res)), all_converged=ok,
                    not_converged=failed[:8], by_size=by_size(rows))

    one = play(1, 0.0)
    rate = 1.5 * one["solves_per_s"]
    batched = play(a.slots, rate)
    out = {"metric": "served CI solves/s (CAS(6-12) geometry-scan stream)",
           "value": batched["solves_per_s"], "unit": "solves/s", "n_gpus": 1,
           "requests": N, "higher_is_better": True,
           "dtype": "f64" if not a.serve_mixed else "mixed fp32->f64",
           "data": "synthetic (seeded integrals, 32-step scans)",
           "config": {"workload": "serving stream", "sizes": [6, 8, 10, 12], "scans": nscan,
                      "slots": a.slots, "arrival_rate_per_s": rate, "restol": 1e-8},
           "plain": plain, "one_slot": one, "batched": batched,
           "speedup_vs_plain": batched["solves_per_s"] / plain["solves_per_s"],
           "speedup_vs_one_slot": batched["solves_per_s"] / one["solves_per_s"]}
    print(json.dumps(out))
    return 0


def run_profile(a):
    """Small fixed workload for ncu: build the space, let the sigma autotuner
    pick its plan outside the profiled range, then run `--steps` sigma
    applications of one vector inside the NVTX range "profile" (capture with
    ncu --nvtx --nvtx-include "profile/")."""
    import torch

    import jayci_b200 as jb
    from jayci_b200.synth import workload_integrals

    (geo, _, _, _) = WORKLOADS[a.workload]
    ints = workload_integrals(a.workload)
    m1, m2 = ints.packed()
    sp = jb.Space(*geo)
    sp.set_integrals(m1, m2, ints.e_nuc, ints.e_fc)
    prec = jb.FP32 if a.profile_fp32 else jb.FP64
    st = torch.cuda.Stream()
    dt = torch.float32 if a.profile_fp32 else torch.float64
    with torch.cuda.stream(st):
        v = torch.randn(sp.ndets, dtype=dt, device="cuda")
        o = torch.empty_like(v)
        sp.sigma_device(v.data_ptr(), o.data_ptr(), 1, sp.ndets, prec, st.cuda_stream)
        torch.cuda.synchronize()
        if a.plan:
            sp.set_sigma_plan(prec, *(int(x) for x in a.plan.split(",")))
            sp.sigma_device(v.data_ptr(), o.data_ptr(), 1, sp.ndets, prec, st.cuda_stream)
            torch.cuda.synchronize()
        if a.profile_davidson:
            # a few Davidson iterations: subspace products (k_gram), residuals,
            # preconditioner and sigma as they run inside a solve
            kmin, kmax, refdim, _ = DALGINFO[a.workload]
            torch.cuda.nvtx.range_push("profile")
            sp.davidson(maxiter=a.steps, krymin=kmin, krymax=kmax, nroots=1, refdim=refdim,
                        restol=1e-8, want_vectors=False)
            torch.cuda.synchronize()
            torch.cuda.nvtx.range_pop()
        else:
            torch.cuda.nvtx.range_push("profile")
            for _ in range(a.steps):
                sp.sigma_device(v.data_ptr(), o.data_ptr(), 1, sp.ndets, prec, st.cuda_stream)
            torch.cuda.synchronize()
            torch.cuda.nvtx.range_pop()
    print(json.dumps({"profile": a.workload, "ndets": sp.ndets,
                      "plan": sp.sigma_tuning(prec)}))
    return 0


def main():
    # the reference's sigma kernel runs its OpenMP loop with schedule(runtime):
    # every CPU timing here uses all host threads and the same schedule
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    os.environ.setdefault("OMP_SCHEDULE", "dynamic,64")
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
    ap.add_argument("--ref-step-frac", type=float, default=0.25,
                    help="fraction of rows per step of --impl reference")
    ap.add_argument("--serve", type=int, default=0,
                    help="run the serving stream with this many requests instead")
    ap.add_argument("--slots", type=int, default=8)
    ap.add_argument("--serve-mixed", action="store_true")
    ap.add_argument("--serve-sample", type=int, default=2,
                    help="scan steps per scan solved by the plain arm")
    ap.add_argument("--profile", action="store_true",
                    help="run --steps sigma calls in an NVTX range for ncu")
    ap.add_argument("--profile-fp32", action="store_true")
    ap.add_argument("--profile-davidson", action="store_true",
                    help="with --profile: --steps Davidson iterations instead of sigma calls")
    ap.add_argument("--plan", default="",
                    help="with --profile: force the sigma plan MODE,THREADS,ROWS,BATCH "
                         "(jci_sigma_set_plan) instead of the autotuned one")
    a = ap.parse_args()
    if a.profile:
        return run_profile(a)
    if a.warmup < 3:
        a.warmup = 3
    if a.serve:
        return run_serve(a)
    if a.impl == "reference":
        return run_reference(a)
    return run_gpu(a)


if __name__ == "__main__":
    sys.exit(main())
