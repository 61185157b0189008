#!/usr/bin/env python
"""bench.py -- sigma-build throughput of the determinant-CI hot path.

Workload (default): FCI(16e,16o), 12 870 x 12 870 = 165 636 900
determinants, 1 root, seeded synthetic integrals (rank 16, seed 104): the
largest configuration of the metric that one GPU holds.  A step is one
sigma = H c build of one vector (the root count) in FP64 with every input
resident in HBM.  The vectors (1.33 GB) are far larger than the 126 MB L2;
a 256 MiB write still flushes it before every step.

value  = determinants x vectors / sigma time  (Gdet/s, all ranks)
e2e    = the same through the public C ABI (jci_sigma) from pinned host
         buffers, host->device copy of the input vector and device->host
         copy of the sigma vector inside every timed step
Extra keys (outside the timed region): the FP32 sigma rate; the one-time
setup costs (host string tables, device tables, the sigma autotuner's
first call); and the full Davidson solve pair of FCI(14e,14o) with two
frozen-core orbitals, 4 roots -- the plain FP64 reference schedule against
the mixed FP32 -> FP64 schedule, each after an untimed warm-up solve.

--impl reference times the reference's own CPU code (oracle/_ref, the
reference's mpi_source compiled unchanged against a single-process GA/MPI
stand-in) on the same workload with every usable host thread: each step is
the reference's sigma (the diagonal term, pdavidson.c:2105, then
compute_cblock_Hfastest, pdavidson.c:1296) on one contiguous block of rows.
ms_per_step is the time of that block; the rows, their fraction of a full
sigma, the reference's fixed cost per call and the full-sigma time
extrapolated from the two are separate keys.  Multi-GPU runs (torchrun)
are replicas: every rank builds the same workload independently (weak
scaling); no data-path collective exists.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
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
# the solve pair reported beside each sigma workload
SOLVES_OF = {"fci16_16": "fci14_14_fc2", "fci14_14_fc2": "fci14_14_fc2",
             "fci12_12": "fci12_12", "cas10_10": "cas10_10"}
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


def sigma_plan_desc(mode, nt, R, B, ms=None):
    streams, groups = mode in (3, 4), mode in (6, 7)
    d = {"mode": mode, "name": PLAN_NAMES[mode],
         ("alpha_pass_threads" if streams else "beta_singles_threads" if groups
          else "row_kernel_threads"): nt}
    if groups and nt == 0:
        d["beta_singles"] = "hole-string products"
    elif groups:
        d["beta_singles"] = "row stream on C^T"
    if mode == 0:
        d["staged_rows"] = R
    elif mode in (4, 5, 7):
        d["product_engine"] = (f"tcgen05 3xTF32, {R}-column chunks" if R in (32, 64) else
                               f"{R} column threads")
    else:
        d["product_ctas_per_sm"] = R % 16
        d["product_panel"] = ("whole alpha row per CTA, compact (the entries the gather reads)"
                              if R >= 64 else
                              "one per alpha row, shared by all CTAs (L2)" if R >= 32 else
                              "256-column blocks" if R >= 16 else "whole alpha row per CTA")
    if groups:
        d["group_kernel"] = (f"{B} column(s) per thread" if B <= 2 else
                             f"targets split over 4 warps, {5 - B} column(s) per lane" if B <= 4
                             else "hole-string pair products, " +
                             {5: "widest column blocks (1 GiB)", 6: "64-column blocks",
                              7: "widest column blocks (4 GiB)"}[B])
    else:
        d["beta_pass_threads" if streams else "rows_per_cta"] = B
    if ms is not None:
        d["autotuner_ms_per_vector"] = ms
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


def profile_key(mode, R, B, nt=None):
    """Key of a sigma plan in the committed traffic summaries: the mode; for
    the string-group plans (6, 7) also the group kernel variant ("7:3"); for
    the panel products (1, 3, 6) a ":blk" suffix when the panel is cut into
    column blocks (16 <= R < 32), ":row" when one panel per alpha row is
    shared by all CTAs (32 <= R < 64), ":cp" for the compact panel (R >= 64);
    ":hs" after the group variant when the beta singles run through hole
    strings (nt = 0)."""
    key = f"{mode}:{B}" if mode in (6, 7) else str(mode)
    if mode in (6, 7) and nt == 0:
        key += ":hs"
    if mode in (1, 3, 6) and R >= 64:
        key += ":cp"
    elif mode in (1, 3, 6) and R >= 32:
        key += ":row"
    elif mode in (1, 3, 6) and R >= 16:
        key += ":blk"
    return key


def committed_profile(workload, mode, B, R=0, nt=None):
    """Per-launch figures of sigma plan (mode, nt, R, B) on `workload` from
    the committed ncu summary (profiles/sigma_<workload>_traffic.json), or
    None when that plan was not captured (keys: profile_key)."""
    key = profile_key(mode, R, B, nt)
    p = os.path.join(ROOT, "profiles", f"sigma_{workload}_traffic.json")
    if os.path.exists(p):
        try:
            return json.load(open(p)).get("plans", {}).get(key)
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


# ---- the reference's own sigma on the host cores ---------------------------

def host_threads(ndets, nvec):
    """Host threads for the reference's sigma: every core, bounded by memory
    and by the reference's own size arithmetic.  compute_hij_eosp keeps a
    private full-length sigma buffer per OpenMP thread (pdavidson.c:1930-2078),
    nvec x ndets doubles each, beside about 5 x that of shared arrays (V, C,
    D, W and the row buffers).  It allocates them as one block whose element
    count nvec x ndets x threads is an int (pdavidson.c:1946, allocate_mem.c:58):
    past 2^31 - 1 the product wraps, the allocation fails and the reference
    crashes, so FCI(16e,16o) runs on at most 12 threads."""
    cores = min(os.cpu_count() or 1, max(1, (2 ** 31 - 1) // max(1, nvec * ndets)))
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        return cores
    try:  # a cgroup limit below the machine's memory
        lim = open("/sys/fs/cgroup/memory.max").read().strip()
        if lim != "max":
            avail = min(avail, int(lim))
    except Exception:
        pass
    per = 8.0 * nvec * ndets
    fit = int((0.8 * avail - 6 * per) // per)
    return max(1, min(cores, fit))


class RefSigma:
    """The reference's sigma (oracle/_ref) prepared once on one workload;
    step(rows) times one contiguous row block at a rotating position."""

    def __init__(self, name, nvec):
        import ctypes

        import numpy as np

        from jayci_b200.synth import workload_integrals
        from oracle.oracle import RefSpace, _ptr
        (e, o, nfc), _, _, _ = WORKLOADS[name]
        ints = workload_integrals(name)
        self.m1, self.m2 = ints.packed()
        self.ref = RefSpace(e, o, nfc)
        self.ndets, self.nvec = self.ref.ndets, nvec
        L = self.ref.lib()
        # the thread count must reach the OpenMP runtime itself: it read
        # OMP_NUM_THREADS when it started, possibly before this process set it
        L.ref_set_threads(int(os.environ.get("OMP_NUM_THREADS", "0")))
        self.threads = L.ref_get_threads()
        L.ref_sigma_step_timed.restype = ctypes.c_double
        L.ref_sigma_step_timed.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        V = np.random.default_rng(0).standard_normal((nvec, self.ndets))
        L.ref_sigma_prepare(_ptr(self.m1), _ptr(self.m2), nvec, _ptr(V))
        del V
        self.L, self.k = L, 0

    def step(self, rows):
        import ctypes
        rows = max(1, min(int(rows), self.ndets))
        # block positions walk through the determinant list (golden ratio)
        frac = (self.k * 0.6180339887498949) % 1.0
        self.k += 1
        r0 = min(self.ndets - rows, int(frac * (self.ndets - rows + 1)))
        d = ctypes.c_double()
        t = self.L.ref_sigma_step_timed(r0, rows, ctypes.byref(d))
        return t, rows

    def close(self):
        self.L.ref_sigma_release()


def calibrate(rs, small, large):
    """The reference's fixed cost per call (buffer setup, whole-vector gets
    and reductions) and its cost per row, from one block of each size after
    an untimed call of the small one (the first call also pays the page
    faults of the reference's full-length buffers).  When the two times do
    not separate (noise larger than the rows' cost), the per-row cost is
    bounded from above by the large block's time per row and the fixed cost
    taken as zero, so a sample sized from them never runs long."""
    rs.step(small)
    t1, r1 = rs.step(small)
    t2, r2 = rs.step(large)
    per_row = (t2 - t1) / max(r2 - r1, 1)
    if not (t2 > 1.2 * t1 and per_row > 0):
        return 0.0, t2 / r2
    return max(t1 - per_row * r1, 0.0), per_row


def sample_rows(fixed, per_row, seconds, large, ndets):
    """Rows of a sample of about `seconds` of reference work: at least 2000,
    at most 64 times the largest calibrated block, at most every row."""
    rows = (seconds - fixed) / per_row if seconds > fixed else 2000
    return int(max(2000, min(ndets, 64 * large, rows)))


def calib_sizes(ndets):
    """Calibration blocks: 2000 rows and about 0.1% of the rows (at least
    20000), so the large one is well above the fixed cost at every size."""
    return 2000, max(20000, ndets // 1000)


def run_reference(a):
    rank = env_int("RANK", 0)
    if rank != 0:
        return 0
    from oracle.oracle import ref_available
    if not ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference build absent"}))
        return 0
    (geo, nroots, s, d) = WORKLOADS[a.workload]
    import math

    from jayci_b200.synth import WORKLOADS as W
    w = W[a.workload]
    ndets = math.comb(w["n"], w["k"]) ** 2
    threads = host_threads(ndets, nroots)
    os.environ["OMP_NUM_THREADS"] = str(threads)
    os.environ.setdefault("OMP_SCHEDULE", "dynamic,64")
    rs = RefSigma(a.workload, nroots)
    # warm-up steps: the first three calibrate the fixed cost and the
    # per-row cost; every timed step then runs the block that fits its share
    small, large = calib_sizes(rs.ndets)
    fixed, per_row = calibrate(rs, small, large)
    for _ in range(max(0, a.warmup - 3)):
        rs.step(small)
    budget = a.ref_seconds / max(a.steps, 1)
    rows = sample_rows(fixed, per_row, budget, large, rs.ndets)
    times, done = [], 0
    for _ in range(a.steps):
        t, r = rs.step(rows)
        times.append(t)
        done += r
    rs.close()
    threads = rs.threads
    tot = sum(times)
    value = done * nroots / tot / 1e9
    sample = (f"{a.steps} blocks of {rows} contiguous rows ({rows / ndets:.4%} of the "
              f"determinants each), at rotating positions")
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Gdet/s",
           "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
           "ms_per_step": tot / a.steps * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded integrals)",
           "config": {"workload": a.workload, "ndets": ndets, "vectors_per_step": nroots,
                      "rows_per_step": rows, "row_fraction_per_step": rows / ndets,
                      "sample": sample},
           "reference_cost_model": {
               "fixed_s_per_call": fixed, "s_per_row": per_row,
               "extrapolated_full_sigma_s": fixed + per_row * ndets,
               "note": f"fixed cost and per-row cost from two calibration blocks "
                       f"({small} and {large} rows, after an untimed call); the "
                       f"full-sigma time is an extrapolation"},
           "cpu_baseline": {"value": value, "unit": "Gdet/s", "cores": threads,
                            "kind": "reference", "sample": sample},
           "e2e": {"value": value, "unit": "Gdet/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def cpu_baseline(name, nvec, seconds):
    """The reference's sigma on one row block of about `seconds` of host
    work (after two calibration blocks), as Gdet/s of the rows it ran."""
    from oracle.oracle import ref_available
    if not ref_available():
        return None
    import math

    from jayci_b200.synth import WORKLOADS as W
    w = W[name]
    ndets = math.comb(w["n"], w["k"]) ** 2
    threads = host_threads(ndets, nvec)
    os.environ["OMP_NUM_THREADS"] = str(threads)
    rs = RefSigma(name, nvec)
    small, large = calib_sizes(rs.ndets)
    fixed, per_row = calibrate(rs, small, large)
    rows = sample_rows(fixed, per_row, seconds, large, rs.ndets)
    t, rows = rs.step(rows)
    rs.close()
    threads = rs.threads
    return {"value": rows * nvec / t / 1e9, "unit": "Gdet/s", "cores": threads,
            "kind": "reference",
            "sample": f"reference sigma (diagonal term + compute_cblock_Hfastest), {nvec} "
                      f"vector(s), one block of {rows} contiguous rows "
                      f"({rows / ndets:.4%} of the determinants) in {t:.1f} s, "
                      f"OMP_SCHEDULE={os.environ.get('OMP_SCHEDULE')}",
            "fixed_s_per_call": fixed, "extrapolated_full_sigma_s": fixed + per_row * ndets}


# ---- the GPU arm -----------------------------------------------------------

def solve_pair(jb, name, world):
    """The plain FP64 reference schedule against the mixed FP32 -> FP64
    schedule on workload `name`, each timed after an untimed warm-up solve
    of a few iterations (autotuning, graph capture, buffer allocation)."""
    import numpy as np

    from jayci_b200.synth import workload_integrals
    (geo, nroots, _, _) = WORKLOADS[name]
    ints = workload_integrals(name)
    m1, m2 = ints.packed()
    t0 = time.perf_counter()
    sp = jb.Space(*geo)
    sp.set_integrals(m1, m2, ints.e_nuc, ints.e_fc)
    setup = time.perf_counter() - t0
    kmin, kmax, refdim, maxiter = DALGINFO[name]
    kw = dict(krymin=kmin, krymax=kmax, nroots=nroots, refdim=refdim, restol=1e-8)
    first = {}
    for p, key in ((jb.FP64, "fp64"), (jb.MIXED, "mixed")):
        t0 = time.perf_counter()
        sp.davidson(maxiter=kmax - kmin + 2, precision=p, want_vectors=False, **kw)
        first[key] = time.perf_counter() - t0
    r64 = sp.davidson(maxiter=maxiter, **kw)
    rmx = sp.davidson(maxiter=maxiter, precision=jb.MIXED, **kw)
    out = {"workload": name, "ndets": sp.ndets, "nroots": nroots,
           "davidson": dict(krymin=kmin, krymax=kmax, refdim=refdim, maxiter=maxiter,
                            restol=1e-8),
           "fp64_solve_s": r64.stats.total_seconds, "fp64_converged": r64.converged,
           "mixed_solve_s": rmx.stats.total_seconds, "mixed_converged": rmx.converged,
           "fp64_sigma_vectors": r64.stats.sigma_vectors,
           "mixed_sigma_vectors": {"fp32": rmx.stats.fp32_sigma_vectors,
                                   "fp64": rmx.stats.sigma_vectors -
                                   rmx.stats.fp32_sigma_vectors},
           "fp64_sigma_s": r64.stats.sigma_seconds, "mixed_sigma_s": rmx.stats.sigma_seconds,
           "fp64_solves_per_s": world / r64.stats.total_seconds,
           "mixed_solves_per_s": world / rmx.stats.total_seconds,
           "mixed_vs_fp64_max_abs_dE": float(np.abs(rmx.energies - r64.energies).max()),
           "energies_fp64": [float(x) for x in r64.energies],
           "mixed_speedup": r64.stats.total_seconds / rmx.stats.total_seconds,
           "sigma_plans": {"fp64": sigma_plan_desc(*sp.sigma_tuning(jb.FP64)[:4]),
                           "fp32": sigma_plan_desc(*sp.sigma_tuning(jb.FP32)[:4])},
           "first_call_s": {"space_and_tables": setup,
                            "warmup_solve_fp64": first["fp64"],
                            "warmup_solve_mixed": first["mixed"]}}
    sp.close()
    return out


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
    setup = {}
    t0 = time.perf_counter()
    sp = jb.Space(*geo)
    setup["space_tables_host_s"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    sp.set_integrals(m1, m2, ints.e_nuc, ints.e_fc)
    torch.cuda.synchronize()
    setup["set_integrals_s"] = time.perf_counter() - t0
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

    # first sigma call of each precision: the autotuner times the plans
    for prec, v, o, key in ((jb.FP64, V, S, "autotune_fp64_s"), (jb.FP32, V32, S32,
                                                                  "autotune_fp32_s")):
        t0 = time.perf_counter()
        with torch.cuda.stream(stream):
            sp.sigma_device(v[0].data_ptr(), o[0].data_ptr(), 1, N, prec, sh)
        torch.cuda.synchronize()
        setup[key] = time.perf_counter() - t0
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
    del V32, S32

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
    e2e_s = 0.0
    for _ in range(a.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rc = jb.lib().jci_sigma(sp.h, nvec, hvn.ctypes.data, hsn.ctypes.data, jb.FP64)
        e2e_s += time.perf_counter() - t0
        if rc:
            raise jb.JciError(rc, "jci_sigma")
    e2e_s, = max_over_ranks(dist, [e2e_s], "cuda")
    e2e = replica_rate(world, N * nvec * a.steps, e2e_s) / 1e9
    del hv, hs, hvn, hsn

    # roofline of the sigma kernel (row-stream algorithmic bytes per vector)
    w = 8
    bytes_per_launch = w * N * (2 + s_exc + d_exc)
    avg_launch_s = statistics.mean(launches) / 1e3
    peak, peak_kind = measured_peaks()
    achieved = bytes_per_launch / avg_launch_s / 1e9
    mode, nt, R, B, tms = sp.sigma_tuning(jb.FP64)
    tune32 = sp.sigma_tuning(jb.FP32)
    prof = committed_profile(a.workload, mode, B, R, nt) or {}
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": prof.get("dram_bytes_per_launch"),
            "algorithmic_bytes_per_launch": bytes_per_launch, "peak_source": peak_kind,
            "kernel_ms_per_launch": avg_launch_s * 1e3,
            "model": "row-stream bytes B = 8 N (2 + s + d) per vector: each sigma row reads "
                     "its own C row and one C row per alpha single and double"}
    for k in ("dram_gb_per_s", "l2_bytes_per_launch", "dominant_kernel", "limiter", "summary"):
        if k in prof:
            roof[k] = prof[k]
    sp.close()
    del V, S
    torch.cuda.empty_cache()

    solves = {}
    if not a.no_solves:
        solves = solve_pair(jb, SOLVES_OF[a.workload], world)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        cpu = cpu_baseline(a.workload, nvec, a.cpu_seconds)
    out = {"metric": METRIC, "value": value, "unit": "Gdet/s", "n_gpus": world,
           "steps": a.steps, "warmup": a.warmup, "ms_per_step": tot_ms / a.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded integrals, random CI vectors)",
           "config": {"workload": a.workload, "ndets": N, "vectors_per_step": nvec,
                      "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                      "l2": "inputs (8 bytes x ndets per vector) larger than L2; a 256 MiB "
                            "write also flushes it before every step",
                      "sigma_plan": sigma_plan_desc(mode, nt, R, B, tms),
                      "sigma_plan_fp32": sigma_plan_desc(*tune32)},
           "roofline": roof, "cpu_baseline": cpu,
           "e2e": {"value": e2e, "unit": "Gdet/s", "h2d_bytes_per_step": nvec * N * 8,
                   "d2h_bytes_per_step": nvec * N * 8},
           "gpu_launches": a.steps * nvec * SIGMA_KERNELS[mode],
           "clocks": clk,
           "fp32_sigma_gdet_s": value32,
           "setup_s": setup,
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

    def by_size(rows, lat=None):
        """Per size class: solve time, iterations, sigma time (means) and,
        with lat (queue + solve seconds per row), latency p50 / p99."""
        out = {}
        for m in sorted(set(x[0] for x in rows)):
            idx = [i for i, x in enumerate(rows) if x[0] == m]
            sel = [rows[i] for i in idx]
            d = dict(n=len(sel), solve_ms=float(np.mean([x[1] for x in sel]) * 1e3),
                     iterations=float(np.mean([x[2] for x in sel])),
                     sigma_ms=float(np.mean([x[3] for x in sel]) * 1e3))
            lt = [lat[i] for i in idx] if lat is not None else [x[1] for x in sel]
            d["p50_ms"] = float(np.percentile(lt, 50) * 1e3)
            d["p99_ms"] = float(np.percentile(lt, 99) * 1e3)
            out[f"cas{m}"] = d
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
                    not_converged=failed[:8], by_size=by_size(rows, list(lat)))

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
    # every CPU timing here uses the same schedule
    os.environ.setdefault("OMP_SCHEDULE", "dynamic,64")
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="jci", choices=["jci", "reference"])
    ap.add_argument("--workload", default="fci16_16", choices=sorted(WORKLOADS))
    ap.add_argument("--no-solves", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="host seconds of the CPU-baseline sample")
    ap.add_argument("--ref-seconds", type=float, default=120.0,
                    help="host seconds of all timed steps of --impl reference together")
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
