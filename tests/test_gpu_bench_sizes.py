"""Parity at the sizes the bench times: FCI(12e,12o), FCI(14e,14o) with two
frozen-core orbitals, and FCI(16e,16o).

The fixtures (tests/golden/bench_*.npz, made by make_golden.py) hold samples, because full
vectors do not fit in the repository:

* fci12_12: the reference's own sigma (compute_cblock_Hfastest over every
  row, pdavidson.c:1296, plus the diagonal term, :2105) of a seeded vector,
  at 4098 sampled rows, with its norm and four seeded projections; and the
  reference's own pdavidson (pdavidson.c:39) energies and result vectors
  (largest components and seeded projections) for 3 roots with krymin 6,
  krymax 24, refdim 12, restol 1e-8.
* fci14_14_fc2, fci16_16: sigma at 4098 sampled rows from the oracle's row
  gather, which test_oracle_rows_match_reference_sigma pins to the
  reference's own sigma.

Input vectors are the counter-hash vectors of tests/golden/seeded.py.  Bars:
sigma FP64 1e-12 and FP32 2e-6 of the largest sampled |sigma|; FP64
energies 1e-10 Eh; mixed energies 1e-8 Eh; result vectors within what
|<c_ref|c>| > 1 - 1e-9 implies (||c - c_ref|| < 4.5e-5) on every stored
component and projection.
"""
import os
import sys

import numpy as np
import pytest

import jayci_b200 as jb
from jayci_b200.synth import workload_integrals

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from seeded import hash_vector  # noqa: E402

GOLDEN = os.path.join(HERE, "golden")
VEC_DIST = float(np.sqrt(2e-9))  # ||c - c_ref|| implied by |<c_ref|c>| > 1 - 1e-9


def _fixture(name):
    return np.load(os.path.join(GOLDEN, "bench_" + name + ".npz"))


def _space(name):
    g = _fixture(name)
    ints = workload_integrals(name)
    m1, m2 = ints.packed()
    assert m1.sum() == pytest.approx(float(g["m1_sum"]), rel=1e-14, abs=1e-14)
    assert m2.sum() == pytest.approx(float(g["m2_sum"]), rel=1e-14, abs=1e-14)
    s = jb.Space(*(int(x) for x in g["general"]))
    s.set_integrals(m1, m2, ints.e_nuc, ints.e_fc)
    assert s.ndets == int(g["ndets"])
    return s, g, m1, m2, ints


def _gpu_sigma(s, v, prec):
    import torch
    dt = torch.float64 if prec == jb.FP64 else torch.float32
    x = torch.from_numpy(v).to(device="cuda", dtype=dt)
    y = torch.full_like(x, float("nan"))
    s.sigma_device(x.data_ptr(), y.data_ptr(), 1, s.ndets, prec, 0)
    torch.cuda.synchronize()
    return y


def test_oracle_rows_match_reference_sigma():
    """CPU: the oracle's row gather equals the reference's own sigma on the
    sampled FCI(12e,12o) rows (this pins the oracle that produced the
    larger fixtures)."""
    from oracle.oracle import OracleSpace
    g = _fixture("fci12_12")
    assert str(g["source"]) == "reference"
    ints = workload_integrals("fci12_12")
    m1, m2 = ints.packed()
    o = OracleSpace(6, 6, 12)
    v = hash_vector(o.ndets, int(g["sigma_seed"]))
    got = o.sigma_rows(m1, m2, v, g["rows"])
    ref = g["sigma_rows"]
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_oracle_rows_reproduce_fixture_fci14():
    """CPU: the FCI(14e,14o) fixture is what the current oracle computes."""
    from oracle.oracle import OracleSpace
    g = _fixture("fci14_14_fc2")
    ints = workload_integrals("fci14_14_fc2")
    m1, m2 = ints.packed()
    o = OracleSpace(7, 7, 14)
    v = hash_vector(o.ndets, int(g["sigma_seed"]))
    rows = g["rows"][::16]
    got = o.sigma_rows(m1, m2, v, rows)
    assert np.array_equal(got, g["sigma_rows"][::16])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["fci12_12", "fci14_14_fc2", "fci16_16"])
@pytest.mark.parametrize("prec", [jb.FP64, jb.FP32])
def test_sigma_at_bench_sizes(name, prec):
    """The autotuned plan's sigma against the pinned rows."""
    s, g, _, _, _ = _space(name)
    v = hash_vector(s.ndets, int(g["sigma_seed"]))
    y = _gpu_sigma(s, v, prec)
    rows = g["rows"]
    import torch
    got = y[torch.from_numpy(rows).cuda()].double().cpu().numpy()
    ref = g["sigma_rows"]
    bar = (1e-12 if prec == jb.FP64 else 2e-6) * np.abs(ref).max()
    assert np.abs(got - ref).max() <= bar, (s.sigma_tuning(prec), np.abs(got - ref).max())
    if name == "fci12_12" and prec == jb.FP64:
        full = y.cpu().numpy()
        n2 = float(g["sigma_norm2"])
        assert abs(full @ full - n2) <= 1e-12 * n2
        for seed, p in zip(g["proj_seeds"], g["sigma_proj"]):
            w = hash_vector(s.ndets, int(seed))
            assert abs(w @ full - p) <= 1e-12 * np.linalg.norm(w) * np.sqrt(n2)
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [jb.FP64, jb.FP32])
def test_every_plan_at_fci12(prec):
    """Every admissible sigma plan at FCI(12e,12o) against the reference's
    own sigma rows."""
    import torch
    s, g, _, _, _ = _space("fci12_12")
    v = hash_vector(s.ndets, int(g["sigma_seed"]))
    rows = torch.from_numpy(g["rows"]).cuda()
    ref = g["sigma_rows"]
    bar = (1e-12 if prec == jb.FP64 else 2e-6) * np.abs(ref).max()
    plans = [(0, 256, 4, 1), (1, 256, 0, 2), (2, 256, 0, 1), (3, 256, 0, 256),
             (4, 256, 16, 256), (5, 256, 16, 2), (5, 256, 8, 1), (6, 512, 0, 2),
             (7, 512, 16, 1), (7, 512, 16, 2), (7, 512, 16, 3), (7, 512, 16, 4),
             (7, 512, 8, 3),
             # the column-blocked panel (product CTAs per SM + 16)
             (1, 256, 17, 2), (3, 256, 16, 256), (6, 512, 18, 2),
             # the same-spin doubles through hole strings (variants 5, 6)
             (6, 512, 0, 5), (6, 512, 2, 6), (7, 512, 16, 5),
             # the compact panel (+ 64) and the beta singles through hole strings (threads 0)
             (6, 512, 66, 5), (6, 0, 66, 5), (7, 0, 16, 3)]
    ran = 0
    for plan in plans:
        try:
            s.set_sigma_plan(prec, *plan)
        except jb.JciError:
            continue
        got = _gpu_sigma(s, v, prec)[rows].double().cpu().numpy()
        assert np.abs(got - ref).max() <= bar, (plan, np.abs(got - ref).max())
        ran += 1
    assert ran >= 13
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [jb.FP64, jb.FP32])
def test_blocked_panel_fci16(prec):
    """FCI(16e,16o): the product through the column-blocked panel against the
    pinned rows."""
    import torch
    s, g, _, _, _ = _space("fci16_16")
    s.set_sigma_plan(prec, 6, 512, 18, 2)
    v = hash_vector(s.ndets, int(g["sigma_seed"]))
    got = _gpu_sigma(s, v, prec)[torch.from_numpy(g["rows"]).cuda()].double().cpu().numpy()
    ref = g["sigma_rows"]
    bar = (1e-12 if prec == jb.FP64 else 2e-6) * np.abs(ref).max()
    assert np.abs(got - ref).max() <= bar
    s.close()


def _aligned(c, idx, val):
    """c restricted to idx with its sign matched to val."""
    x = c[idx]
    return x if x @ val >= 0 else -x


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [jb.FP64, jb.MIXED])
def test_fci12_davidson_matches_reference(precision):
    """3 roots of FCI(12e,12o) with the reference's schedule and the bench's
    &dalginfo, against the reference's own pdavidson."""
    from oracle.oracle import OracleSpace
    s, g, m1, m2, ints = _space("fci12_12")
    kmin, kmax, nroots, refdim = (int(x) for x in g["dav_opts"])
    r = s.davidson(maxiter=500, krymin=kmin, krymax=kmax, nroots=nroots, refdim=refdim,
                   restol=1e-8, precision=precision)
    assert r.converged
    bar = 1e-10 if precision == jb.FP64 else 1e-8
    assert np.abs(r.energies - g["energies"]).max() <= bar, r.energies - g["energies"]
    for k in range(nroots):
        c = r.civec[k]
        idx, val = g["civec_idx"][k], g["civec_val"][k]
        x = _aligned(c, idx, val)
        sgn = 1.0 if c[idx] @ val >= 0 else -1.0
        assert np.abs(x - val).max() <= VEC_DIST
        for seed, p in zip(g["proj_seeds"], g["civec_proj"][k]):
            w = hash_vector(s.ndets, int(seed))
            assert abs(sgn * (w @ c) - p) <= VEC_DIST * np.linalg.norm(w)
    # residual of the GPU's ground state on the sampled rows, with H applied
    # by the oracle (independent of the GPU sigma)
    o = OracleSpace(6, 6, 12)
    rows = g["rows"]
    c0 = r.civec[0]
    hc = o.sigma_rows(m1, m2, c0, rows)
    res = hc - (r.energies[0] - ints.e_nuc) * c0[rows]
    assert np.abs(res).max() <= 1e-7  # each element is bounded by ||r|| (restol 1e-8)
    s.close()
