"""CUDA sigma / Hdiag parity through the C ABI (needs a GPU).

Tolerances: FP64 sigma within 1e-12 of max|sigma| (rounding only: the
kernels gather each row in a different order than the reference's
upper-triangle accumulation); FP32 sigma (FP32 storage and accumulation)
within 2e-6 of max|sigma|.  Integer tables are checked bit-exactly in the
CPU tests.
"""
import glob
import os

import numpy as np
import pytest

import jayci_b200 as jb
from jayci_b200.synth import make_integrals, workload_integrals
from oracle.oracle import OracleSpace

pytestmark = pytest.mark.gpu

GOLDEN = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
                if not os.path.basename(p).startswith(("dyson_", "bench_")))
NAMES = [os.path.basename(p)[:-4] for p in GOLDEN]


def load(name):
    return np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))


def space_for(g):
    e, o, nfc, nd, na, nfv, x = (int(v) for v in g["general"])
    s = jb.Space(e, o, nfc, nd, na, nfv, x)
    s.set_integrals(g["m1"], g["m2"], float(g["e_nuc"]), 0.0)
    return s


@pytest.mark.parametrize("name", NAMES)
def test_hdiag(name):
    g = load(name)
    s = space_for(g)
    np.testing.assert_allclose(s.hdiag(), g["hdiag"], rtol=1e-13, atol=1e-12)


@pytest.mark.parametrize("name", NAMES)
def test_sigma_fp64(name):
    g = load(name)
    s = space_for(g)
    S = s.sigma(g["sigma_v"], jb.FP64)
    ref = g["sigma"]
    assert np.abs(S - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("name", NAMES)
def test_sigma_fp32(name):
    g = load(name)
    s = space_for(g)
    S = s.sigma(g["sigma_v"], jb.FP32)
    ref = g["sigma"]
    assert np.abs(S - ref).max() <= 2e-6 * np.abs(ref).max()


@pytest.mark.parametrize("gen", [
    (8, 10, 0, 2, 5, 0, 2),        # truncated, several groups: generic kernel
    (9, 10, 0, 0, 10, 0, 0),       # odd electrons, FCI kernel with Na != Nb
    (8, 12, 0, 1, 6, 0, 0),        # DOCC + ACTV + unused VIRT, xlevel 0 (one group)
    (10, 11, 0, 0, 11, 0, 0),      # FCI(10e,11o), 213 444 determinants
])
def test_sigma_against_oracle(gen):
    s = jb.Space(*gen)
    o = OracleSpace(s.na, s.nb, s.norb, gen[3], gen[4], gen[6])
    ints = make_integrals(s.norb, s.norb, 31)
    m1, m2 = ints.packed()
    s.set_integrals(m1, m2, ints.e_nuc, 0.0)
    V = np.random.default_rng(7).standard_normal((1, s.ndets))
    ref = o.sigma(m1, m2, V)
    got = s.sigma(V, jb.FP64)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    np.testing.assert_allclose(s.hdiag(), o.hdiag(m1, m2), rtol=1e-13, atol=1e-12)


@pytest.mark.parametrize("name", ["cas6_6", "cas7_7", "cas10_10"])
@pytest.mark.parametrize("plan", [(0, 128, 1, 1), (0, 256, 4, 1), (0, 512, 16, 1),
                                  (1, 128, 1, 1), (1, 256, 2, 2), (1, 128, 0, 4),
                                  (1, 1024, 4, 1), (1, 512, 1, 4), (2, 256, 1, 2),
                                  (2, 512, 2, 1), (2, 128, 0, 4), (3, 128, 1, 128),
                                  (3, 256, 0, 512), (3, 1024, 2, 256), (4, 256, 8, 256),
                                  (4, 128, 16, 512), (5, 256, 8, 2), (5, 128, 16, 1),
                                  (6, 128, 0, 1), (6, 256, 2, 2), (6, 128, 0, 3),
                                  (6, 256, 1, 4), (7, 128, 8, 2), (7, 256, 16, 1),
                                  (7, 256, 16, 3), (7, 128, 8, 4)])
@pytest.mark.parametrize("prec", [jb.FP64, jb.FP32])
def test_every_fci_plan(name, plan, prec):
    """Each launch plan the autotuner may pick gives the reference's sigma."""
    g = load(name)
    s = space_for(g)
    mode, nt, R, B = plan
    try:
        s.set_sigma_plan(prec, mode, nt, R, B)
    except jb.JciError:
        pytest.skip("plan not admissible for this size")
    S = s.sigma(g["sigma_v"], prec)
    ref = g["sigma"]
    tol = 1e-12 if prec == jb.FP64 else 2e-6
    assert np.abs(S - ref).max() <= tol * np.abs(ref).max()


@pytest.mark.parametrize("prec", [jb.FP64, jb.FP32])
def test_fused_product_and_groups_wide_rows(prec):
    """CAS(12e,14o), 3003 x 3003 strings: the fused product (16 strings per
    thread in the gather, 94 or 47 column chunks) and the string-group
    doubles (several column segments per row; the union split over warps
    in variants 3 and 4) give the sigma of the panel plan, whose parity with
    the reference is tested above."""
    s = jb.Space(12, 14)
    ints = make_integrals(14, 14, 5)
    m1, m2 = ints.packed()
    s.set_integrals(m1, m2, ints.e_nuc, 0.0)
    V = np.random.default_rng(11).standard_normal((1, s.ndets))
    s.set_sigma_plan(prec, 3, 256, 0, 256)
    ref = s.sigma(V, prec)
    tol = 1e-12 if prec == jb.FP64 else 5e-6  # two FP32 sums in different orders
    for plan in ((4, 256, 8, 256), (4, 256, 16, 256), (6, 256, 0, 1), (7, 256, 16, 2),
                 (6, 256, 0, 3), (7, 256, 16, 4)):
        s.set_sigma_plan(prec, *plan)
        got = s.sigma(V, prec)
        assert np.abs(got - ref).max() <= tol * np.abs(ref).max()
        assert np.array_equal(s.sigma(V, prec), got)     # bitwise reproducible


def test_sigma_multivector_and_determinism():
    s = jb.Space(10, 10)
    ints = workload_integrals("cas10_10")
    m1, m2 = ints.packed()
    s.set_integrals(m1, m2, ints.e_nuc, 0.0)
    V = np.random.default_rng(2).standard_normal((5, s.ndets))
    S = s.sigma(V)
    for k in range(5):
        Sk = s.sigma(V[k])
        assert np.array_equal(S[k], Sk[0])           # batch == single, bitwise
    assert np.array_equal(s.sigma(V), S)             # rerun is bitwise identical


@pytest.mark.slow
def test_full_size_properties_fci14():
    """FCI(14e,14o) with two frozen cores, 11 778 624 determinants: checks
    that hold at any size -- symmetry u.Hv = v.Hu, linearity, determinism."""
    s = jb.Space(18, 16, 2)
    ints = workload_integrals("fci14_14_fc2")
    m1, m2 = ints.packed()
    s.set_integrals(m1, m2, ints.e_nuc, ints.e_fc)
    rng = np.random.default_rng(4)
    U = rng.standard_normal((2, s.ndets))
    S = s.sigma(U)
    a, b = U[0] @ S[1], U[1] @ S[0]
    assert abs(a - b) <= 1e-10 * abs(a)
    W = s.sigma(0.5 * U[0] - 2.0 * U[1])[0]
    lin = 0.5 * S[0] - 2.0 * S[1]
    assert np.abs(W - lin).max() <= 1e-11 * np.abs(lin).max()
    assert np.array_equal(s.sigma(U), S)
    # FP32 sigma tracks FP64 to single precision
    S32 = s.sigma(U, jb.FP32)
    assert np.abs(S32 - S).max() <= 5e-6 * np.abs(S).max()
