"""Dyson orbitals (the reference's pdycicalc program): the oracle against the
reference's own dysoncomp.c (committed fixtures and, where the reference
build exists, live), the dycicalc.in reader and the dysonorb.dat writer.
No GPU needed."""
import glob
import os

import numpy as np
import pytest

import jayci_b200 as jb
from oracle import oracle

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "dyson_*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_reference_fixtures(path):
    g = np.load(path)
    d = oracle.dyson(tuple(g["general0"]), tuple(g["general1"]), g["v0"], g["v1"],
                     g["states0"], g["states1"])
    np.testing.assert_allclose(d, g["dyorb"], rtol=0, atol=1e-13)
    # the fixtures are not trivial: unit-norm states give O(1) amplitudes
    assert np.abs(g["dyorb"]).max() > 0.1


CASES = [  # (N+1)-electron &wavefcn0, N-electron &wavefcn1, states0, states1
    ((7, 6, 0, 0, 6, 0, 0), (6, 6, 0, 0, 6, 0, 0), [1], [1]),        # alpha removed
    ((8, 6, 0, 0, 6, 0, 0), (7, 6, 0, 0, 6, 0, 0), [1, 2], [1, 2, 3]),  # beta removed
    ((10, 9, 1, 1, 4, 1, 2), (9, 9, 1, 1, 4, 1, 2), [1], [1, 2]),      # truncated, beta
    ((9, 9, 1, 1, 4, 1, 2), (8, 9, 1, 1, 4, 1, 2), [1, 2], [1]),       # truncated, alpha
]


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_live_reference(case):
    g0, g1, st0, st1 = case
    n0, n1 = oracle.ci_space(g0).ndets, oracle.ci_space(g1).ndets
    rng = np.random.default_rng(sum(g0) + len(st1))
    v0, v1 = rng.standard_normal((3, n0)), rng.standard_normal((3, n1))
    d = oracle.dyson(g0, g1, v0, v1, st0, st1)
    r = oracle.ref_dyson(g0, g1, v0, v1, st0, st1)
    np.testing.assert_allclose(d, r, rtol=0, atol=1e-12 * np.abs(r).max())


def test_oracle_linearity_and_prefactor():
    """Size-independent properties: bilinear in (v0, v1), scaled by sqrt(N+1)."""
    g0, g1 = (9, 8, 0, 0, 8, 0, 0), (8, 8, 0, 0, 8, 0, 0)
    n0, n1 = oracle.ci_space(g0).ndets, oracle.ci_space(g1).ndets
    rng = np.random.default_rng(3)
    a, b = rng.standard_normal((2, n0)), rng.standard_normal((1, n1))
    da = oracle.dyson(g0, g1, a[:1], b, [1], [1])
    db = oracle.dyson(g0, g1, a[1:], b, [1], [1])
    dab = oracle.dyson(g0, g1, a[:1] + 2 * a[1:], b, [1], [1])
    np.testing.assert_allclose(dab, da + 2 * db, rtol=1e-12, atol=1e-12)
    # one (N+1) determinant against an all-ones N vector: each of its 5
    # alpha electrons contributes sqrt(9) to its own orbital
    e0 = np.zeros((1, n0))
    e0[0, 0] = 1.0
    d = oracle.dyson(g0, g1, e0, np.ones((1, n1)), [1], [1])
    assert np.count_nonzero(d) == 5 and np.allclose(d[d != 0], 3.0)


def test_read_dycicalc(tmp_path):
    p = tmp_path / "dycicalc.in"
    p.write_text(""" &wavefcn0
  electrons = 9, orbitals = 12, nfrozen = 1, ndocc = 2, nactive = 6,
  nfrzvirt = 1, xlevel = 1, nstates = 3   ! anion
 /
 &wavefcn1
  electrons = 8, orbitals = 12, nfrozen = 1, ndocc = 2, nactive = 6,
  nfrzvirt = 1, xlevel = 1, nstates = 2
 /
 &dysonorbital
  states0 = 1, 2
  states1(2) = 2
 /
""")
    w0, w1, s0, s1 = jb.read_dycicalc(p)
    assert w0.general() == (9, 12, 1, 2, 6, 1, 1) and w0.nstates == 3
    assert w1.general() == (8, 12, 1, 2, 6, 1, 1) and w1.nstates == 2
    np.testing.assert_array_equal(s0, [1, 2])
    np.testing.assert_array_equal(s1, [1, 2])  # states1(1) keeps its default 1
    # defaults: one state each; the count is the last nonzero position
    p.write_text("&wavefcn0 electrons=3 /\n&wavefcn1 electrons=2 /\n&dysonorbital /\n")
    w0, w1, s0, s1 = jb.read_dycicalc(p)
    np.testing.assert_array_equal(s0, [1])
    np.testing.assert_array_equal(s1, [1])
    p.write_text("&wavefcn0 electrons=3 /\n&wavefcn1 electrons=2 /\n"
                 "&dysonorbital states0 = 3 /\n")
    assert list(jb.read_dycicalc(p)[2]) == [3]
    for bad in ("&wavefcn0 electrons=3 /\n&wavefcn1 bogus=1 /\n&dysonorbital /\n",
                "&wavefcn0 electrons=3 /\n&wavefcn1 electrons=2 /\n"
                "&dysonorbital states0 = 1 2 3 4 5 6 /\n",
                "&wavefcn0 electrons=3 /\n"):
        p.write_text(bad)
        with pytest.raises(jb.JciError):
            jb.read_dycicalc(p)
    with pytest.raises(jb.JciError) as ei:
        jb.read_dycicalc(tmp_path / "missing.in")
    assert ei.value.status == 6


def test_write_dysonorb_format(tmp_path):
    """print_dysonorbitals_to_file (run_pdycicalc.c:674-712): counts, orbital
    count, both state lists, then each orbital's values as %15.8lf and a blank
    line."""
    d = np.array([[0.5, -1.25, 0.0], [1e-9, 2.0, -3.5]])
    p = tmp_path / "dysonorb.dat"
    jb.write_dysonorb(p, d, [1], [1, 2])
    lines = p.read_text().split("\n")
    assert lines[:4] == [" 2 1 2", " 3", " 1", " 1 2"]
    assert lines[4:8] == ["     0.50000000", "    -1.25000000", "     0.00000000", ""]
    assert lines[8:12] == ["     0.00000000", "     2.00000000", "    -3.50000000", ""]


def test_dyson_needs_a_device():
    """No CPU fallback: without a CUDA device jci_dyson refuses."""
    if jb.device_count() > 0:
        pytest.skip("a device is present")
    s0, s1 = jb.Space(7, 6), jb.Space(6, 6)
    with pytest.raises(jb.JciError) as ei:
        jb.dyson(s0, s1, np.ones((1, s0.ndets)), np.ones((1, s1.ndets)))
    assert ei.value.status == 5
