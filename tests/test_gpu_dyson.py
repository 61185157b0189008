"""Dyson orbitals on the GPU (jci_dyson) against the reference's fixtures and
the oracle, and the jci_dyson program end to end.  Bar: 1e-12 of the largest
amplitude (FP64 sums in a different order)."""
import glob
import os
import subprocess

import numpy as np
import pytest

import jayci_b200 as jb
from oracle import oracle

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "dyson_*.npz")))


def spaces(g0, g1):
    return jb.Space(*g0), jb.Space(*g1)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_dyson_matches_reference_fixtures(path):
    g = np.load(path)
    s0, s1 = spaces(tuple(int(x) for x in g["general0"]), tuple(int(x) for x in g["general1"]))
    d = jb.dyson(s0, s1, g["v0"], g["v1"], g["states0"], g["states1"])
    ref = g["dyorb"]
    np.testing.assert_allclose(d, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("g0,g1,st0,st1", [
    # 13e -> 12e on 12 orbitals: 731 808 -> 853 776 determinants, alpha removed
    ((13, 12, 0, 0, 12, 0, 0), (12, 12, 0, 0, 12, 0, 0), [1, 2], [1, 2]),
    # 12e -> 11e, beta removed, all 5 x 5 state pairs
    ((12, 10, 0, 0, 10, 0, 0), (11, 10, 0, 0, 10, 0, 0), [1, 2, 3, 4, 5], [5, 4, 3, 2, 1]),
    # frozen core, DOCC/ACTV/VIRT, excitation level 2
    ((12, 14, 1, 2, 6, 1, 2), (11, 14, 1, 2, 6, 1, 2), [2], [1, 3]),
])
def test_dyson_matches_oracle(g0, g1, st0, st1):
    s0, s1 = spaces(g0, g1)
    rng = np.random.default_rng(g0[0] * 100 + g0[1])
    v0 = rng.standard_normal((max(st0), s0.ndets))
    v1 = rng.standard_normal((max(st1), s1.ndets))
    d = jb.dyson(s0, s1, v0, v1, st0, st1)
    ref = oracle.dyson(g0, g1, v0, v1, st0, st1)
    np.testing.assert_allclose(d, ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    # deterministic: the same call gives the same bits
    np.testing.assert_array_equal(d, jb.dyson(s0, s1, v0, v1, st0, st1))


def test_dyson_rejects_mismatched_wavefunctions():
    s0, s1 = jb.Space(8, 6), jb.Space(6, 6)  # two electrons apart
    with pytest.raises(jb.JciError) as ei:
        jb.dyson(s0, s1, np.ones((1, s0.ndets)), np.ones((1, s1.ndets)))
    assert ei.value.status == 1
    s0, s1 = jb.Space(7, 6), jb.Space(6, 7)  # different orbitals
    with pytest.raises(jb.JciError):
        jb.dyson(s0, s1, np.ones((1, s0.ndets)), np.ones((1, s1.ndets)))
    s0, s1 = jb.Space(7, 6), jb.Space(6, 6)
    with pytest.raises(jb.JciError):  # state 2 of a one-state vector set
        jb.dyson(s0, s1, np.ones((1, s0.ndets)), np.ones((1, s1.ndets)), [1], [2])


def test_dyson_program(tmp_path):
    """jci_dyson: dycicalc.in + anion.ci + neutral.ci -> dysonorb.dat, the
    reference pdycicalc flow; compared with the reference's fixture."""
    g = np.load(os.path.join(HERE, "golden", "dyson_trunc8_8_x2.npz"))
    g0 = tuple(int(x) for x in g["general0"])
    g1 = tuple(int(x) for x in g["general1"])
    keys = ("electrons", "orbitals", "nfrozen", "ndocc", "nactive", "nfrzvirt", "xlevel")

    def nml(name, gen, n):
        body = ", ".join(f"{k} = {v}" for k, v in zip(keys, gen))
        return f" &{name}\n  {body}, nstates = {n}\n /\n"
    st0 = ", ".join(str(int(x)) for x in g["states0"])
    st1 = ", ".join(str(int(x)) for x in g["states1"])
    (tmp_path / "dycicalc.in").write_text(
        nml("wavefcn0", g0, g["v0"].shape[0]) + nml("wavefcn1", g1, g["v1"].shape[0]) +
        f" &dysonorbital\n  states0 = {st0}\n  states1 = {st1}\n /\n")
    jb.write_vectors(tmp_path / "anion.ci", g["v0"])
    jb.write_vectors(tmp_path / "neutral.ci", g["v1"])
    exe = os.path.join(os.path.dirname(jb.LIBPATH), "jci_dyson")
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = (tmp_path / "dysonorb.dat").read_text().split("\n")
    nd, n0, n1 = (int(x) for x in lines[0].split())
    norbs = int(lines[1])
    assert (nd, n0, n1, norbs) == (g["dyorb"].shape[0], len(g["states0"]), len(g["states1"]),
                                   g0[1])
    vals = np.array([float(x) for x in lines[4:] if x.strip()]).reshape(nd, norbs)
    np.testing.assert_allclose(vals, g["dyorb"], rtol=0, atol=1e-8)  # %15.8f
