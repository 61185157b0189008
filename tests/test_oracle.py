"""The CPU oracle (C restatement) pinned against the reference's golden vectors.

The fixtures in tests/golden were produced by the reference's own code
(tests/golden/make_golden.py).  Integer work (strings, groups, pairs,
determinant order, excitation lists and phases) must match bit for bit;
<i|H|i> and sigma to rounding (1e-12 relative); Davidson energies to 1e-10 Eh.
"""
import glob
import os

import numpy as np
import pytest

from oracle.oracle import OracleSpace, canonical_excitation, ref_available, RefSpace, symeig

GOLDEN = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
                if not os.path.basename(p).startswith(("dyson_", "bench_")))
NAMES = [os.path.basename(p)[:-4] for p in GOLDEN]


def load(name):
    return np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))


def oracle_for(g):
    e, o, nfc, nd, na, nfv, x = (int(v) for v in g["general"])
    s = g["sizes"]
    return OracleSpace(int(s[0]), int(s[1]), int(s[2]), nd, na, x)


@pytest.mark.parametrize("name", NAMES)
def test_strings_groups_pairs(name):
    g = load(name)
    o = oracle_for(g)
    s = g["sizes"]
    assert (o.nastr, o.nbstr, o.pegrps, o.qegrps, o.npq, o.ndets) == tuple(
        int(x) for x in s[[3, 4, 5, 6, 7, 8]])
    for sp in (0, 1):
        assert np.array_equal(o.strings(sp), g[f"istr{sp}"])
        assert np.array_equal(o.eospaces(sp), g[f"eosp{sp}"][:, :5])
    assert np.array_equal(o.pq(), g["pq"])


@pytest.mark.parametrize("name", NAMES)
def test_excitation_lists_and_phases(name):
    g = load(name)
    o = oracle_for(g)
    for sp in (0, 1):
        rows = g[f"exc{sp}"]
        keys = sorted(set((int(r[0]), int(r[1]), int(r[2])) for r in rows))
        for s, grp, nrep in keys:
            ref = sorted(canonical_excitation(r[3:]) for r in rows
                         if r[0] == s and r[1] == grp and r[2] == nrep)
            got = sorted(canonical_excitation(r) for r in o.excitations(sp, nrep, s, grp))
            assert got == ref, (sp, s, grp, nrep)


@pytest.mark.parametrize("name", [n for n in NAMES if n != "cas10_10"])
def test_yij_cij_tables(name):
    """yij = phase of electron e -> orbital o, cij = resulting string index,
    compared on every entry the reference fills (compute_yij_lists)."""
    g = load(name)
    o = oracle_for(g)
    for sp in (0, 1):
        istr = g[f"istr{sp}"]
        y, c = g[f"yij{sp}"], g[f"cij{sp}"]
        ne = istr.shape[1]
        for s in range(istr.shape[0]):
            occ = set(istr[s])
            for e in range(ne):
                for orb in range(1, y.shape[2]):
                    if orb in occ:
                        continue
                    new = sorted((occ - {istr[s][e]}) | {orb})
                    idx = OracleSpace.lib().jo_string_index(
                        o.h, sp, np.array(new, np.int32).ctypes.data_as(__import__("ctypes").c_void_p))
                    between = sum(1 for x in occ if min(orb, istr[s][e]) < x < max(orb, istr[s][e]))
                    assert y[s, e, orb] == (-1) ** between
                    if idx >= 0:
                        assert c[s, e, orb] == idx


@pytest.mark.parametrize("name", NAMES)
def test_hdiag_and_sigma(name):
    g = load(name)
    o = oracle_for(g)
    hd = o.hdiag(g["m1"], g["m2"])
    np.testing.assert_allclose(hd, g["hdiag"], rtol=1e-13, atol=1e-12)
    S = o.sigma(g["m1"], g["m2"], g["sigma_v"])
    scale = np.abs(g["sigma"]).max()
    assert np.abs(S - g["sigma"]).max() <= 1e-12 * scale


@pytest.mark.parametrize("name", [n for n in NAMES if n != "cas10_10"])
def test_davidson_energies(name):
    g = load(name)
    o = oracle_for(g)
    kmin, kmax, nroots, refdim = (int(x) for x in g["dav_opts"])
    e, civ, it = o.davidson(g["m1"], g["m2"], float(g["e_nuc"]), maxiter=500,
                            krymin=kmin, krymax=kmax, nroots=nroots, refdim=refdim,
                            restol=1e-9)
    np.testing.assert_allclose(e, g["energies"], rtol=0, atol=1e-10)
    ov = np.abs(np.einsum("ij,ij->i", civ, g["civec"]))
    assert (ov > 1 - 1e-9).all()


def test_symeig_against_numpy():
    a = np.random.default_rng(3).standard_normal((9, 9))
    a = a + a.T
    w, z = symeig(a)
    np.testing.assert_allclose(w, np.linalg.eigvalsh(a), atol=1e-12)
    np.testing.assert_allclose(z @ a @ z.T, np.diag(w), atol=1e-11)


@pytest.mark.skipif(not ref_available(), reason="reference build (oracle/_ref) absent")
@pytest.mark.parametrize("gen", [
    (6, 6, 0, 0, 6, 0, 0), (8, 10, 0, 2, 5, 0, 2), (7, 9, 1, 1, 5, 0, 2),
    (10, 12, 0, 3, 4, 1, 2), (6, 8, 0, 2, 4, 0, 1)])
def test_oracle_against_reference_build(gen):
    """Live comparison with the reference compiled from its own sources."""
    from jayci_b200.synth import make_integrals
    ref = RefSpace(*gen)
    o = OracleSpace(ref.na, ref.nb, ref.norb, gen[3], gen[4], gen[6])
    assert o.ndets == ref.ndets
    for sp in (0, 1):
        assert np.array_equal(o.strings(sp), ref.strings(sp)[0])
    ints = make_integrals(ref.norb, 6, 5)
    m1, m2 = ints.packed()
    V = np.random.default_rng(9).standard_normal((1, ref.ndets))
    S1, S2 = ref.sigma(m1, m2, V), o.sigma(m1, m2, V)
    assert np.abs(S1 - S2).max() <= 1e-12 * np.abs(S1).max()
