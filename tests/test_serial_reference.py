"""The reference's serial jayci path against its pjayci path (no GPU needed).

The serial program (source/, built unchanged as
oracle/_ref/libjayci_serial.so: citrunc_rtnlist, the O(N^2) cimap of
generate_cimap, compute_hdgls, compute_hv and dvdalg) is the second
reference program for the same CI.  The engine follows pjayci
(mpi_source/), the reference of record; these tests pin how far the two
reference programs agree:

* every diagonal element, single replacement and opposite-spin double
  of the serial Hamiltonian equals pjayci's (through the oracle, which is
  pinned to pjayci) to 1e-12;
* every same-spin double differs: the serial eval2_20_cas
  (source/action_util.c:511-513) evaluates (i0 i1|f0 f1) - (i0 f0|i1 f1)
  on chemists'-packed integrals, with its own phase (pindex_double_rep_cas),
  where pjayci's hmatels_2xaa (mpi_source/action_util.c:237-245) evaluates
  the Slater-rule element (i0 f0|i1 f1) - (i0 f1|i1 f0).  The magnitudes
  match the serial formula on every element;
* the serial Davidson itself is sound: its energies are the eigenvalues of
  its own Hamiltonian.
"""
import ctypes
import os

import numpy as np
import pytest

from oracle.oracle import SERIAL_SO, OracleSpace, _ptr, ref_serial_solve, serial_available

pytestmark = pytest.mark.skipif(not serial_available(), reason="serial reference not built")
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _serial_hamiltonian(g):
    """Dense H of the serial path (one compute_hv per unit vector) in the
    pjayci determinant order, and the pjayci H from the oracle."""
    L = ctypes.CDLL(SERIAL_SO)
    L.ref_serial_sigma.restype = ctypes.c_longlong
    L.ref_serial_sigma.argtypes = [ctypes.c_int] * 7 + [ctypes.c_void_p] * 2 + [ctypes.c_int] + \
        [ctypes.c_void_p] * 4
    gen = [int(x) for x in g["general"]]
    m1 = np.ascontiguousarray(g["m1"])
    m2 = np.ascontiguousarray(g["m2"])
    e, o, nfc, nd, na, nfv, x = gen
    sp = OracleSpace((e + 1) // 2, e // 2, o, nd, na, x)
    n = sp.ndets
    C = np.zeros((n, n))
    dets = np.zeros(2 * n, np.int64)
    assert L.ref_serial_sigma(*gen, _ptr(m1), _ptr(m2), n, _ptr(np.eye(n)), _ptr(C), None,
                              _ptr(dets)) == n
    sa, sb = sp.strings(0), sp.strings(1)

    def mask(lst):
        return sum(1 << (int(v) - 1) for v in lst)
    ia = {mask(s): i for i, s in enumerate(sa)}
    ib = {mask(s): i for i, s in enumerate(sb)}
    perm = np.array([ia[int(dets[2 * i])] * len(sb) + ib[int(dets[2 * i + 1])]
                     for i in range(n)])
    Hs = np.zeros((n, n))
    Hs[np.ix_(perm, perm)] = C
    Hp = sp.sigma(m1, m2, np.eye(n))
    return Hs, Hp, sa, sb, m1, m2, o


@pytest.mark.parametrize("name", ["cas6_6", "cas7_7"])
def test_serial_hamiltonian_against_pjayci(name):
    from jayci_b200.synth import unpack_integrals
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    Hs, Hp, sa, sb, m1, m2, norb = _serial_hamiltonian(g)
    _, eri = unpack_integrals(m1, m2, norb)
    nb = len(sb)
    ma = [set(int(v) for v in s) for s in sa]
    mb = [set(int(v) for v in s) for s in sb]
    same, other = 0, 0
    for i in range(Hs.shape[0]):
        ai, bi = divmod(i, nb)
        for j in range(Hs.shape[0]):
            aj, bj = divmod(j, nb)
            da, db = len(ma[ai] - ma[aj]), len(mb[bi] - mb[bj])
            if da + db > 2:
                assert Hs[i, j] == 0.0 and abs(Hp[i, j]) < 1e-14
                continue
            if (da, db) in ((2, 0), (0, 2)):
                si, sj = (ma[ai], ma[aj]) if da else (mb[bi], mb[bj])
                i0, i1 = sorted(si - sj)
                f0, f1 = sorted(sj - si)
                ser = eri[i0 - 1, i1 - 1, f0 - 1, f1 - 1] - eri[i0 - 1, f0 - 1, i1 - 1, f1 - 1]
                assert abs(abs(Hs[i, j]) - abs(ser)) <= 1e-12
                same += 1
            else:
                assert abs(Hs[i, j] - Hp[i, j]) <= 1e-12, (i, j, da, db)
                other += 1
    assert same > 0 and other > 0
    # the two reference programs therefore have different spectra
    assert abs(np.linalg.eigvalsh(Hs)[0] - np.linalg.eigvalsh(Hp)[0]) > 1e-3


def test_serial_davidson_solves_its_own_hamiltonian():
    g = np.load(os.path.join(GOLDEN, "cas6_6.npz"))
    Hs, Hp, *_ = _serial_hamiltonian(g)
    e, _, times = ref_serial_solve(g["general"], g["m1"], g["m2"], float(g["e_nuc"]), 0.0,
                                   maxiter=500, krymin=4, krymax=10, nroots=2, refdim=8,
                                   restol=1e-9, want_vectors=False)
    w = np.linalg.eigvalsh(Hs)[:2] + float(g["e_nuc"])
    assert np.abs(e - w).max() <= 1e-9
    assert set(times) == {"cimap", "hdgls", "dvdalg"}
    # and the pjayci energies (golden) are those of the pjayci Hamiltonian
    assert np.abs(np.linalg.eigvalsh(Hp)[:2] + float(g["e_nuc"]) - g["energies"]).max() <= 1e-9
