"""libjci's host-side string space through the C ABI (no GPU needed).

The space is built by the product code (jayci_b200/csrc/jci_space.cpp) and
compared with the reference's golden vectors: strings, groups, pairs,
addresses and excitation phases must be bit-exact.
"""
import glob
import os

import numpy as np
import pytest

import jayci_b200 as jb
from oracle.oracle import canonical_excitation

GOLDEN = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
                if not os.path.basename(p).startswith(("dyson_", "bench_")))
NAMES = [os.path.basename(p)[:-4] for p in GOLDEN]


def load(name):
    return np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))


def space_for(g):
    e, o, nfc, nd, na, nfv, x = (int(v) for v in g["general"])
    return jb.Space(e, o, nfc, nd, na, nfv, x)


@pytest.mark.parametrize("name", NAMES)
def test_space_matches_reference(name):
    g = load(name)
    s = space_for(g)
    assert (s.na, s.nb, s.norb, s.nastr, s.nbstr, s.pegrps, s.qegrps, s.npq, s.ndets) == \
        tuple(int(x) for x in g["sizes"])
    for sp in (0, 1):
        assert np.array_equal(s.strings(sp), g[f"istr{sp}"])
        assert np.array_equal(s.eospaces(sp), g[f"eosp{sp}"][:, :5])
    assert np.array_equal(s.pq(), g["pq"])


@pytest.mark.parametrize("name", NAMES)
def test_excitations_match_reference(name):
    g = load(name)
    s = space_for(g)
    for sp in (0, 1):
        rows = g[f"exc{sp}"]
        keys = sorted(set((int(r[0]), int(r[1]), int(r[2])) for r in rows))
        for st, grp, nrep in keys:
            ref = sorted(canonical_excitation(r[3:]) for r in rows
                         if r[0] == st and r[1] == grp and r[2] == nrep)
            got = sorted(canonical_excitation(r) for r in s.excitations(sp, nrep, st, grp))
            assert got == ref, (sp, st, grp, nrep)


@pytest.mark.parametrize("name", NAMES)
def test_string_addresses(name):
    """occstr2address / str_adrfind: every string's orbital list maps to its
    own index; lists outside the expansion map to -1."""
    g = load(name)
    s = space_for(g)
    for sp in (0, 1):
        istr = g[f"istr{sp}"]
        for i in range(0, istr.shape[0], max(1, istr.shape[0] // 500)):
            assert s.string_index(sp, istr[i]) == i
        bad = np.arange(1, istr.shape[1] + 1, dtype=np.int32)[::-1].copy()
        if istr.shape[1] > 1:
            assert s.string_index(sp, bad) == -1  # not sorted


def test_workload_sizes():
    """Determinant counts of the named workloads."""
    for (e, o, nfc, n) in [(10, 10, 0, 63504), (12, 12, 0, 853776), (18, 16, 2, 11778624)]:
        s = jb.Space(e, o, nfc)
        assert s.ndets == n
        s.close()


def test_space_limits_rejected():
    with pytest.raises(jb.JciError) as ei:
        jb.Space(44, 44)  # 22 alpha electrons > 20 (execute_pjayci.c:145)
    assert ei.value.status == 2
    with pytest.raises(jb.JciError):
        jb.Space(10, 70, 0, 0, 70)  # 70 internal orbitals > 64


def test_sigma_plan_calls_checked_on_the_host():
    """jci_sigma_set_plan refuses bad modes and precisions (JCI_ERR_ARG) and
    any plan before jci_set_integrals (JCI_ERR_STATE); jci_sigma_tuning
    reports zeros before the first sigma.  No device is touched."""
    s = jb.Space(6, 6)
    for args in ((jb.FP64, 8, 256, 1, 1), (jb.FP64, -1, 256, 1, 1),
                 (jb.MIXED, 1, 256, 1, 1), (7, 1, 256, 1, 1)):
        with pytest.raises(jb.JciError) as ei:
            s.set_sigma_plan(*args)
        assert ei.value.status == 1
    with pytest.raises(jb.JciError) as ei:
        s.set_sigma_plan(jb.FP64, 7, 256, 16, 3)
    assert ei.value.status == 12
    assert s.sigma_tuning(jb.FP64) == (0, 0, 0, 0, 0.0)
    assert s.sigma_tuning(jb.FP32) == (0, 0, 0, 0, 0.0)
    s.close()
