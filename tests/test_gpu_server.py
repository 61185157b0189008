"""Continuous-batching server (jci_server_*): results are the same alone and
in a concurrent mix, warm starts along a geometry scan, admission by HBM
footprint.  Bar: FP64 energies within 1e-10 Eh of the single-solve path,
|<c_alone|c_mix>| > 1-1e-9."""
import numpy as np
import pytest

import jayci_b200 as jb
from jayci_b200.synth import make_integrals, perturb

pytestmark = pytest.mark.gpu

MIX = [  # (electrons, orbitals), nroots, integral seed
    ((6, 6), 2, 1),
    ((8, 8), 1, 2),
    ((8, 8), 3, 3),
    ((7, 7), 1, 4),
    ((10, 10), 1, 5),
    ((6, 6), 4, 6),
]


def general(e, o):
    return (e, o, 0, 0, o, 0, 0)


def submit_all(srv, items):
    tickets = []
    for (e, o), nroots, seed in items:
        ints = make_integrals(o, o, seed)
        m1, m2 = ints.packed()
        tickets.append(srv.submit(general(e, o), m1, m2, ints.e_nuc, 0.0, nroots=nroots,
                                  krymin=max(4, nroots), krymax=16, refdim=8, restol=1e-9))
    return tickets


def test_same_result_alone_and_in_mix():
    alone = []
    one = jb.Server(slots=1)
    for item in MIX:
        t = submit_all(one, [item])[0]
        r = one.wait(t)
        assert r.status == 0 and r.converged
        alone.append((np.array(r.energies[:r.nroots]), one.vectors(t, r.nroots)))
    one.close()
    srv = jb.Server(slots=4)
    tickets = submit_all(srv, MIX)
    for (item, t, (e0, c0)) in zip(MIX, tickets, alone):
        r = srv.wait(t)
        assert r.status == 0 and r.converged
        e = np.array(r.energies[:r.nroots])
        np.testing.assert_allclose(e, e0, rtol=0, atol=1e-10)
        c = srv.vectors(t, r.nroots)
        ov = np.abs(np.einsum("ij,ij->i", c, c0))
        assert (ov > 1 - 1e-9).all()
    srv.close()
    # and the same as the plain single-solve API
    (e, o), nroots, seed = MIX[2]
    ints = make_integrals(o, o, seed)
    m1, m2 = ints.packed()
    s = jb.Space(e, o)
    s.set_integrals(m1, m2, ints.e_nuc, 0.0)
    ref = s.davidson(maxiter=1000, krymin=4, krymax=16, nroots=nroots, refdim=8,
                     restol=1e-9, block=True)
    np.testing.assert_allclose(alone[2][0], ref.energies, rtol=0, atol=1e-10)


def test_warm_started_scan():
    srv = jb.Server(slots=2)
    base = make_integrals(8, 8, 77)
    steps = [base]
    for k in range(4):
        steps.append(perturb(steps[-1], 7700 + k))
    prev = -1
    warm_iters, cold_iters = [], []
    for ints in steps:
        m1, m2 = ints.packed()
        kw = dict(nroots=2, krymin=4, krymax=16, refdim=8, restol=1e-9)
        tw = srv.submit(general(8, 8), m1, m2, ints.e_nuc, 0.0, warm_from=prev, **kw)
        tc = srv.submit(general(8, 8), m1, m2, ints.e_nuc, 0.0, **kw)
        rw, rc = srv.wait(tw), srv.wait(tc)
        assert rw.converged and rc.converged
        np.testing.assert_allclose(rw.energies[:2], rc.energies[:2], rtol=0, atol=1e-10)
        if prev > 0:
            assert rw.warm_started
            warm_iters.append(rw.iterations)
            cold_iters.append(rc.iterations)
        prev = tw
    assert sum(warm_iters) < sum(cold_iters)
    srv.close()


def test_admission_by_footprint():
    ints = make_integrals(10, 10, 9)
    m1, m2 = ints.packed()
    tiny = jb.Server(budget_bytes=1 << 20, slots=2)
    with pytest.raises(jb.JciError) as ei:
        tiny.submit(general(10, 10), m1, m2, ints.e_nuc, 0.0)
    assert ei.value.status == 11  # JCI_ERR_BUSY: can never fit
    tiny.close()
    # a budget that holds only a few CAS(10,10) solves: all still finish
    srv = jb.Server(budget_bytes=1500 << 20, slots=3)
    ts = [srv.submit(general(10, 10), m1, m2, ints.e_nuc, 0.0, restol=1e-8) for _ in range(3)]
    es = [srv.wait(t).energies[0] for t in ts]
    assert max(es) - min(es) < 1e-10
    srv.close()
