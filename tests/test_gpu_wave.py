"""The product through row panels shared by all CTAs (k_sigma_wave, plan rows
= 32 + CTAs per SM): one alpha row's panel is built by many CTAs and gathered
by many others from a work queue, so it stays in L2.

Checked through jci_sigma_device against the reference's own sigma (the
CAS(10,10) golden vectors and the FCI(12e,12o) rows) and the oracle-pinned
rows of FCI(14e,14o) fc2 and FCI(16e,16o) (tests/golden), with the bars of
the other sigma tests (FP64 1e-12, FP32 2e-6 of the largest |sigma|).  Each
panel element and each sigma element is summed in the order of the per-CTA
panel kernel, so the result must be bitwise that of plan rows = 1 (same
mode, threads and group variant), and bitwise the same on a repeated call
whatever order the CTAs claimed the work in.
"""
import os
import sys

import numpy as np
import pytest

import jayci_b200 as jb
from jayci_b200.synth import workload_integrals

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
sys.path.insert(0, GOLDEN)
from seeded import hash_vector  # noqa: E402

BAR = {jb.FP64: 1e-12, jb.FP32: 2e-6}


def _sigma(s, v, prec):
    import torch
    dt = torch.float64 if prec == jb.FP64 else torch.float32
    x = torch.as_tensor(v).to(device="cuda", dtype=dt)
    y = torch.full_like(x, float("nan"))
    s.sigma_device(x.data_ptr(), y.data_ptr(), 1, s.ndets, prec, 0)
    torch.cuda.synchronize()
    return y


@pytest.mark.parametrize("prec", [jb.FP64, jb.FP32])
@pytest.mark.parametrize("plan", [(6, 256, 32, 1), (6, 256, 33, 2), (3, 256, 32, 256),
                                  (1, 256, 34, 2)])
def test_shared_panel_cas10(plan, prec):
    g = np.load(os.path.join(GOLDEN, "cas10_10.npz"))
    s = jb.Space(*(int(x) for x in g["general"]))
    s.set_integrals(g["m1"], g["m2"], float(g["e_nuc"]), 0.0)
    mode, nt, R, B = plan
    for k in range(2):
        v = g["sigma_v"][k]
        s.set_sigma_plan(prec, mode, nt, 1, B)
        base = _sigma(s, v, prec).cpu().numpy()
        s.set_sigma_plan(prec, *plan)
        y = _sigma(s, v, prec).cpu().numpy()
        ref = g["sigma"][k]
        assert np.abs(y.astype(np.float64) - ref).max() <= BAR[prec] * np.abs(ref).max()
        assert np.array_equal(y, base), plan
        assert np.array_equal(_sigma(s, v, prec).cpu().numpy(), y)
    s.close()


@pytest.mark.parametrize("name", ["fci12_12", "fci14_14_fc2", "fci16_16"])
@pytest.mark.parametrize("prec", [jb.FP64, jb.FP32])
def test_shared_panel_bench_sizes(name, prec):
    import torch
    g = np.load(os.path.join(GOLDEN, f"bench_{name}.npz"))
    ints = workload_integrals(name)
    m1, m2 = ints.packed()
    s = jb.Space(*(int(x) for x in g["general"]))
    s.set_integrals(m1, m2, ints.e_nuc, ints.e_fc)
    v = hash_vector(s.ndets, int(g["sigma_seed"]))
    rows = torch.from_numpy(g["rows"]).cuda()
    s.set_sigma_plan(prec, 6, 512, 32, 2)
    y = _sigma(s, v, prec)
    got = y[rows].double().cpu().numpy()
    ref = g["sigma_rows"]
    assert np.abs(got - ref).max() <= BAR[prec] * np.abs(ref).max()
    assert torch.equal(_sigma(s, v, prec), y)
    s.set_sigma_plan(prec, 6, 512, 1, 2)
    assert torch.equal(_sigma(s, v, prec), y)
    s.close()


def test_bounded_wait_expires_and_space_recovers():
    """A dependency that nothing satisfies (jci_test_expire_next_wait: the
    panel work of the first two alpha rows is skipped): the gathers that
    need it give up after their one-second bound, the kernel returns, the
    host reads JCI_ERR_TIMEOUT, and the next sigma on the same space is
    right again."""
    import ctypes
    import time
    g = np.load(os.path.join(GOLDEN, "cas10_10.npz"))
    s = jb.Space(*(int(x) for x in g["general"]))
    s.set_integrals(g["m1"], g["m2"], float(g["e_nuc"]), 0.0)
    s.set_sigma_plan(jb.FP64, 6, 256, 32, 1)
    v = np.ascontiguousarray(g["sigma_v"][0])
    ref = g["sigma"][0]
    bar = BAR[jb.FP64] * np.abs(ref).max()
    assert np.abs(s.sigma(v[None, :])[0] - ref).max() <= bar
    L = jb.lib()
    L.jci_test_expire_next_wait.argtypes = [ctypes.c_void_p]
    assert L.jci_test_expire_next_wait(s.h) == 0
    with pytest.raises(jb.JciError) as e:
        t0 = time.time()
        s.sigma(v[None, :])
    assert e.value.status == 10  # JCI_ERR_TIMEOUT
    assert 0.5 < time.time() - t0 < 60
    assert np.abs(s.sigma(v[None, :])[0] - ref).max() <= bar
    s.close()
