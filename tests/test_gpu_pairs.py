"""Same-spin doubles through (N-2)-electron hole strings (jci_fci_pairs.cu,
group kernel variants 5 and 6 of plans 6 and 7): dense products over the
free pairs of each hole string, then a pull of the C(N,2) hole rows of every
string; and the beta singles through (N-1)-electron hole strings (threads 0
of plans 6 and 7).

Checked through jci_sigma_device against the reference's own sigma (the
CAS(10,10) golden vectors, the FCI(12e,12o) rows) and the oracle-pinned rows
of FCI(14e,14o) fc2 and FCI(16e,16o), at the bars of the other sigma tests
(FP64 1e-12, FP32 2e-6 of the largest |sigma|); against the oracle on a CAS
with doubly occupied inactive orbitals (orbitals common to every string,
which enter the phases); and for bitwise equality on a repeated call.
"""
import os
import sys

import numpy as np
import pytest

import jayci_b200 as jb
from jayci_b200.synth import make_integrals, workload_integrals

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
@pytest.mark.parametrize("plan", [(6, 256, 0, 5), (6, 256, 0, 6), (7, 256, 16, 5),
                                  (6, 256, 2, 6),
                                  # threads 0: the beta singles through hole strings too
                                  (6, 0, 66, 5), (7, 0, 16, 2), (6, 0, 0, 1)])
def test_hole_pairs_cas10(plan, prec):
    g = np.load(os.path.join(GOLDEN, "cas10_10.npz"))
    s = jb.Space(*(int(x) for x in g["general"]))
    s.set_integrals(g["m1"], g["m2"], float(g["e_nuc"]), 0.0)
    s.set_sigma_plan(prec, *plan)
    for k in range(2):
        v = g["sigma_v"][k]
        y = _sigma(s, v, prec).cpu().numpy()
        ref = g["sigma"][k]
        assert np.abs(y.astype(np.float64) - ref).max() <= BAR[prec] * np.abs(ref).max(), plan
        assert np.array_equal(_sigma(s, v, prec).cpu().numpy(), y)
    s.close()


@pytest.mark.parametrize("prec", [jb.FP64, jb.FP32])
def test_hole_pairs_with_inactive_orbitals(prec):
    """CAS(6e,6o) inside 10 orbitals with 2 doubly occupied inactive orbitals
    (general = 10 electrons, 10 orbitals, ndocc 2, 6 active, excitation
    level 0): the inactive orbitals are in every string."""
    from oracle.oracle import OracleSpace
    s = jb.Space(10, 10, 0, 2, 6, 0, 0)
    ints = make_integrals(10, 10, 31)
    m1, m2 = ints.packed()
    s.set_integrals(m1, m2, ints.e_nuc, 0.0)
    o = OracleSpace(5, 5, 10, ndocc=2, nactv=6)
    v = np.random.default_rng(4).standard_normal(s.ndets)
    ref = o.sigma(m1, m2, v[None, :])[0]
    for nt in (128, 0):  # 20 strings per spin: 128-thread streams, or hole-string singles
        s.set_sigma_plan(prec, 6, nt, 0, 5)
        y = _sigma(s, v, prec).double().cpu().numpy()
        assert np.abs(y - ref).max() <= BAR[prec] * np.abs(ref).max(), nt
    s.close()


@pytest.mark.parametrize("name", ["fci12_12", "fci14_14_fc2", "fci16_16"])
@pytest.mark.parametrize("prec", [jb.FP64, jb.FP32])
def test_hole_pairs_bench_sizes(name, prec):
    import torch
    g = np.load(os.path.join(GOLDEN, f"bench_{name}.npz"))
    ints = workload_integrals(name)
    m1, m2 = ints.packed()
    s = jb.Space(*(int(x) for x in g["general"]))
    s.set_integrals(m1, m2, ints.e_nuc, ints.e_fc)
    v = hash_vector(s.ndets, int(g["sigma_seed"]))
    rows = torch.from_numpy(g["rows"]).cuda()
    ref = g["sigma_rows"]
    for nt, variant in ((512, 5), (512, 6), (0, 5), (512, 7)):
        s.set_sigma_plan(prec, 6, nt, 2, variant)
        y = _sigma(s, v, prec)
        got = y[rows].double().cpu().numpy()
        assert np.abs(got - ref).max() <= BAR[prec] * np.abs(ref).max(), variant
        y2 = _sigma(s, v, prec)
        diff = (y2 != y).sum().item()
        assert diff == 0, (nt, variant, diff, torch.isnan(y).sum().item(),
                           torch.isnan(y2).sum().item(), (y2 - y).abs().max().item())
    s.close()


@pytest.mark.parametrize("name", ["cas10_10", "fci12_12", "fci14_14_fc2", "fci16_16"])
@pytest.mark.parametrize("prec", [jb.FP64, jb.FP32])
def test_compact_panel_is_bitwise_the_full_panel(name, prec):
    """The product panel stored compact (plan rows + 64: only the entries the
    gather reads, at positions from per-chunk masks) sums the same terms in
    the same order as the full panel, so sigma is bitwise the same."""
    import torch
    if name == "cas10_10":
        g = np.load(os.path.join(GOLDEN, "cas10_10.npz"))
        s = jb.Space(*(int(x) for x in g["general"]))
        s.set_integrals(g["m1"], g["m2"], float(g["e_nuc"]), 0.0)
        v = g["sigma_v"][0]
        nt = 256
    else:
        g = np.load(os.path.join(GOLDEN, f"bench_{name}.npz"))
        ints = workload_integrals(name)
        m1, m2 = ints.packed()
        s = jb.Space(*(int(x) for x in g["general"]))
        s.set_integrals(m1, m2, ints.e_nuc, ints.e_fc)
        v = hash_vector(s.ndets, int(g["sigma_seed"]))
        nt = 512
    s.set_sigma_plan(prec, 6, nt, 2, 2)
    full = _sigma(s, v, prec)
    s.set_sigma_plan(prec, 6, nt, 64 + 2, 2)
    cp = _sigma(s, v, prec)
    assert torch.equal(cp, full)
    if name == "cas10_10":
        ref = g["sigma"][0]
        got = cp.double().cpu().numpy()
        assert np.abs(got - ref).max() <= BAR[prec] * np.abs(ref).max()
    s.close()
