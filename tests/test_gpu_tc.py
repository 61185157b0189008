"""The FP32 product on the tcgen05 tensor cores (jci_fci_tc.cu), forced as
the product engine of the fused plans (rows = 32 or 64: tensor-memory engine
with chunks of that many columns) and checked against the reference's own
sigma: the CAS(10,10) golden sigma, and the sampled rows of FCI(12e,12o)
FCI(14e,14o) fc2 and FCI(16e,16o) (tests/golden; 512 threads per CTA for the
12 870 beta strings of FCI(16,16)).  Bar: FP32 2e-6 of max|sigma|;
repeated calls are bitwise identical."""
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


def _sigma32(s, v):
    import torch
    x = torch.as_tensor(v, dtype=torch.float32).cuda()
    y = torch.full_like(x, float("nan"))
    s.sigma_device(x.data_ptr(), y.data_ptr(), 1, s.ndets, jb.FP32, 0)
    torch.cuda.synchronize()
    return y


@pytest.mark.parametrize("plan", [(5, 256, 64, 1), (5, 256, 32, 1), (7, 256, 64, 2),
                                  (4, 256, 64, 256)])
def test_tc_engine_cas10(plan):
    g = np.load(os.path.join(GOLDEN, "cas10_10.npz"))
    s = jb.Space(*(int(x) for x in g["general"]))
    s.set_integrals(g["m1"], g["m2"], float(g["e_nuc"]), 0.0)
    s.set_sigma_plan(jb.FP32, *plan)
    for k in range(2):
        v = g["sigma_v"][k]
        y = _sigma32(s, v)
        ref = g["sigma"][k]
        got = y.double().cpu().numpy()
        assert np.abs(got - ref).max() <= 2e-6 * np.abs(ref).max(), (plan, k)
        assert np.array_equal(_sigma32(s, v).cpu().numpy(), y.cpu().numpy())
    s.close()


@pytest.mark.parametrize("name,rows", [("fci12_12", 32), ("fci12_12", 64),
                                       ("fci14_14_fc2", 32), ("fci14_14_fc2", 64),
                                       ("fci16_16", 32)])
def test_tc_engine_bench_sizes(name, rows):
    import torch
    g = np.load(os.path.join(GOLDEN, f"bench_{name}.npz"))
    ints = workload_integrals(name)
    m1, m2 = ints.packed()
    s = jb.Space(*(int(x) for x in g["general"]))
    s.set_integrals(m1, m2, ints.e_nuc, ints.e_fc)
    s.set_sigma_plan(jb.FP32, 7, 512, rows, 2)
    v = hash_vector(s.ndets, int(g["sigma_seed"]))
    y = _sigma32(s, v)
    got = y[torch.from_numpy(g["rows"]).cuda()].double().cpu().numpy()
    ref = g["sigma_rows"]
    assert np.abs(got - ref).max() <= 2e-6 * np.abs(ref).max()
    s.close()
