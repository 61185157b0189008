"""The allocation-free sigma entry point (jci_sigma_device_noalloc).

Some callers cannot call cudaMalloc while sigma runs -- a driver that
captures its Davidson iteration into a CUDA graph, a process held to a fixed
device-memory budget, an application whose allocator forbids device
allocation after start-up.  For them libjci offers a sigma whose scratch
panels live in a fixed 64 MiB device array inside the library.  This file
checks it through the C ABI against the ordinary entry point
(jci_sigma_device) on two consecutive calls, with the same tolerances as the
other sigma tests (FP64 1e-12, FP32 2e-6 of max|sigma|).  It is named so that
pytest collects it last.
"""
import ctypes
import os

import numpy as np
import pytest

import jayci_b200 as jb
from jayci_b200.synth import make_integrals

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _space(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    e, o, nfc, nd, na, nfv, x = (int(v) for v in g["general"])
    s = jb.Space(e, o, nfc, nd, na, nfv, x)
    s.set_integrals(g["m1"], g["m2"], float(g["e_nuc"]), 0.0)
    return s, g


def _noalloc(s, v_ptr, o_ptr, prec, stream):
    f = jb.lib().jci_sigma_device_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                  ctypes.c_void_p]
    return f(s.h, ctypes.c_void_p(v_ptr), ctypes.c_void_p(o_ptr), prec,
             ctypes.c_void_p(stream))


@pytest.mark.parametrize("name", ["cas10_10", "cas7_7"])
@pytest.mark.parametrize("prec", [jb.FP64, jb.FP32])
def test_noalloc_matches_sigma_device(name, prec):
    import torch
    s, g = _space(name)
    dt = torch.float64 if prec == jb.FP64 else torch.float32
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        v = torch.tensor(g["sigma_v"][0], dtype=dt, device="cuda").contiguous()
        ref = torch.empty_like(v)
        s.sigma_device(v.data_ptr(), ref.data_ptr(), 1, s.ndets, prec, st.cuda_stream)
        torch.cuda.synchronize()
        tol = (1e-12 if prec == jb.FP64 else 2e-6) * ref.abs().max().item()
        for _ in range(2):  # two calls in a row share the static scratch array
            out = torch.full_like(v, float("nan"))
            assert _noalloc(s, v.data_ptr(), out.data_ptr(), prec, st.cuda_stream) == 0
            torch.cuda.synchronize()
            assert (out - ref).abs().max().item() <= tol
    golden = g["sigma"][0]
    assert np.abs(out.double().cpu().numpy() - golden).max() <= 2 * tol


def test_noalloc_rejects_unsupported_space():
    import torch
    # truncated space with several occupation groups: not a one-group space
    s, g = _space("trunc6_8_x2")
    v = torch.zeros(s.ndets, dtype=torch.float64, device="cuda")
    o = torch.zeros_like(v)
    assert _noalloc(s, v.data_ptr(), o.data_ptr(), jb.FP64, 0) == 2
    # CAS(4,4) inside 40 orbitals: the product panel has 821 rows, more than
    # the kernel's 144-row tile, so the call is refused
    s2 = jb.Space(4, 40, 0, 0, 4, 0, 0)
    ints = make_integrals(40, 4, 3)
    m1, m2 = ints.packed()
    s2.set_integrals(m1, m2, ints.e_nuc, 0.0)
    v2 = torch.zeros(s2.ndets, dtype=torch.float64, device="cuda")
    o2 = torch.zeros_like(v2)
    assert _noalloc(s2, v2.data_ptr(), o2.data_ptr(), jb.FP64, 0) == 2
