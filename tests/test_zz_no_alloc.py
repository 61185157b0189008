"""The allocation-free sigma entry point (jci_sigma_device_noalloc).

Some callers cannot call cudaMalloc while sigma runs -- a driver that
captures its Davidson iteration into a CUDA graph, a process held to a fixed
device-memory budget, an application whose allocator forbids device
allocation after start-up.  For them libjci offers a sigma whose scratch
panels live in a fixed 64 MiB device array inside the library.  This file
checks it through the C ABI against the ordinary entry point
(jci_sigma_device) on two consecutive calls, with the tolerances of the
other sigma tests (FP64 1e-12, FP32 2e-6 of max|sigma| from the exact sigma,
so two FP32 results agree within 4e-6), and checks that the device's free
memory does not move across its first call on a fresh space.
It is named so that pytest collects it last.
"""
import ctypes
import os

import numpy as np
import pytest

import jayci_b200 as jb
from jayci_b200.synth import make_integrals

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = {jb.FP64: 1e-12, jb.FP32: 2e-6}


def _space(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    e, o, nfc, nd, na, nfv, x = (int(v) for v in g["general"])
    s = jb.Space(e, o, nfc, nd, na, nfv, x)
    s.set_integrals(g["m1"], g["m2"], float(g["e_nuc"]), 0.0)
    return s, g


def _cas(n, seed):
    """CAS(n, n) with nalpha = nbeta: one occupation group per spin."""
    s = jb.Space(n, n)
    ints = make_integrals(n, n, seed)
    m1, m2 = ints.packed()
    s.set_integrals(m1, m2, ints.e_nuc, 0.0)
    return s


def _noalloc(s, v_ptr, o_ptr, prec, stream):
    f = jb.lib().jci_sigma_device_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                  ctypes.c_void_p]
    return f(s.h, ctypes.c_void_p(v_ptr), ctypes.c_void_p(o_ptr), prec,
             ctypes.c_void_p(stream))


def _vector(n, prec, seed):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    dt = torch.float64 if prec == jb.FP64 else torch.float32
    return torch.randn(n, dtype=torch.float64, device="cuda", generator=g).to(dt)


def _check_two_calls(s, v, ref, prec, stream):
    """Two noalloc calls in a row into NaN-filled outputs, each against ref,
    the existing entry point's output in the same precision.  The two may
    sum in different orders (the entry point runs its tuned plan): in FP64
    they agree to 1e-12; in FP32 each lies within 2e-6 of the exact sigma,
    so they agree within twice that."""
    import torch
    tol = (1 if prec == jb.FP64 else 2) * TOL[prec] * ref.abs().max().item()
    out = None
    for _ in range(2):  # consecutive calls share the static scratch array
        out = torch.full_like(v, float("nan"))
        assert _noalloc(s, v.data_ptr(), out.data_ptr(), prec, stream) == 0
        torch.cuda.synchronize()
        assert not torch.isnan(out).any().item()
        assert (out - ref).abs().max().item() <= tol
    return out


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
        out = _check_two_calls(s, v, ref, prec, st.cuda_stream)
    golden = g["sigma"][0]
    tol = TOL[prec] * np.abs(golden).max()
    assert np.abs(out.double().cpu().numpy() - golden).max() <= 2 * tol


# CAS(10,10), FCI(12e,12o) (853 776 determinants) and FCI(14e,14o) (11 778 624
# determinants, Nbeta = 3432 > 2048: the row kernel's wider default shape)
@pytest.mark.parametrize("n", [10, 12, 14])
@pytest.mark.parametrize("prec", [jb.FP64, jb.FP32])
def test_noalloc_first_call_allocates_nothing(n, prec):
    """The noalloc call is the first sigma on a freshly built space; device
    free memory is read before and after it.  A space of the same shape is
    run first so that the kernels this shape uses are already loaded (the
    CUDA runtime loads a kernel's code on its first launch, which is the
    library's code, not an allocation made by the call)."""
    import torch
    warm = _cas(n, 1)
    wv = _vector(warm.ndets, prec, 5)
    wo = torch.empty_like(wv)
    assert _noalloc(warm, wv.data_ptr(), wo.data_ptr(), prec, 0) == 0
    torch.cuda.synchronize()
    del wv, wo
    warm.close()

    s = _cas(n, 2)
    v = _vector(s.ndets, prec, 6)
    out = torch.full_like(v, float("nan"))
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    rc = _noalloc(s, v.data_ptr(), out.data_ptr(), prec, 0)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert rc == 0
    assert free1 == free0, f"free device memory moved by {free0 - free1} bytes"
    ref = torch.empty_like(v)
    s.sigma_device(v.data_ptr(), ref.data_ptr(), 1, s.ndets, prec, 0)
    torch.cuda.synchronize()
    tol = (1 if prec == jb.FP64 else 2) * TOL[prec] * ref.abs().max().item()
    assert (out - ref).abs().max().item() <= tol
    _check_two_calls(s, v, ref, prec, 0)
    s.close()


# (mode, threads, rows, batch) as jci_sigma_set_plan takes them, with the edge
# thread counts of each kernel; the noalloc call must pick its own row-kernel
# shape whatever plan the space was left with
PLANS = [(0, 128, 2, 1), (0, 512, 4, 1), (1, 128, 0, 1), (1, 1024, 0, 1), (2, 256, 0, 2),
         (3, 128, 0, 1024), (3, 1024, 0, 128), (4, 512, 16, 512), (5, 256, 8, 1),
         (6, 128, 0, 2), (6, 1024, 0, 1), (7, 512, 16, 3), (7, 128, 8, 4),
         # compact panel, hole-string doubles (5, 6) and beta singles (threads 0)
         (6, 512, 66, 5), (6, 0, 68, 6), (7, 0, 16, 5)]


@pytest.mark.parametrize("prec", [jb.FP64, jb.FP32])
def test_noalloc_after_every_forced_plan(prec):
    """FCI(14e,14o): every admissible forced plan, then noalloc against
    jci_sigma_device under that plan; in FP32 also against the FP64 sigma
    of the same vector at the FP32 bar."""
    import torch
    s = _cas(14, 3)
    v = _vector(s.ndets, prec, 9)
    ref = torch.empty_like(v)
    v64 = v.double()
    exact = torch.empty_like(v64)
    s.sigma_device(v64.data_ptr(), exact.data_ptr(), 1, s.ndets, jb.FP64, 0)
    torch.cuda.synchronize()
    bar = TOL[prec] * exact.abs().max().item()
    ran = 0
    for mode, nt, rows, batch in PLANS:
        try:
            s.set_sigma_plan(prec, mode, nt, rows, batch)
        except jb.JciError as e:
            assert e.status == 1, (mode, nt, rows, batch, e)
            continue
        ref.fill_(float("nan"))
        s.sigma_device(v.data_ptr(), ref.data_ptr(), 1, s.ndets, prec, 0)
        torch.cuda.synchronize()
        out = _check_two_calls(s, v, ref, prec, 0)
        assert (out.double() - exact).abs().max().item() <= bar
        ran += 1
    assert ran >= 10
    s.close()


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
