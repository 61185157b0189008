"""Davidson solves on the GPU against the reference's energies (needs a GPU).

Bars: FP64 energies within 1e-10 Eh of the reference, |<c_ref|c>| > 1-1e-9;
mixed FP32->FP64 energies within 1e-8 Eh.
"""
import ctypes
import glob
import os

import numpy as np
import pytest

import jayci_b200 as jb
from jayci_b200.synth import workload_integrals
from oracle.oracle import OracleSpace

pytestmark = pytest.mark.gpu

GOLDEN = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
                if not os.path.basename(p).startswith(("dyson_", "bench_")))
NAMES = [os.path.basename(p)[:-4] for p in GOLDEN]


def load(name):
    return np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))


def space_for(g):
    e, o, nfc, nd, na, nfv, x = (int(v) for v in g["general"])
    s = jb.Space(e, o, nfc, nd, na, nfv, x)
    s.set_integrals(g["m1"], g["m2"], float(g["e_nuc"]), 0.0)
    return s


def check(res, g, tol=1e-10, ovl=1e-9):
    np.testing.assert_allclose(res.energies, g["energies"], rtol=0, atol=tol)
    ov = np.abs(np.einsum("ij,ij->i", res.civec, g["civec"]))
    assert (ov > 1 - ovl).all(), ov


@pytest.mark.parametrize("name", NAMES)
def test_reference_schedule_fp64(name):
    g = load(name)
    s = space_for(g)
    kmin, kmax, nroots, refdim = (int(x) for x in g["dav_opts"])
    r = s.davidson(maxiter=500, krymin=kmin, krymax=kmax, nroots=nroots, refdim=refdim,
                   restol=1e-9)
    assert r.converged
    check(r, g)


@pytest.mark.parametrize("name", NAMES)
def test_block_fp64(name):
    g = load(name)
    s = space_for(g)
    kmin, kmax, nroots, refdim = (int(x) for x in g["dav_opts"])
    r = s.davidson(maxiter=500, krymin=kmin, krymax=kmax, nroots=nroots, refdim=refdim,
                   restol=1e-9, block=True)
    assert r.converged
    check(r, g)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("block", [False, True])
def test_mixed_precision(name, block):
    g = load(name)
    s = space_for(g)
    kmin, kmax, nroots, refdim = (int(x) for x in g["dav_opts"])
    r = s.davidson(maxiter=500, krymin=kmin, krymax=kmax, nroots=nroots, refdim=refdim,
                   restol=1e-9, precision=jb.MIXED, block=block)
    assert r.converged
    assert r.stats.fp32_sigma_vectors > 0
    check(r, g, tol=1e-8, ovl=1e-8)


def test_fci12_three_roots_all_schedules_agree():
    """The 853 776-determinant FCI(12e,12o), 3 roots: the reference schedule
    (FP64), block FP64 and block mixed solves agree, and each FP64 result
    vector satisfies ||H c - E c|| below the residual tolerance."""
    ints = workload_integrals("fci12_12")
    m1, m2 = ints.packed()
    s = jb.Space(12, 12)
    s.set_integrals(m1, m2, ints.e_nuc, 0.0)
    base = s.davidson(maxiter=2000, krymin=6, krymax=24, nroots=3, refdim=12, restol=1e-8)
    assert base.converged
    for prec, block, tol in [(jb.FP64, True, 1e-10), (jb.MIXED, True, 1e-8),
                             (jb.MIXED, False, 1e-8)]:
        r = s.davidson(maxiter=2000, krymin=6, krymax=24, nroots=3, refdim=12,
                       restol=1e-8, precision=prec, block=block)
        assert r.converged
        np.testing.assert_allclose(r.energies, base.energies, rtol=0, atol=tol)
        ov = np.abs(np.einsum("ij,ij->i", r.civec, base.civec))
        assert (ov > 1 - 1e-8).all()
    S = s.sigma(base.civec)
    res = S - (base.energies - ints.e_nuc)[:, None] * base.civec
    assert np.linalg.norm(res, axis=1).max() < 2e-8


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("prec", [jb.FP64, jb.MIXED])
def test_graph_iterations_match_host_loop(name, prec):
    """The CUDA-graph iterations (control state on the device, batches of
    launches) and the host-driven iterations run the same kernels in the same
    order: energies, vectors and iteration counts are bitwise equal."""
    g = load(name)
    s = space_for(g)
    kmin, kmax, nroots, refdim = (int(x) for x in g["dav_opts"])
    kw = dict(maxiter=500, krymin=kmin, krymax=kmax, nroots=nroots, refdim=refdim,
              restol=1e-9, precision=prec)
    rg = s.davidson(**kw)
    rh = s.davidson(host_loop=True, **kw)
    assert rg.converged and rh.converged
    assert rg.stats.iterations == rh.stats.iterations
    assert rg.stats.sigma_vectors == rh.stats.sigma_vectors
    np.testing.assert_array_equal(rg.energies, rh.energies)
    np.testing.assert_array_equal(rg.civec, rh.civec)
    check(rg, g, tol=1e-10 if prec == jb.FP64 else 1e-8, ovl=1e-9 if prec == jb.FP64 else 1e-8)


def test_graph_iterations_fci12():
    """853 776 determinants, 3 roots: graph and host-driven reference
    schedules agree bitwise."""
    ints = workload_integrals("fci12_12")
    m1, m2 = ints.packed()
    s = jb.Space(12, 12)
    s.set_integrals(m1, m2, ints.e_nuc, 0.0)
    kw = dict(maxiter=500, krymin=6, krymax=24, nroots=3, refdim=12, restol=1e-8)
    rg = s.davidson(**kw)
    rh = s.davidson(host_loop=True, **kw)
    assert rg.converged and rh.converged
    assert rg.stats.iterations == rh.stats.iterations
    np.testing.assert_array_equal(rg.energies, rh.energies)
    np.testing.assert_array_equal(rg.civec, rh.civec)


def test_restart_from_files(tmp_path, monkeypatch):
    """civec / ci.restart written like the reference; prediagr=3 restarts."""
    g = load("cas6_6")
    s = space_for(g)
    monkeypatch.chdir(tmp_path)
    r = s.davidson(maxiter=3, krymin=4, krymax=6, nroots=2, refdim=8, restol=1e-12,
                   write_files=True)
    assert not r.converged
    assert os.path.exists("civec") and os.path.exists("ci.restart")
    assert os.path.exists("hvvec")
    r2 = s.davidson(maxiter=500, krymin=4, krymax=10, nroots=2, prediagr=3, restol=1e-9,
                    write_files=True)
    assert r2.converged
    check(r2, g)
    civ = jb.read_vectors("civec", 2, s.ndets)
    np.testing.assert_array_equal(civ, r2.civec)


def _ref_structs(g):
    """Build reference-layout struct occstr / eospace arrays from golden data."""
    sizes = [int(x) for x in g["sizes"]]
    out = []
    for sp in (0, 1):
        istr = g[f"istr{sp}"]
        arr = (jb_occstr * istr.shape[0])()
        for i in range(istr.shape[0]):
            arr[i].byte1 = int(g[f"byte1_{sp}"][i])
            for k in range(istr.shape[1]):
                arr[i].istr[k] = int(istr[i, k])
        eo = g[f"eosp{sp}"]
        earr = (jb_eospace * eo.shape[0])()
        for k in range(eo.shape[0]):
            earr[k].docc, earr[k].actv, earr[k].virt = (int(x) for x in eo[k, :3])
            earr[k].nstr, earr[k].start = int(eo[k, 3]), int(eo[k, 4])
        out.append((arr, earr, eo.shape[0]))
    pq = g["pq"]
    rows = [(ctypes.c_int * 2)(int(a), int(b)) for a, b in pq]
    pqp = (ctypes.POINTER(ctypes.c_int) * len(rows))(
        *[ctypes.cast(r, ctypes.POINTER(ctypes.c_int)) for r in rows])
    return out, pqp, rows, sizes


class jb_occstr(ctypes.Structure):
    _fields_ = [("byte1", ctypes.c_longlong), ("virtx", ctypes.c_int * 2),
                ("nvrtx", ctypes.c_int), ("istr", ctypes.c_int * 20),
                ("yij", (ctypes.c_int * 200) * 20), ("cij", (ctypes.c_int * 200) * 20)]


class jb_eospace(ctypes.Structure):
    _fields_ = [("docc", ctypes.c_int), ("actv", ctypes.c_int), ("virt", ctypes.c_int),
                ("nstr", ctypes.c_int), ("start", ctypes.c_int),
                ("pairs", ctypes.c_int * 20), ("npairs", ctypes.c_int)]


@pytest.mark.parametrize("name", ["cas6_6", "trunc6_8_x2"])
def test_pdavidson_drop_in(name, tmp_path, monkeypatch):
    """jci_pdavidson called with the reference's own argument list."""
    g = load(name)
    (pa, pe, ng_p), (qa, qe, ng_q) = _ref_structs(g)[0]
    _, pqp, keep, sizes = _ref_structs(g)
    na, nb, norb, nastr, nbstr, pegrps, qegrps, npq, ndets = sizes
    e, o, nfc, nd, nact, nfv, x = (int(v) for v in g["general"])
    kmin, kmax, nroots, refdim = (int(v) for v in g["dav_opts"])
    m1 = np.ascontiguousarray(g["m1"])
    m2 = np.ascontiguousarray(g["m2"])
    L = jb.lib()
    f = L.jci_pdavidson
    f.restype = ctypes.c_int
    monkeypatch.chdir(tmp_path)
    rc = f(pa, pe, ng_p, qa, qe, ng_q, pqp, npq, m1.ctypes.data_as(ctypes.c_void_p),
           m2.ctypes.data_as(ctypes.c_void_p), na, nb, nd + nact, ndets,
           ctypes.c_double(float(g["e_nuc"])), ctypes.c_double(0.0), 0, 500, kmin, kmax,
           nroots, 1, refdim, ctypes.c_double(1e-9), 0, norb, nd, nact)
    assert rc == 0
    civ = jb.read_vectors("civec", nroots, ndets)
    ov = np.abs(np.einsum("ij,ij->i", civ, g["civec"]))
    assert (ov > 1 - 1e-9).all()


def test_jci_program_end_to_end(tmp_path):
    """The jci driver reads jayci.in + a SIFS moints file like pjayci and
    writes civec (execute_pjayci.c flow on one GPU)."""
    import subprocess
    g = load("cas6_6")
    kmin, kmax, nroots, refdim = (int(x) for x in g["dav_opts"])
    (tmp_path / "jayci.in").write_text(
        f" &general\n electrons=6, orbitals=6, nfrozen=0, ndocc=0, nactive=6, xlevel=0\n /\n"
        f" &dalginfo\n maxiter=500, krymin={kmin}, krymax={kmax}, nroots={nroots},\n"
        f" prediagr=1, restol=1.0d-9, refdim={refdim}\n /\n &gpuinfo exactrestol=1 /\n")
    jb.write_moints(tmp_path / "moints", 6, g["m1"], g["m2"], float(g["e_nuc"]), 0.0)
    exe = os.path.join(os.path.dirname(jb.LIBPATH), "jci")
    if not os.path.exists(exe):
        from jayci_b200 import build
        build.build()
    r = subprocess.run([exe], cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    e = [float(l.split()[-1]) for l in r.stdout.splitlines() if "Root #" in l]
    np.testing.assert_allclose(e, g["energies"], atol=1e-10)
    civ = jb.read_vectors(str(tmp_path / "civec"), nroots, 400)
    ov = np.abs(np.einsum("ij,ij->i", civ, g["civec"]))
    assert (ov > 1 - 1e-9).all()
