"""jayci_b200 -- Python host mirror of the libjci C ABI (include/jci.h).

The engine itself is the in-tree shared library ``libjci.so`` (C++ host code
plus sm_100a CUDA kernels).  This module binds it with ctypes and mirrors the
reference's interface for the determinant-CI hot path:

* :class:`Space` -- ``citrunc`` (string space), ``generate_*_excitations``,
  ``compute_diagonal_iHi``, sigma (``perform_hvispacefast``) and the
  Davidson solve (``pdavidson``);
* :func:`read_moints` / :func:`write_moints` -- SIFS integrals
  (``readmoints.f90``);
* :func:`read_namelists` -- ``jayci.in`` (``readgeninput`` /
  ``readdaiinput``);
* :func:`write_vectors` / :func:`read_vectors` -- civec / ci.restart.

There is no CPU fallback: every call fails loudly (:class:`JciError`) when
the library or a CUDA device is missing.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libjci.so")

FP64, FP32, MIXED = 0, 1, 2

STATUS = {0: "ok", 1: "invalid argument", 2: "CI space outside the supported limits",
          3: "out of memory", 4: "CUDA runtime error", 5: "no CUDA device",
          6: "file I/O error", 7: "malformed input file", 8: "not converged",
          9: "subspace eigensolve failed", 10: "bounded device wait expired",
          11: "server admission refused", 12: "call out of order"}
NOCONV = 8


class JciError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        super().__init__(f"libjci {what}: {STATUS.get(status, status)} ({status})")


class DavidsonOpts(ctypes.Structure):
    _fields_ = [("maxiter", ctypes.c_int), ("krymin", ctypes.c_int),
                ("krymax", ctypes.c_int), ("nroots", ctypes.c_int),
                ("prediagr", ctypes.c_int), ("refdim", ctypes.c_int),
                ("restol", ctypes.c_double), ("precision", ctypes.c_int),
                ("switch_tol", ctypes.c_double), ("printlvl", ctypes.c_int),
                ("write_files", ctypes.c_int), ("block", ctypes.c_int),
                ("init", ctypes.c_void_p), ("host_loop", ctypes.c_int)]


class DavidsonStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("sigma_calls", ctypes.c_int),
                ("sigma_vectors", ctypes.c_longlong), ("sigma_seconds", ctypes.c_double),
                ("total_seconds", ctypes.c_double), ("converged", ctypes.c_int),
                ("rnorm", ctypes.c_double), ("fp32_sigma_vectors", ctypes.c_int)]


class General(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int) for k in ("electrons", "orbitals", "nfrozen", "ndocc",
                                           "nactive", "xlevel", "nfrzvirt", "printlvl",
                                           "printwvf")]


class Dalginfo(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int) for k in ("maxiter", "krymin", "krymax", "nroots",
                                           "prediagr", "refdim", "buflen")] + \
        [("restol", ctypes.c_double)]


class Gpuinfo(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("switch_tol", ctypes.c_double),
                ("block", ctypes.c_int), ("exact_restol", ctypes.c_int)]


_lib = None


def lib():
    """Load libjci.so (building it first if it is absent)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            from . import build as _b
            _b.build()
        L = ctypes.CDLL(LIBPATH)
        vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.jci_status_string.restype = ctypes.c_char_p
        L.jci_space_create.argtypes = [ip] * 7 + [ctypes.POINTER(vp)]
        L.jci_space_destroy.argtypes = [vp]
        L.jci_space_sizes.argtypes = [vp, vp]
        L.jci_space_strings.argtypes = [vp, ip, vp]
        L.jci_space_eospaces.argtypes = [vp, ip, vp]
        L.jci_space_pq.argtypes = [vp, vp]
        L.jci_space_string_index.argtypes = [vp, ip, vp, ctypes.POINTER(ip)]
        L.jci_space_excitations.argtypes = [vp, ip, ip, ip, ip, vp, ctypes.POINTER(ip)]
        L.jci_set_integrals.argtypes = [vp, vp, vp, ip, dp, dp]
        L.jci_hdiag.argtypes = [vp, vp]
        L.jci_sigma.argtypes = [vp, ip, vp, vp, ip]
        L.jci_sigma_device.argtypes = [vp, ip, vp, vp, ctypes.c_longlong, ip, vp]
        L.jci_davidson_defaults.argtypes = [ctypes.POINTER(DavidsonOpts)]
        L.jci_davidson.argtypes = [vp, ctypes.POINTER(DavidsonOpts), vp, vp,
                                   ctypes.POINTER(DavidsonStats)]
        L.jci_sigma_tuning.argtypes = [vp, ip, ctypes.POINTER(ip), ctypes.POINTER(ip),
                                       ctypes.POINTER(ip), ctypes.POINTER(ip),
                                       ctypes.POINTER(ctypes.c_float)]
        L.jci_sigma_set_plan.argtypes = [vp, ip, ip, ip, ip, ip]
        L.jci_read_namelists.argtypes = [ctypes.c_char_p, vp, vp, vp]
        L.jci_read_moints.argtypes = [ctypes.c_char_p, vp, ctypes.c_longlong, vp,
                                      ctypes.c_longlong, ctypes.POINTER(ip),
                                      ctypes.POINTER(dp), ctypes.POINTER(dp)]
        L.jci_write_moints.argtypes = [ctypes.c_char_p, ip, vp, vp, dp, dp]
        L.jci_write_vectors.argtypes = [ctypes.c_char_p, ip, ip, vp]
        L.jci_read_vectors.argtypes = [ctypes.c_char_p, ip, ip, vp]
        L.jci_read_dycicalc.argtypes = [ctypes.c_char_p, vp, vp, vp, ctypes.POINTER(ip), vp,
                                        ctypes.POINTER(ip)]
        L.jci_dyson.argtypes = [vp, vp, vp, ip, vp, ip, vp, ip, vp, ip, vp]
        L.jci_write_dysonorb.argtypes = [ctypes.c_char_p, ip, ip, vp, vp, ip, vp, ip]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _check(st, what):
    if st != 0:
        raise JciError(st, what)


def device_count() -> int:
    return lib().jci_device_count()


@dataclass
class SolveResult:
    energies: np.ndarray
    civec: np.ndarray | None
    stats: DavidsonStats
    converged: bool


class Space:
    """Truncated alpha/beta CI string space (citrunc, citruncate.c:55) with
    its device tables.  Arguments are the &general namelist values."""

    def __init__(self, electrons, orbitals, nfrozen=0, ndocc=0, nactive=None,
                 nfrzvirt=0, xlevel=0):
        if nactive is None:
            nactive = orbitals - nfrozen - nfrzvirt - ndocc
        h = ctypes.c_void_p()
        _check(lib().jci_space_create(electrons, orbitals, nfrozen, ndocc, nactive,
                                      nfrzvirt, xlevel, ctypes.byref(h)), "space_create")
        self.h = h
        sz = np.zeros(10, np.int64)
        lib().jci_space_sizes(h, _p(sz))
        (self.na, self.nb, self.norb, self.nastr, self.nbstr, self.pegrps,
         self.qegrps, self.npq, self.ndets, self.intorb) = (int(x) for x in sz)
        self.ndocc, self.nactv, self.xlvl = ndocc, nactive, xlevel
        self.electrons, self.orbitals = electrons, orbitals

    def close(self):
        if getattr(self, "h", None):
            try:
                lib().jci_space_destroy(self.h)
            except Exception:  # interpreter shutdown
                pass
            self.h = None

    __del__ = close

    def strings(self, spin):
        ns, ne = (self.nastr, self.na) if spin == 0 else (self.nbstr, self.nb)
        out = np.zeros(ns * ne, np.int32)
        _check(lib().jci_space_strings(self.h, spin, _p(out)), "strings")
        return out.reshape(ns, ne)

    def eospaces(self, spin):
        ng = self.pegrps if spin == 0 else self.qegrps
        out = np.zeros(5 * ng, np.int32)
        _check(lib().jci_space_eospaces(self.h, spin, _p(out)), "eospaces")
        return out.reshape(ng, 5)

    def pq(self):
        out = np.zeros(2 * self.npq, np.int32)
        _check(lib().jci_space_pq(self.h, _p(out)), "pq")
        return out.reshape(self.npq, 2)

    def string_index(self, spin, orbs):
        o = np.ascontiguousarray(orbs, np.int32)
        idx = ctypes.c_int()
        _check(lib().jci_space_string_index(self.h, spin, _p(o), ctypes.byref(idx)),
               "string_index")
        return idx.value

    def excitations(self, spin, nrep, istr, teosp):
        ns = self.nastr if spin == 0 else self.nbstr
        out = np.zeros(6 * (ns + 1), np.int32)
        n = ctypes.c_int()
        _check(lib().jci_space_excitations(self.h, spin, nrep, istr, teosp, _p(out),
                                           ctypes.byref(n)), "excitations")
        return out[: 6 * n.value].reshape(n.value, 6)

    def set_integrals(self, moints1, moints2, nucrep=0.0, frzcore=0.0):
        self._m1 = np.ascontiguousarray(moints1, np.float64)
        self._m2 = np.ascontiguousarray(moints2, np.float64)
        _check(lib().jci_set_integrals(self.h, _p(self._m1), _p(self._m2), self.norb,
                                       nucrep, frzcore), "set_integrals")

    def hdiag(self):
        out = np.zeros(self.ndets)
        _check(lib().jci_hdiag(self.h, _p(out)), "hdiag")
        return out

    def sigma(self, v, precision=FP64):
        v = np.ascontiguousarray(np.atleast_2d(v), np.float64)
        out = np.zeros_like(v)
        _check(lib().jci_sigma(self.h, v.shape[0], _p(v), _p(out), precision), "sigma")
        return out

    def sigma_device(self, v_ptr, s_ptr, nvec, ld, precision=FP64, stream=None):
        """sigma on device buffers (e.g. torch tensors' data_ptr())."""
        _check(lib().jci_sigma_device(self.h, nvec, ctypes.c_void_p(v_ptr),
                                      ctypes.c_void_p(s_ptr), ld, precision,
                                      ctypes.c_void_p(stream or 0)), "sigma_device")

    def sigma_tuning(self, precision=FP64):
        """(mode, threads, rows, batch, ms per vector) chosen by the autotuner,
        with the meanings of jci_sigma_tuning (include/jci.h)."""
        m, a, b, g, c = (ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int(),
                         ctypes.c_float())
        _check(lib().jci_sigma_tuning(self.h, precision, ctypes.byref(m), ctypes.byref(a),
                                      ctypes.byref(b), ctypes.byref(g), ctypes.byref(c)),
               "sigma_tuning")
        return m.value, a.value, b.value, g.value, c.value

    def set_sigma_plan(self, precision, mode, threads, rows=1, batch=1):
        """Fix the FCI sigma plan (modes 0-7 of jci_sigma_set_plan)."""
        _check(lib().jci_sigma_set_plan(self.h, precision, mode, threads, rows, batch),
               "sigma_set_plan")

    def davidson(self, maxiter=500, krymin=4, krymax=12, nroots=1, prediagr=1,
                 refdim=8, restol=1e-8, precision=FP64, switch_tol=1e-4,
                 block=False, printlvl=0, write_files=False, init=None,
                 want_vectors=True, host_loop=False) -> SolveResult:
        o = DavidsonOpts()
        lib().jci_davidson_defaults(ctypes.byref(o))
        o.maxiter, o.krymin, o.krymax, o.nroots = maxiter, krymin, krymax, nroots
        o.prediagr, o.refdim, o.restol = prediagr, refdim, restol
        o.precision, o.switch_tol, o.block = precision, switch_tol, int(block)
        o.printlvl, o.write_files = printlvl, int(write_files)
        o.host_loop = int(host_loop)
        if init is not None:
            init = np.ascontiguousarray(init, np.float64)
            o.init = init.ctypes.data
        e = np.zeros(nroots)
        civ = np.zeros((nroots, self.ndets)) if want_vectors else None
        st = DavidsonStats()
        r = lib().jci_davidson(self.h, ctypes.byref(o), _p(e),
                               _p(civ) if civ is not None else None, ctypes.byref(st))
        if r not in (0, NOCONV):
            raise JciError(r, "davidson")
        return SolveResult(e, civ, st, r == 0)


MAX_ROOTS = 16


class Request(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int) for k in ("electrons", "orbitals", "nfrozen", "ndocc",
                                           "nactive", "nfrzvirt", "xlevel")] + [
        ("moints1", ctypes.c_void_p), ("moints2", ctypes.c_void_p),
        ("nucrep", ctypes.c_double), ("frzcore", ctypes.c_double)] + [
        (k, ctypes.c_int) for k in ("nroots", "krymin", "krymax", "maxiter", "refdim")] + [
        ("restol", ctypes.c_double), ("precision", ctypes.c_int),
        ("switch_tol", ctypes.c_double), ("block", ctypes.c_int),
        ("warm_from", ctypes.c_longlong)]


class Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("converged", ctypes.c_int),
                ("nroots", ctypes.c_int), ("energies", ctypes.c_double * MAX_ROOTS),
                ("iterations", ctypes.c_int), ("warm_started", ctypes.c_int),
                ("ndets", ctypes.c_longlong), ("queue_seconds", ctypes.c_double),
                ("solve_seconds", ctypes.c_double), ("sigma_vectors", ctypes.c_longlong),
                ("sigma_seconds", ctypes.c_double)]


class Server:
    """Continuous-batching CI solve server (jci_server_*): `slots` solves in
    flight, admitted by estimated HBM footprint within `budget_bytes`."""

    def __init__(self, budget_bytes=0, slots=4):
        L = lib()
        vp = ctypes.c_void_p
        L.jci_server_create.argtypes = [ctypes.c_size_t, ctypes.c_int, ctypes.POINTER(vp)]
        L.jci_server_submit.argtypes = [vp, ctypes.POINTER(Request),
                                        ctypes.POINTER(ctypes.c_longlong)]
        L.jci_server_wait.argtypes = [vp, ctypes.c_longlong, ctypes.c_double,
                                      ctypes.POINTER(Result)]
        L.jci_server_vectors.argtypes = [vp, ctypes.c_longlong, vp]
        L.jci_server_release.argtypes = [vp, ctypes.c_longlong]
        L.jci_server_destroy.argtypes = [vp]
        h = vp()
        _check(L.jci_server_create(budget_bytes, slots, ctypes.byref(h)), "server_create")
        self.h = h
        self._ndets = {}

    def submit(self, general, moints1, moints2, nucrep=0.0, frzcore=0.0, nroots=1,
               krymin=None, krymax=24, maxiter=1000, refdim=8, restol=1e-8,
               precision=FP64, switch_tol=1e-4, block=True, warm_from=-1):
        """general = (electrons, orbitals, nfrozen, ndocc, nactive, nfrzvirt, xlevel)."""
        m1 = np.ascontiguousarray(moints1, np.float64)
        m2 = np.ascontiguousarray(moints2, np.float64)
        r = Request(*general, m1.ctypes.data, m2.ctypes.data, nucrep, frzcore, nroots,
                    krymin or max(nroots, 4), krymax, maxiter, refdim, restol, precision,
                    switch_tol, int(block), warm_from)
        t = ctypes.c_longlong()
        _check(lib().jci_server_submit(self.h, ctypes.byref(r), ctypes.byref(t)), "submit")
        self._ndets[t.value] = None
        return t.value

    def wait(self, ticket, timeout=-1.0):
        res = Result()
        _check(lib().jci_server_wait(self.h, ticket, timeout, ctypes.byref(res)), "wait")
        self._ndets[ticket] = res.ndets
        return res

    def vectors(self, ticket, nroots):
        n = self._ndets.get(ticket)
        if n is None:
            n = self.wait(ticket).ndets
        out = np.zeros((nroots, n))
        _check(lib().jci_server_vectors(self.h, ticket, _p(out)), "vectors")
        return out

    def release(self, ticket):
        _check(lib().jci_server_release(self.h, ticket), "release")
        self._ndets.pop(ticket, None)

    def close(self):
        if getattr(self, "h", None):
            try:
                lib().jci_server_destroy(self.h)
            except Exception:
                pass
            self.h = None

    __del__ = close


def read_namelists(path):
    g, d, u = General(), Dalginfo(), Gpuinfo()
    _check(lib().jci_read_namelists(str(path).encode(), ctypes.byref(g), ctypes.byref(d),
                                    ctypes.byref(u)), "read_namelists")
    return g, d, u


def moint_sizes(norb):
    m1 = norb * (norb + 1) // 2
    return m1, m1 * (m1 + 1) // 2


def sifs_nbft(path):
    """Orbital count from SIFS header 1 (seven INTEGER*8, readmoints.f90:101)."""
    try:
        with open(path, "rb") as f:
            head = f.read(4 + 56)
    except OSError:
        raise JciError(6, "read_moints") from None
    if len(head) < 60:
        raise JciError(7, "read_moints")
    return int(np.frombuffer(head[4:60], np.int64)[3])


def read_moints(path, path2=None):
    """SIFS integrals -> (moints1, moints2, nbft, nucrep, frzcore).  Files
    with fsplit = 2 take their 2-e records from path2 (default: path + "2")."""
    m1len, m2len = moint_sizes(sifs_nbft(path))
    m1 = np.zeros(m1len)
    m2 = np.zeros(m2len)
    nb, en, fc = ctypes.c_int(), ctypes.c_double(), ctypes.c_double()
    if path2 is None:
        st = lib().jci_read_moints(str(path).encode(), _p(m1), m1len, _p(m2), m2len,
                                   ctypes.byref(nb), ctypes.byref(en), ctypes.byref(fc))
    else:
        f = lib().jci_read_moints_split
        f.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_longlong,
                      ctypes.c_void_p, ctypes.c_longlong, ctypes.POINTER(ctypes.c_int),
                      ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
        st = f(str(path).encode(), str(path2).encode(), _p(m1), m1len, _p(m2), m2len,
               ctypes.byref(nb), ctypes.byref(en), ctypes.byref(fc))
    _check(st, "read_moints")
    a, b = moint_sizes(nb.value)
    return m1[:a].copy(), m2[:b].copy(), nb.value, en.value, fc.value


def write_moints(path, nbft, moints1, moints2, nucrep, frzcore=0.0, path2=None):
    """Write SIFS integrals; with path2 the file has fsplit = 2 and its 2-e
    records go to path2."""
    m1 = np.ascontiguousarray(moints1, np.float64)
    m2 = np.ascontiguousarray(moints2, np.float64)
    if path2 is None:
        st = lib().jci_write_moints(str(path).encode(), nbft, _p(m1), _p(m2), nucrep, frzcore)
    else:
        f = lib().jci_write_moints_split
        f.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_void_p,
                      ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
        st = f(str(path).encode(), str(path2).encode(), nbft, _p(m1), _p(m2), nucrep, frzcore)
    _check(st, "write_moints")


def write_vectors(path, v):
    v = np.ascontiguousarray(np.atleast_2d(v), np.float64)
    _check(lib().jci_write_vectors(str(path).encode(), v.shape[0], v.shape[1], _p(v)),
           "write_vectors")


def read_vectors(path, dim, length):
    v = np.zeros((dim, length))
    _check(lib().jci_read_vectors(str(path).encode(), dim, length, _p(v)), "read_vectors")
    return v


class Wavefcn(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int) for k in ("electrons", "orbitals", "nfrozen", "ndocc",
                                           "nactive", "nfrzvirt", "xlevel", "nstates")]

    def general(self):
        return (self.electrons, self.orbitals, self.nfrozen, self.ndocc, self.nactive,
                self.nfrzvirt, self.xlevel)


def read_dycicalc(path):
    """dycicalc.in: (wavefcn0, wavefcn1, states0, states1), states 1-based
    and truncated after the last nonzero entry as the reference counts."""
    w0, w1 = Wavefcn(), Wavefcn()
    s0, s1 = np.zeros(5, np.int32), np.zeros(5, np.int32)
    n0, n1 = ctypes.c_int(0), ctypes.c_int(0)
    _check(lib().jci_read_dycicalc(str(path).encode(), ctypes.byref(w0), ctypes.byref(w1),
                                   _p(s0), ctypes.byref(n0), _p(s1), ctypes.byref(n1)),
           "read_dycicalc")
    return w0, w1, s0[:n0.value].copy(), s1[:n1.value].copy()


def dyson(space0, space1, v0, v1, states0=(1,), states1=(1,)):
    """Dyson orbitals between the (N+1)-electron space0 and the N-electron
    space1 (jci_dyson): (len(states0) * len(states1)) x orbitals."""
    v0 = np.ascontiguousarray(np.atleast_2d(v0), np.float64)
    v1 = np.ascontiguousarray(np.atleast_2d(v1), np.float64)
    st0 = np.ascontiguousarray(states0, np.int32)
    st1 = np.ascontiguousarray(states1, np.int32)
    out = np.zeros((len(st0) * len(st1), space0.orbitals))
    _check(lib().jci_dyson(space0.h, space1.h, _p(v0), v0.shape[0], _p(v1), v1.shape[0],
                           _p(st0), len(st0), _p(st1), len(st1), _p(out)), "dyson")
    return out


def write_dysonorb(path, dyorb, states0, states1):
    dyorb = np.ascontiguousarray(np.atleast_2d(dyorb), np.float64)
    st0 = np.ascontiguousarray(states0, np.int32)
    st1 = np.ascontiguousarray(states1, np.int32)
    _check(lib().jci_write_dysonorb(str(path).encode(), dyorb.shape[0], dyorb.shape[1],
                                    _p(dyorb), _p(st0), len(st0), _p(st1), len(st1)),
           "write_dysonorb")
