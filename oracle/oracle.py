"""ctypes bindings for the CPU oracle libraries.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()``
and bench.py's CPU-baseline leg as the checker; the product package never
imports this module.

* :class:`OracleSpace` wraps ``liboracle.so`` -- the C restatement of the
  reference algorithm (jci_oracle.c).
* :class:`RefSpace` wraps ``_ref/libjayci_ref.so`` -- the reference's own
  mpi_source C code compiled unchanged against a single-process GA/MPI
  stand-in (only present where the reference tree was available at build
  time; see Makefile).
* :func:`ref_serial_solve` wraps ``_ref/libjayci_serial.so`` -- the
  reference's serial source/ path (the jayci program) compiled unchanged.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libjayci_ref.so")
SERIAL_SO = os.path.join(HERE, "_ref", "libjayci_serial.so")

_c_int_p = ctypes.POINTER(ctypes.c_int)


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


REF_ENV = "JAYCI_REF"


def reference_tree():
    """The reference checkout named by the JAYCI_REF environment variable
    (the directory holding mpi_source/), or None when it is unset or absent."""
    root = os.environ.get(REF_ENV)
    if root and os.path.isfile(os.path.join(root, "mpi_source", "pdavidson.c")):
        return root
    return None


def build(ref: bool = True) -> None:
    """Compile the oracle libraries (make -C oracle): always the C
    restatement; with ref=True also the reference build, from the tree
    reference_tree() names (skipped when there is none)."""
    root = reference_tree() if ref else None
    target = ["all", f"REF={root}"] if root else ["liboracle.so"]
    subprocess.run(["make", "-s", "-C", HERE] + target, check=True)


def _load(path):
    if not os.path.exists(path):
        build(ref=path == REF_SO)
    return ctypes.CDLL(path)


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def serial_available() -> bool:
    return os.path.exists(SERIAL_SO)


_serial = None


def ref_serial_solve(general, m1, m2, nucrep, frzcore=0.0, maxiter=500, krymin=4,
                     krymax=12, nroots=1, prediagr=1, refdim=8, restol=1e-8, printlvl=0,
                     want_vectors=True):
    """The reference's serial jayci path (oracle/_ref/libjayci_serial.so,
    source/*.c compiled unchanged): citrunc_rtnlist, the O(N^2) cimap,
    compute_hdgls and dvdalg.  general = (electrons, orbitals, nfrozen,
    ndocc, nactive, nfrzvirt, xlevel).  Returns (energies including
    nucrep + frzcore, civec nroots x ndets or None, times {cimap, hdgls,
    dvdalg} in seconds)."""
    global _serial
    if _serial is None:
        if not os.path.exists(SERIAL_SO):
            raise FileNotFoundError(SERIAL_SO)
        L = ctypes.CDLL(SERIAL_SO)
        L.ref_serial_solve.restype = ctypes.c_longlong
        L.ref_serial_solve.argtypes = [ctypes.c_int] * 7 + [ctypes.c_void_p] * 2 + \
            [ctypes.c_double] * 2 + [ctypes.c_int] * 6 + [ctypes.c_double, ctypes.c_int] + \
            [ctypes.c_void_p] * 3
        _serial = L
    e, o, nfc, nd, na, nfv, x = (int(v) for v in general)
    ci_e = e - 2 * nfc
    sp = OracleSpace((ci_e + 1) // 2, ci_e // 2, o - nfc - nfv, nd, na, x)
    n = sp.ndets
    del sp
    m1 = np.ascontiguousarray(m1, float)
    m2 = np.ascontiguousarray(m2, float)
    en = np.zeros(nroots)
    civ = np.zeros((nroots, n)) if want_vectors else None
    times = np.zeros(3)
    r = _serial.ref_serial_solve(e, o, nfc, nd, na, nfv, x, _ptr(m1), _ptr(m2), nucrep,
                                 frzcore, maxiter, krymin, krymax, nroots, prediagr, refdim,
                                 restol, printlvl, _ptr(en),
                                 _ptr(civ) if civ is not None else None, _ptr(times))
    if r < 0:
        raise RuntimeError(f"reference serial solve failed ({r})")
    if r != n:
        raise RuntimeError(f"reference serial space has {r} determinants, expected {n}")
    return en, civ, dict(cimap=times[0], hdgls=times[1], dvdalg=times[2])


class OracleSpace:
    """String space + Slater-rule sigma + Davidson, restated in C."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = _load(ORACLE_SO)
            lib.jo_space_build.restype = ctypes.c_void_p
            lib.jo_space_build.argtypes = [ctypes.c_int] * 6
            lib.jo_space_free.argtypes = [ctypes.c_void_p]
            lib.jo_space_info.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            lib.jo_strings.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
            lib.jo_eospaces.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
            lib.jo_pq.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            lib.jo_string_index.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
            lib.jo_excitations.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
            lib.jo_hdiag.argtypes = [ctypes.c_void_p] * 4
            lib.jo_hmatel.restype = ctypes.c_double
            lib.jo_hmatel.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_longlong] * 2
            lib.jo_sigma.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
            lib.jo_davidson.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_double] + [ctypes.c_int] * 6 + [
                                        ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p]
            lib.jo_symeig.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p]
            cls._lib = lib
        return cls._lib

    def __init__(self, ci_aelec, ci_belec, ci_orbs, ndocc=0, nactv=None, xlvl=0):
        if nactv is None:
            nactv = ci_orbs - ndocc
        self.na, self.nb, self.norb = ci_aelec, ci_belec, ci_orbs
        self.ndocc, self.nactv, self.xlvl = ndocc, nactv, xlvl
        self.h = self.lib().jo_space_build(ci_aelec, ci_belec, ci_orbs, ndocc,
                                           nactv, xlvl)
        if not self.h:
            raise ValueError("oracle: invalid space")
        info = np.zeros(6, np.int64)
        self.lib().jo_space_info(self.h, _ptr(info))
        (self.nastr, self.nbstr, self.pegrps, self.qegrps, self.npq,
         self.ndets) = (int(x) for x in info)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib().jo_space_free(self.h)
            self.h = None

    def strings(self, spin):
        ns, ne = (self.nastr, self.na) if spin == 0 else (self.nbstr, self.nb)
        out = np.zeros(ns * ne, np.int32)
        self.lib().jo_strings(self.h, spin, _ptr(out))
        return out.reshape(ns, ne)

    def eospaces(self, spin):
        ng = self.pegrps if spin == 0 else self.qegrps
        out = np.zeros(5 * ng, np.int32)
        self.lib().jo_eospaces(self.h, spin, _ptr(out))
        return out.reshape(ng, 5)

    def pq(self):
        out = np.zeros(2 * self.npq, np.int32)
        self.lib().jo_pq(self.h, _ptr(out))
        return out.reshape(self.npq, 2)

    def excitations(self, spin, nrep, istr, teosp):
        ns = self.nastr if spin == 0 else self.nbstr
        out = np.zeros(6 * (ns + 1), np.int32)
        n = self.lib().jo_excitations(self.h, spin, nrep, istr, teosp, _ptr(out))
        return out[: 6 * n].reshape(n, 6)

    def hdiag(self, m1, m2):
        out = np.zeros(self.ndets)
        self.lib().jo_hdiag(self.h, _ptr(np.ascontiguousarray(m1, float)),
                            _ptr(np.ascontiguousarray(m2, float)), _ptr(out))
        return out

    def hmatel(self, m1, m2, i, j):
        return self.lib().jo_hmatel(self.h, _ptr(m1), _ptr(m2), i, j)

    def sigma(self, m1, m2, V):
        V = np.ascontiguousarray(np.atleast_2d(V), float)
        S = np.zeros_like(V)
        self.lib().jo_sigma(self.h, _ptr(m1), _ptr(m2), V.shape[0], _ptr(V), _ptr(S))
        return S

    def sigma_rows(self, m1, m2, v, rows):
        """(H v)[rows] for one vector v (ndets) at the listed determinants."""
        lib = self.lib()
        lib.jo_sigma_rows.argtypes = [ctypes.c_void_p] * 5 + [ctypes.c_longlong,
                                                              ctypes.c_void_p]
        v = np.ascontiguousarray(v, float)
        rows = np.ascontiguousarray(rows, np.int64)
        out = np.zeros(len(rows))
        lib.jo_sigma_rows(self.h, _ptr(np.ascontiguousarray(m1, float)),
                          _ptr(np.ascontiguousarray(m2, float)), _ptr(v), _ptr(rows),
                          len(rows), _ptr(out))
        return out

    def davidson(self, m1, m2, totcore, maxiter=500, krymin=4, krymax=12,
                 nroots=1, prediagr=1, refdim=8, restol=1e-8, init=None):
        e = np.zeros(nroots)
        civ = np.zeros((nroots, self.ndets))
        init_p = None
        if init is not None:
            init = np.ascontiguousarray(init, float)
            init_p = _ptr(init)
        it = self.lib().jo_davidson(self.h, _ptr(m1), _ptr(m2), totcore, maxiter,
                                    krymin, krymax, nroots, prediagr, refdim,
                                    restol, init_p, _ptr(e), _ptr(civ))
        if it < 0:
            raise ValueError(f"oracle davidson failed ({it})")
        return e, civ, it


def ci_space(general):
    """OracleSpace of a &general / &wavefcn tuple (electrons, orbitals,
    nfrozen, ndocc, nactive, nfrzvirt, xlevel), with the reference's alpha /
    beta split (abecalc.c: alpha takes the odd electron)."""
    e, o, nfc, nd, na, nfv, x = general
    ci_e = e - 2 * nfc
    return OracleSpace((ci_e + 1) // 2, ci_e // 2, o - nfc - nfv, nd, na, x)


def dyson(general0, general1, v0, v1, states0, states1):
    """Dyson orbitals of the restatement (jo_dyson): (len(states0) *
    len(states1)) x orbitals0, states 1-based."""
    s0, s1 = ci_space(general0), ci_space(general1)
    lib = OracleSpace.lib()
    lib.jo_dyson.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                             ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    v0 = np.ascontiguousarray(v0, np.float64)
    v1 = np.ascontiguousarray(v1, np.float64)
    st0 = np.asarray(states0, np.int32)
    st1 = np.asarray(states1, np.int32)
    out = np.zeros((len(st0) * len(st1), general0[1]))
    lib.jo_dyson(s0.h, s1.h, general0[0], general0[1], _ptr(v0), _ptr(v1), len(st0), _ptr(st0),
                 len(st1), _ptr(st1), _ptr(out))
    return out


def ref_dyson(general0, general1, v0, v1, states0, states1):
    """Dyson orbitals of the reference's own dysoncomp.c (oracle/_ref)."""
    lib = RefSpace.lib()
    lib.ref_dyson.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                              ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                              ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    g0 = np.asarray(general0, np.int32)
    g1 = np.asarray(general1, np.int32)
    v0 = np.ascontiguousarray(v0, np.float64)
    v1 = np.ascontiguousarray(v1, np.float64)
    st0 = np.asarray(states0, np.int32)
    st1 = np.asarray(states1, np.int32)
    out = np.zeros((len(st0) * len(st1), general0[1]))
    r = lib.ref_dyson(_ptr(g0), _ptr(g1), v0.shape[0], _ptr(v0), v1.shape[0], _ptr(v1),
                      len(st0), _ptr(st0), len(st1), _ptr(st1), _ptr(out))
    if r:
        raise ValueError(f"reference dyson failed: {r}")
    return out


def symeig(a):
    a = np.array(a, float, order="C")
    n = a.shape[0]
    w = np.zeros(n)
    z = np.zeros((n, n))
    OracleSpace.lib().jo_symeig(n, _ptr(a), _ptr(w), _ptr(z))
    return w, z


class RefSpace:
    """The reference's own code (oracle/_ref) driven through ref_harness.c.

    The reference keeps its state in globals, so one RefSpace is live at a
    time (building a new one replaces the previous space)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = _load(REF_SO)
            lib.ref_build_space.argtypes = [ctypes.c_int] * 7
            lib.ref_pdavidson.argtypes = [ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_double, ctypes.c_double] + \
                [ctypes.c_int] * 7 + [ctypes.c_double, ctypes.c_char_p, ctypes.c_void_p]
            cls._lib = lib
        return cls._lib

    def __init__(self, electrons, orbitals, nfrzc=0, ndocc=0, nactv=None,
                 nfrzv=0, xlvl=0):
        if nactv is None:
            nactv = orbitals - nfrzc - nfrzv - ndocc
        nd = self.lib().ref_build_space(electrons, orbitals, nfrzc, ndocc, nactv,
                                        nfrzv, xlvl)
        if nd < 0:
            raise ValueError("reference: invalid space")
        sz = np.zeros(10, np.int32)
        self.lib().ref_sizes(_ptr(sz))
        (self.na, self.nb, self.norb, self.nastr, self.nbstr, self.pegrps,
         self.qegrps, self.npq, self.ndets, self.intorb) = (int(x) for x in sz)
        self.ndocc, self.nactv, self.xlvl = ndocc, nactv, xlvl

    def strings(self, spin):
        ns, ne = (self.nastr, self.na) if spin == 0 else (self.nbstr, self.nb)
        istr = np.zeros(ns * ne, np.int32)
        b1 = np.zeros(ns, np.int64)
        vx = np.zeros(2 * ns, np.int32)
        nv = np.zeros(ns, np.int32)
        self.lib().ref_get_strings(spin, _ptr(istr), _ptr(b1), _ptr(vx), _ptr(nv))
        return istr.reshape(ns, ne), b1, vx.reshape(ns, 2), nv

    def eospaces(self, spin):
        ng = self.pegrps if spin == 0 else self.qegrps
        out = np.zeros(26 * ng, np.int32)
        self.lib().ref_get_eospaces(spin, _ptr(out))
        return out.reshape(ng, 26)

    def pq(self):
        out = np.zeros(2 * self.npq, np.int32)
        self.lib().ref_get_pq(_ptr(out))
        return out.reshape(self.npq, 2)

    def yij_cij(self, spin):
        ns, ne = (self.nastr, self.na) if spin == 0 else (self.nbstr, self.nb)
        w = self.norb + 1
        y = np.zeros(ns * ne * w, np.int32)
        c = np.zeros(ns * ne * w, np.int32)
        self.lib().ref_get_yij_cij(spin, _ptr(y), _ptr(c))
        return y.reshape(ns, ne, w), c.reshape(ns, ne, w)

    def excitations(self, spin, nrep, istr, teosp):
        ns = self.nastr if spin == 0 else self.nbstr
        out = np.zeros(6 * (ns + 1), np.int32)
        n = self.lib().ref_excitations(spin, nrep, istr, teosp, _ptr(out))
        return out[: 6 * n].reshape(n, 6)

    def wlist(self):
        out = np.zeros(3 * self.ndets, np.int32)
        self.lib().ref_get_wlist(_ptr(out))
        return out.reshape(self.ndets, 3)

    def hdiag(self, m1, m2):
        out = np.zeros(self.ndets)
        self.lib().ref_hdiag(_ptr(m1), _ptr(m2), _ptr(out))
        return out

    def sigma(self, m1, m2, V):
        V = np.ascontiguousarray(np.atleast_2d(V), float)
        C = np.zeros_like(V)
        self.lib().ref_sigma(_ptr(m1), _ptr(m2), V.shape[0], _ptr(V), _ptr(C))
        return C

    def davidson(self, m1, m2, nucrep, frzcore, maxiter=500, krymin=4,
                 krymax=12, nroots=1, prediagr=1, refdim=8, restol=1e-8,
                 printlvl=0, workdir=None):
        civ = np.zeros((nroots, self.ndets))
        wd = workdir or tempfile.mkdtemp(prefix="jci_ref_")
        rc = self.lib().ref_pdavidson(_ptr(m1), _ptr(m2), nucrep, frzcore, printlvl,
                                      maxiter, krymin, krymax, nroots, prediagr,
                                      refdim, restol, wd.encode(), _ptr(civ))
        if rc != 0:
            raise RuntimeError(f"reference pdavidson returned {rc}")
        return civ, wd


def canonical_excitation(row):
    """(index, io_hi, io_lo, fo_lo, fo_hi, phase) with the phase adjusted to
    that pairing; the matrix element permx[(io0 fo0|io1 fo1)-(io0 fo1|io1 fo0)]
    is invariant under this normalisation."""
    idx, i0, i1, f0, f1, p = (int(x) for x in row)
    if i1 == 0:
        return (idx, i0, 0, f0, 0, p)
    if i0 < i1:                       # swap the two (io, fo) pairs jointly
        i0, i1, f0, f1 = i1, i0, f1, f0
    if f0 > f1:                       # swapping only the targets flips sign
        f0, f1, p = f1, f0, -p
    return (idx, i0, i1, f0, f1, p)
