"""Boundary formats: SIFS integrals, jayci.in namelists, vector files and the
C ABI symbol table (no GPU needed)."""
import ctypes
import os
import re
import struct

import numpy as np
import pytest

import jayci_b200 as jb
from jayci_b200.synth import make_integrals, unpack_integrals

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_abi_exports_every_declared_symbol():
    text = open(os.path.join(ROOT, "include", "jci.h")).read()
    names = set(re.findall(r"\b(jci_[a-z0-9_]+)\s*\(", text))
    names -= {"jci_status"}
    lib = ctypes.CDLL(jb.LIBPATH)
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    assert len(names) >= 20


@pytest.mark.parametrize("nfrozen", [0, 2])
def test_sifs_round_trip(tmp_path, nfrozen):
    ints = make_integrals(8, 8, 21, nfrozen=nfrozen)
    m1, m2 = ints.packed()
    p = tmp_path / "moints"
    jb.write_moints(p, 8, m1, m2, ints.e_nuc, ints.e_fc)
    r1, r2, nb, en, fc = jb.read_moints(p)
    assert nb == 8
    assert en == ints.e_nuc
    assert fc == ints.e_fc
    np.testing.assert_array_equal(r1, m1)
    np.testing.assert_array_equal(r2, m2)
    h, eri = unpack_integrals(r1, r2, 8)
    np.testing.assert_allclose(eri, eri.transpose(1, 0, 2, 3))
    np.testing.assert_allclose(eri, eri.transpose(2, 3, 0, 1))


def test_sifs_fsplit2_separate_two_electron_file(tmp_path):
    """fsplit = 2 (info(1) of header 2): the 2-e records sit on a second
    file with no headers, one l2rec-word Fortran record each (colib sifo2f /
    aiopen / airead, colib8.f:1720, colib2.f:34,89).  The reference's
    readmoints.f90:278-282 refuses such files; this reader takes them."""
    ints = make_integrals(7, 7, 23, nfrozen=1)
    m1, m2 = ints.packed()
    one = tmp_path / "one" / "moints"
    one.parent.mkdir()
    jb.write_moints(one, 7, m1, m2, ints.e_nuc, ints.e_fc)
    p, p2 = tmp_path / "moints", tmp_path / "moints2"
    jb.write_moints(p, 7, m1, m2, ints.e_nuc, ints.e_fc, path2=p2)
    # header 2 says fsplit = 2; the 1-e file is shorter by the 2-e records
    raw, raw2 = p.read_bytes(), p2.read_bytes()
    n2 = struct.unpack("<i", raw[64:68])[0]  # header 2 follows the 64-byte header 1
    off = 68 + 80 + 8 + 4                     # title, nbpsy, slabel
    info = struct.unpack("<6q", raw[off:off + 48])
    assert info[0] == 2 and info[3] == 4096
    assert n2 > 0 and len(raw) + len(raw2) == len(one.read_bytes())
    # the 2-e file starts with a 2-e record (itypea 3 in the dword)
    assert struct.unpack("<i", raw2[:4])[0] == 8 * info[3]
    dword = struct.unpack("<Q", raw2[4:12])[0]
    assert ((dword >> 16) & 0xffff) >> 10 & 7 == 3
    for got in (jb.read_moints(p), jb.read_moints(p, p2)):
        r1, r2, nb, en, fc = got
        assert (nb, en, fc) == (7, ints.e_nuc, ints.e_fc)
        np.testing.assert_array_equal(r1, m1)
        np.testing.assert_array_equal(r2, m2)
    # a missing 2-e file is an I/O error, a truncated one a format error
    p2.rename(tmp_path / "elsewhere")
    with pytest.raises(jb.JciError) as e:
        jb.read_moints(p)
    assert e.value.status == 6
    (tmp_path / "moints2").write_bytes(raw2[: len(raw2) // 2])
    with pytest.raises(jb.JciError) as e:
        jb.read_moints(p)
    assert e.value.status == 7
    # an fsplit = 1 file never opens the named 2-e file
    r1, r2, *_ = jb.read_moints(one, tmp_path / "absent")
    np.testing.assert_array_equal(r2, m2)


def test_sifs_record_layout(tmp_path):
    """Header 1 is seven INTEGER*8 in one Fortran record (readmoints.f90:101);
    the first 1-e record's dword carries num/lab1/types/last as four 16-bit
    fields, most significant first (colib ulab16 / sifd1)."""
    ints = make_integrals(6, 6, 22)
    m1, m2 = ints.packed()
    p = tmp_path / "moints"
    jb.write_moints(p, 6, m1, m2, 10.0, 0.0)
    raw = p.read_bytes()
    n0 = struct.unpack("<i", raw[:4])[0]
    assert n0 == 56
    h1 = struct.unpack("<7q", raw[4:60])
    assert h1 == (2, 1, 1, 6, 6, 1, 0)
    off = 60 + 4
    n1 = struct.unpack("<i", raw[off:off + 4])[0]
    off += 4 + n1 + 4
    n2 = struct.unpack("<i", raw[off:off + 4])[0]
    assert n2 == 4096 * 8
    dword = struct.unpack("<Q", raw[off + 4:off + 12])[0]
    num, lab1 = dword >> 48, (dword >> 32) & 0xffff
    last, ifmt = dword & 3, (dword >> 2) & 7
    assert num == 6 and lab1 == num + 3 and ifmt == 0 and last == 1  # S1 = identity


def test_sifs_rejects_bad_file(tmp_path):
    p = tmp_path / "moints"
    p.write_bytes(b"\x00" * 10)
    with pytest.raises(jb.JciError):
        jb.read_moints(p)
    with pytest.raises(jb.JciError) as ei:
        jb.read_moints(tmp_path / "missing")
    assert ei.value.status == 6


def test_namelists(tmp_path):
    p = tmp_path / "jayci.in"
    p.write_text(""" &general
  electrons = 18, orbitals = 16,
  nfrozen = 2, ndocc = 0, nactive = 14, xlevel = 0  ! frozen core
 /
 &dalginfo
  maxiter = 500, krymin = 8, krymax = 24, nroots = 4,
  prediagr = 1, restol = 1.0d-8, refdim = 16, buflen = 0
 /
""")
    g, d, u = jb.read_namelists(p)
    assert (g.electrons, g.orbitals, g.nfrozen, g.ndocc, g.nactive, g.xlevel) == \
        (18, 16, 2, 0, 14, 0)
    assert (d.maxiter, d.krymin, d.krymax, d.nroots, d.refdim, d.buflen) == \
        (500, 8, 24, 4, 16, 0)
    # the reference writes restol with f10.5 and reads it back (0.00000)
    assert d.restol == 0.0
    assert u.precision == 0
    p.write_text(p.read_text() + " &gpuinfo precision=2, exactrestol=1, switchtol=1d-4 /\n")
    g, d, u = jb.read_namelists(p)
    assert d.restol == 1e-8 and u.precision == 2 and u.switch_tol == 1e-4


def test_namelist_defaults_and_errors(tmp_path):
    p = tmp_path / "jayci.in"
    p.write_text("&general electrons=4, orbitals=4 /\n&dalginfo /\n")
    g, d, u = jb.read_namelists(p)
    assert (d.maxiter, d.krymin, d.krymax, d.nroots, d.prediagr, d.refdim) == \
        (20, 3, 8, 1, 1, 3)
    assert d.restol == 1e-5
    p.write_text("&general electrons=4, bogus=1 /\n&dalginfo /\n")
    with pytest.raises(jb.JciError):
        jb.read_namelists(p)
    with pytest.raises(jb.JciError):
        jb.read_namelists(tmp_path / "nope.in")


def test_server_needs_a_device():
    """Without a CUDA device the server refuses to start (no CPU fallback)."""
    if jb.device_count() > 0:
        pytest.skip("a device is present")
    with pytest.raises(jb.JciError) as ei:
        jb.Server(slots=2)
    assert ei.value.status == 5


def test_vector_files(tmp_path):
    v = np.random.default_rng(1).standard_normal((3, 17))
    p = tmp_path / "civec"
    jb.write_vectors(p, v)
    raw = p.read_bytes()
    assert struct.unpack("<ii", raw[:8]) == (3, 17)
    assert len(raw) == 8 + 3 * 17 * 8
    np.testing.assert_array_equal(jb.read_vectors(p, 3, 17), v)
    with pytest.raises(jb.JciError):
        jb.read_vectors(p, 2, 17)  # read_gavectorsfile_dbl_ufmt error 5
