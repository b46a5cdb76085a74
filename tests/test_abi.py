"""The C ABI library loads and exports every symbol include/qcb.h declares (no GPU needed).
Also exercises the host-only LIME/ILDG record parser (qcb_ildg_probe) on crafted files."""
import os
import re
import struct

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "qcb.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(qcb_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol(qcb):
    lib = qcb.load_library()
    names = declared_symbols()
    assert len(names) >= 35
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header(qcb):
    assert sorted(qcb.exported_symbols()) == declared_symbols()


def test_version_and_launch_counter(qcb):
    assert b"sm_100a" in qcb.lib().qcb_version()
    assert qcb.launch_count() >= 0


def lime_record(rtype: bytes, payload: bytes, mb: bool, me: bool) -> bytes:
    hdr = struct.pack(">IHBB Q", 0x456789AB, 1, (0x80 if mb else 0) | (0x40 if me else 0), 0, len(payload))
    hdr = hdr.replace(b" ", b"")
    hdr += rtype.ljust(128, b"\0")
    assert len(hdr) == 144
    pad = (-len(payload)) % 8
    return hdr + payload + b"\0" * pad


def ildg_xml(L, prec=64):
    return ("<?xml version=\"1.0\" encoding=\"UTF-8\"?>\n<ildgFormat><version>1.0</version><field>su3gauge</field>"
            f"<precision>{prec}</precision><lx>{L[0]}</lx><ly>{L[1]}</ly><lz>{L[2]}</lz><lt>{L[3]}</lt>"
            "</ildgFormat>").encode()


def test_ildg_probe_reads_format_record(qcb, tmp_path):
    p = tmp_path / "a.ildg"
    L = (4, 6, 2, 8)
    V = L[0] * L[1] * L[2] * L[3]
    p.write_bytes(lime_record(b"ildg-format", ildg_xml(L, 32), True, True) +
                  lime_record(b"ildg-binary-data", b"\0" * (V * 72 * 4), False, True))
    assert qcb.ildg_probe(str(p)) == (L, 32)


def test_ildg_probe_errors(qcb, tmp_path):
    with pytest.raises(qcb.QcbError) as e:
        qcb.ildg_probe(str(tmp_path / "missing"))
    assert e.value.code == -3
    bad = tmp_path / "bad"
    bad.write_bytes(b"\x12\x34" * 100)
    with pytest.raises(qcb.QcbError) as e:
        qcb.ildg_probe(str(bad))
    assert e.value.code == -4
    trunc = tmp_path / "trunc"
    trunc.write_bytes(lime_record(b"ildg-format", ildg_xml((4, 4, 4, 4)), True, True)[:100])
    with pytest.raises(qcb.QcbError) as e:
        qcb.ildg_probe(str(trunc))
    assert e.value.code == -4
    noxml = tmp_path / "noxml"
    noxml.write_bytes(lime_record(b"ildg-binary-data", b"\0" * 64, True, True))
    with pytest.raises(qcb.QcbError) as e:
        qcb.ildg_probe(str(noxml))
    assert e.value.code == -4


def scidac_sums_zlib(payload: bytes, site_bytes: int):
    """Independent restatement of the SciDAC checksum with zlib's CRC-32."""
    import zlib

    rotl = lambda v, r: ((v << r) | (v >> (32 - r))) & 0xFFFFFFFF if r else v
    a = b = 0
    for r in range(len(payload) // site_bytes):
        c = zlib.crc32(payload[r * site_bytes:(r + 1) * site_bytes])
        a ^= rotl(c, r % 29)
        b ^= rotl(c, r % 31)
    return a, b


def scidac_record(a: int, b: int) -> bytes:
    return (f"<?xml version=\"1.0\" encoding=\"UTF-8\"?><scidacChecksum><version>1.0</version>"
            f"<suma>{a:x}</suma><sumb>{b:x}</sumb></scidacChecksum>").encode()


def test_scidac_checksum_known_answer(qcb):
    # CRC-32 check value of "123456789"; one record at rank 0 is rotated by 0 in both sums
    assert qcb.scidac_checksum(b"123456789", 9) == (0xCBF43926, 0xCBF43926)
    assert qcb.scidac_checksum(b"", 8) == (0, 0)


@pytest.mark.parametrize("n_sites,site_bytes", [(1, 576), (29, 576), (31, 13), (1000, 288), (20000, 24), (9000, 7)])
def test_scidac_checksum_matches_zlib(qcb, n_sites, site_bytes):
    import numpy as np

    payload = np.random.default_rng(n_sites + site_bytes).integers(0, 256, n_sites * site_bytes, dtype=np.uint8)
    payload = payload.tobytes()
    assert qcb.scidac_checksum(payload, site_bytes) == scidac_sums_zlib(payload, site_bytes)


def test_ildg_probe_scidac_record(qcb, tmp_path):
    L = (2, 2, 2, 2)
    body = b"\0" * (16 * 72 * 8)
    good = tmp_path / "good"
    good.write_bytes(lime_record(b"ildg-format", ildg_xml(L), True, True) +
                     lime_record(b"ildg-binary-data", body, False, False) +
                     lime_record(b"scidac-checksum", scidac_record(*scidac_sums_zlib(body, 576)), False, True))
    assert qcb.ildg_probe(str(good)) == (L, 64)
    bad = tmp_path / "bad"
    bad.write_bytes(lime_record(b"ildg-format", ildg_xml(L), True, True) +
                    lime_record(b"ildg-binary-data", body, False, False) +
                    lime_record(b"scidac-checksum", b"<scidacChecksum><suma>zz</suma></scidacChecksum>", False, True))
    with pytest.raises(qcb.QcbError) as e:
        qcb.ildg_probe(str(bad))
    assert e.value.code == -4


def test_checked_library_exports_every_declared_symbol(qcb):
    import ctypes

    assert os.path.exists(qcb.CHECKED_LIB_PATH), "build() also makes libqcb_checked.so"
    lib = ctypes.CDLL(qcb.CHECKED_LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    lib.qcb_version.restype = ctypes.c_char_p
    assert b"checked" in lib.qcb_version() and b"checked" not in qcb.lib().qcb_version()


def test_argument_validation_needs_no_device(qcb):
    """Invalid arguments are refused on the host with QCB_EINVAL before any device call, so this
    runs without a GPU: odd, too small and too large extents, unknown precision or storage, a
    non-positive coupling, null handles and pointers."""
    import ctypes as C

    lib = qcb.load_library()
    h = C.c_void_p()
    L4 = lambda *v: (C.c_int * 4)(*v)  # noqa: E731
    dummy = C.c_void_p(256)
    for L, prec, store in [((3, 4, 4, 4), 64, 0), ((4, 4, 4, 0), 64, 0), ((2048, 2048, 2048, 2), 64, 0),
                           ((4, 4, 4, 4), 16, 0), ((4, 4, 4, 4), 64, 2)]:
        assert lib.qcb_field_create(L4(*L), prec, store, C.byref(h)) == -1, (L, prec, store)
    assert lib.qcb_field_create(L4(4, 4, 4, 4), 64, 0, None) == -1
    seeds = (C.c_uint64 * 2)(1, 2)
    assert lib.qcb_batch_create(2, (C.c_int * 8)(4, 4, 4, 4, 4, 4, 4, 5), (C.c_double * 2)(6.0, 6.0), seeds,
                                64, 0, C.byref(h)) == -1
    assert b"lattice 1" in lib.qcb_last_error()
    assert lib.qcb_batch_create(2, (C.c_int * 8)(*([4] * 8)), (C.c_double * 2)(6.0, 0.0), seeds, 64, 0,
                                C.byref(h)) == -1
    assert b"beta" in lib.qcb_last_error()
    assert lib.qcb_batch_create(0, None, None, None, 64, 0, C.byref(h)) == -1
    assert lib.qcb_serve_create(1 << 30, 64, 0, 0, 0, C.byref(h)) == -1  # n_rk < 1
    assert lib.qcb_serve_submit(None, 1, L4(4, 4, 4, 4), dummy, 0.02, 5) == -1
    assert lib.qcb_plaquette_noalloc(L4(4, 4, 4, 3), dummy, dummy, None) == -1
    # misaligned caller pointers are refused before any device call: links must be 16-byte aligned
    # (read as (re, im) pairs), the output 8-byte aligned
    assert lib.qcb_plaquette_noalloc(L4(4, 4, 4, 4), C.c_void_p(256 + 8), dummy, None) == -1
    assert b"16-byte" in lib.qcb_last_error()
    assert lib.qcb_plaquette_noalloc(L4(4, 4, 4, 4), dummy, C.c_void_p(256 + 4), None) == -1
    # extents whose product overflows 64 bits are refused, not wrapped
    big = L4(65536, 65536, 65536, 65536)
    assert lib.qcb_field_create(big, 64, 0, C.byref(h)) == -1
    assert lib.qcb_plaquette_noalloc(big, dummy, dummy, None) == -1
    assert lib.qcb_batch_create(1, big, (C.c_double * 1)(6.0), seeds, 64, 0, C.byref(h)) == -1
    for call in (lambda: lib.qcb_hb_sweep(None, 6.0, 1, 1, 0), lambda: lib.qcb_plaquette(None, None),
                 lambda: lib.qcb_field_prefetch_aos(None, None), lambda: lib.qcb_field_commit_prefetch(None),
                 lambda: lib.qcb_debug_probe_link(None, 0, 0, 0), lambda: lib.qcb_ildg_write_ex(None, b"x", 0),
                 lambda: lib.qcb_ildg_read(None, b"x")):
        assert call() == -1
