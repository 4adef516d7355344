"""C-ABI library loads and exports every symbol include/kmhd_sph.h declares (CPU)."""
import ctypes
import os
import re

from kemorin_mhd_b200 import build as kbuild
from kemorin_mhd_b200 import sph_trans

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols(header="kmhd_sph.h"):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(kmhd_\w+)\s*\(", src)))


def test_header_matches_wrapper():
    assert declared_symbols() == sorted(sph_trans.EXPORTS)


def test_library_exports_all_symbols():
    kbuild.build()
    lib = ctypes.CDLL(kbuild.LIB)
    for hdr in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if hdr.endswith(".h"):
            for name in declared_symbols(hdr):
                assert hasattr(lib, name), (hdr, name)


def test_strerror_without_gpu():
    lib = sph_trans.load_library()
    assert lib.kmhd_strerror(0) == b"ok"
    assert lib.kmhd_strerror(2) == b"unsupported size"
    assert lib.kmhd_strerror(99) == b"unknown status"


def test_create_rejects_bad_descriptors():
    # validation runs before any device call: bad sizes return an error code
    lib = sph_trans.load_library()
    d = sph_trans.Desc()
    h = ctypes.c_void_p()
    d.ltr = 0
    assert lib.kmhd_sph_create(ctypes.byref(d), ctypes.byref(h)) == 2
    d.ltr, d.nth, d.nph, d.nr = 31, 48, 62, 4       # nph <= 2L+1
    assert lib.kmhd_sph_create(ctypes.byref(d), ctypes.byref(h)) == 2
    d.nph = 96                                       # radius NULL
    assert lib.kmhd_sph_create(ctypes.byref(d), ctypes.byref(h)) == 1
    r = (ctypes.c_double * 4)(1.0, 1.1, 1.2, 1.3)
    d.radius = r
    d.nvector_b, d.nscalar_b = 1, 1
    d.nph = 7 * 16                                   # factor 7 unsupported
    assert lib.kmhd_sph_create(ctypes.byref(d), ctypes.byref(h)) == 2
    d.nph, d.nvector_b, d.nscalar_b = 96, 6, 0       # too many vectors per group (at most 5)
    assert lib.kmhd_sph_create(ctypes.byref(d), ctypes.byref(h)) == 2
    d.nvector_b, d.nscalar_b, d.nvector_f, d.nscalar_f = 1, 1, 1, 0
    prods = (sph_trans.Product * 1)(sph_trans.Product(0, 0, 3, 1.0))  # cross with bad index
    d.nproduct, d.products = 1, prods
    assert lib.kmhd_sph_create(ctypes.byref(d), ctypes.byref(h)) == 1


def test_create_rejects_bad_flags():
    # on-the-fly P is an FP64-tier option; unknown flag bits are refused
    lib = sph_trans.load_library()
    d = sph_trans.Desc()
    h = ctypes.c_void_p()
    r = (ctypes.c_double * 4)(1.0, 1.1, 1.2, 1.3)
    d.ltr, d.nth, d.nph, d.nr, d.radius = 31, 48, 96, 4, r
    d.nvector_b, d.nscalar_b = 1, 1
    d.tier, d.flags = 1, sph_trans.FLAG_P_ON_THE_FLY
    assert lib.kmhd_sph_create(ctypes.byref(d), ctypes.byref(h)) == 1
    d.tier, d.flags = 0, 8
    assert lib.kmhd_sph_create(ctypes.byref(d), ctypes.byref(h)) == 1
