"""Loads oracle/_ref/libxamg_ref.so: entry points over the reference's own
narrowing / bit-hash / core-split headers, built by `make -C oracle ref` from
the reference sources. Test infrastructure."""
import ctypes as C
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libxamg_ref.so")


def load():
    """The pins library, built on first use where the reference sources are
    present (oracle/Makefile's XAMG_REF_SRC); None where they are not."""
    if not os.path.exists(REF_LIB):
        subprocess.call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"])
    if not os.path.exists(REF_LIB):
        return None
    L = C.CDLL(REF_LIB)
    L.ref_define_int_type.restype = C.c_uint16
    L.ref_define_int_type.argtypes = [C.c_uint64]
    L.ref_encode_hash.restype = C.c_uint16
    L.ref_encode_hash.argtypes = [C.c_uint64] * 4 + [C.c_int]
    L.ref_parse_bit_hash.argtypes = [C.c_uint16, C.POINTER(C.c_uint16)]
    L.ref_split_range_f64.restype = C.c_uint64
    L.ref_split_range_f64.argtypes = [C.c_uint64, C.c_int]
    L.ref_search_range.restype = C.c_uint32
    L.ref_search_range.argtypes = [C.c_uint64, C.POINTER(C.c_uint64), C.c_uint64]
    return L
