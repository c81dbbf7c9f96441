"""ctypes bindings to the in-tree native libraries.  Nothing here falls back to Python: a missing or
unloadable library raises immediately."""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_int64, c_uint64, c_void_p

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")

_gen = None
_core = None


class NativeLibraryMissing(RuntimeError):
    pass


def _load(name: str) -> ctypes.CDLL:
    path = os.path.join(LIB_DIR, name)
    if not os.path.exists(path):
        raise NativeLibraryMissing(f"{path} is not built; run `python -m dmolp_b200.build` (or __graft_entry__.build())")
    return ctypes.CDLL(path, mode=ctypes.RTLD_GLOBAL)


def gen() -> ctypes.CDLL:
    global _gen
    if _gen is None:
        lib = _load("libdmolp_gen.so")
        lib.dmolp_gen_last_error.restype = c_char_p
        lib.dmolp_gen_rmat.argtypes = [c_int, c_int, c_double, c_double, c_double, c_uint64, c_int, POINTER(c_void_p)]
        lib.dmolp_gen_knn.argtypes = [c_int64, c_int, c_int, c_uint64, POINTER(c_void_p)]
        lib.dmolp_gen_ba.argtypes = [c_int64, c_int, c_uint64, POINTER(c_void_p)]
        lib.dmolp_gen_band.argtypes = [c_int64, c_int, c_int, c_uint64, POINTER(c_void_p)]
        lib.dmolp_csr_from_arrays.argtypes = [c_int64, c_int64, c_void_p, c_void_p, POINTER(c_void_p)]
        lib.dmolp_csr_nv.argtypes = [c_void_p]
        lib.dmolp_csr_nv.restype = c_int64
        lib.dmolp_csr_narcs.argtypes = [c_void_p]
        lib.dmolp_csr_narcs.restype = c_int64
        lib.dmolp_csr_copy.argtypes = [c_void_p, c_void_p, c_void_p]
        lib.dmolp_csr_write_adjtext.argtypes = [c_void_p, c_char_p]
        lib.dmolp_csr_free.argtypes = [c_void_p]
        lib.dmolp_csr_free.restype = None
        lib.dmolp_fnv1a.argtypes = [c_void_p, c_int64]
        lib.dmolp_fnv1a.restype = c_uint64
        _gen = lib
    return _gen


def core_path() -> str:
    return os.path.join(LIB_DIR, "libdmolp_b200.so")


def core() -> ctypes.CDLL:
    """The CUDA library behind include/dmolp_b200.h."""
    global _core
    if _core is None:
        from . import cabi

        _core = cabi.bind(_load("libdmolp_b200.so"))
    return _core
