"""ctypes wrapper of the CPU oracle (liboracle.so, built from mbe_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference legs of bench.py, always as the checker or the timed
CPU baseline, never as the engine.  See mbe_oracle.c for what each
enumerator restates and where in the reference it comes from.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")


def build(quiet: bool = True):
    """Builds liboracle.so (gcc; always possible)."""
    subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def _load():
    if not os.path.exists(LIB):
        build()
    lib = C.CDLL(LIB)
    P32 = C.POINTER(C.c_int32)
    lib.orc_brute_force.argtypes = [C.c_int32, C.c_int32, P32, P32, C.c_void_p]
    lib.orc_mbea.argtypes = [C.c_int32, C.c_int32, P32, P32, C.c_int32, C.c_int32, C.c_void_p]
    lib.orc_gmbe.argtypes = [C.c_int32, C.c_int32, P32, P32, C.c_int32, C.c_int32, C.c_int32,
                             C.c_int32, C.c_void_p]
    lib.orc_gmbe_range.argtypes = [C.c_int32, C.c_int32, P32, P32, C.c_int32, C.c_int32,
                                   C.c_int32, C.c_int32, C.c_int64, C.c_int64,
                                   C.POINTER(C.c_int64), C.c_void_p]
    lib.orc_gmbe_strided.argtypes = [C.c_int32, C.c_int32, P32, P32, C.c_int32, C.c_int32,
                                     C.c_int32, C.c_int32, C.c_int64, C.c_int64, C.c_void_p]
    lib.orc_internal_order.argtypes = [C.c_int32, C.c_int32, P32, P32, C.c_int32, C.c_int32,
                                       P32, P32]
    return lib


class OrcResult(C.Structure):
    _fields_ = [("count", C.c_uint64), ("set_hash", C.c_uint64), ("non_maximal", C.c_uint64),
                ("alg_bytes", C.c_uint64), ("nodes", C.c_uint64)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _arrs(row_off, col):
    ro = np.ascontiguousarray(row_off, dtype=np.int32)
    co = np.ascontiguousarray(col, dtype=np.int32)
    if co.size == 0:
        co = np.zeros(1, np.int32)
    P = C.POINTER(C.c_int32)
    return ro, co, ro.ctypes.data_as(P), co.ctypes.data_as(P)


def brute_force(row_off, col, nU):
    """Closure of V-neighbourhood intersections (|U| <= 64)."""
    ro, co, pr, pc = _arrs(row_off, col)
    r = OrcResult()
    if lib().orc_brute_force(len(ro) - 1, nU, pr, pc, C.byref(r)) != 0:
        raise ValueError("brute force needs |U| <= 64")
    return r


def mbea(row_off, col, nU, uvtrans=0, order=1):
    """MbeaFinder restatement (src/BicliqueFinder.cu:20-57)."""
    ro, co, pr, pc = _arrs(row_off, col)
    r = OrcResult()
    lib().orc_mbea(len(ro) - 1, nU, pr, pc, uvtrans, order, C.byref(r))
    return r


def gmbe(row_off, col, nU, uvtrans=1, order=1, prune=1, threads=0):
    """GMBE per-root restatement, OpenMP over roots (threads 0 = all)."""
    ro, co, pr, pc = _arrs(row_off, col)
    r = OrcResult()
    lib().orc_gmbe(len(ro) - 1, nU, pr, pc, uvtrans, order, prune, threads, C.byref(r))
    return r


def gmbe_range(row_off, col, nU, root_begin, root_end, uvtrans=1, order=1, prune=1, threads=0,
               stats=False):
    """Roots [root_begin, root_end) of the internal order only."""
    ro, co, pr, pc = _arrs(row_off, col)
    r = OrcResult()
    st = None
    stp = None
    if stats:
        st = np.zeros((max(len(ro) - 1, nU), 5), dtype=np.int64)
        stp = st.ctypes.data_as(C.POINTER(C.c_int64))
    lib().orc_gmbe_range(len(ro) - 1, nU, pr, pc, uvtrans, order, prune, threads,
                         root_begin, root_end, stp, C.byref(r))
    return (r, st) if stats else r


def gmbe_strided(row_off, col, nU, offset, stride, uvtrans=1, order=1, prune=1, threads=0):
    """Roots at positions offset, offset+stride, ... from the top of the
    internal order (a stratified sample of a degree-sorted root list)."""
    ro, co, pr, pc = _arrs(row_off, col)
    r = OrcResult()
    lib().orc_gmbe_strided(len(ro) - 1, nU, pr, pc, uvtrans, order, prune, threads, offset,
                           stride, C.byref(r))
    return r


def ref_binary(name: str) -> str | None:
    """Path of a reference program built by `make -C oracle ref`, if present."""
    p = os.path.join(REF_DIR, name)
    return p if os.path.exists(p) else None
