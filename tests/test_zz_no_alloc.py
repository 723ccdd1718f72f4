"""The allocation-free entry point, through the C ABI.

mbe_enumerate_device_noalloc exists for callers that cannot call cudaMalloc
(a framework that owns all device memory, work recorded into a CUDA graph,
a fixed device-memory budget): it takes its working memory from a static
pool inside the library instead of allocating.  These tests give it device
buffers owned by the test (the caller) and check that, on two calls in a
row, it returns exactly what the allocating entry point mbe_enumerate returns
for the same graph (count and set hash are integers: the tolerance is zero).

The file name sorts last among the test files and its tests carry the `last`
marker, which the conftest's ordering puts after every unmarked test; among
the `last` tests collection order holds, so a run that stops at the first
failure has run every other test before these.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.last]


def _lib(gm):
    lib = C.CDLL(gm.LIB_PATH)
    f = lib.mbe_enumerate_device_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                  C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
    return f


def _transpose(ro, co, nU):
    nV = len(ro) - 1
    rows = np.repeat(np.arange(nV, dtype=np.int32), np.diff(ro))
    order = np.lexsort((rows, co))
    rev_col = rows[order].astype(np.int32)
    rev_off = np.zeros(nU + 1, np.int32)
    np.add.at(rev_off, co + 1, 1)
    return np.cumsum(rev_off).astype(np.int32), rev_col


def test_no_alloc_matches_allocating_entry_point_twice():
    import torch
    import gmbe_b200 as gm

    g = gm.config_graph("small")
    # The allocating entry point on the same numbering (no side swap, input order).
    with gm.Graph.from_csr(g.row_off, g.col, g.nU, uvtrans=0, order=0) as G:
        want = G.enumerate()
    assert want.status == 0 and want.count > 0

    rev_off, rev_col = _transpose(g.row_off, g.col, g.nU)
    dev = torch.device("cuda", 0)
    t_ro = torch.from_numpy(np.ascontiguousarray(g.row_off)).to(dev)
    t_co = torch.from_numpy(np.ascontiguousarray(g.col)).to(dev)
    t_rro = torch.from_numpy(rev_off).to(dev)
    t_rco = torch.from_numpy(rev_col).to(dev)
    out = torch.zeros(4, dtype=torch.int64, device=dev)
    f = _lib(gm)
    torch.cuda.synchronize()
    for call in range(2):
        out.fill_(-1)
        torch.cuda.synchronize()
        rc = f(t_ro.data_ptr(), t_co.data_ptr(), g.nV, t_rro.data_ptr(), t_rco.data_ptr(), g.nU,
               g.nE, 0, None, out.data_ptr(), None)
        assert rc == 0, gm.last_error()
        torch.cuda.synchronize()
        got = [int(x) & ((1 << 64) - 1) for x in out.cpu().tolist()]
        assert got[3] == 0, f"device status {got[3]} on call {call}"
        assert (got[0], got[1]) == (want.count, want.set_hash), f"call {call}"


def test_no_alloc_rejects_graphs_beyond_its_pool():
    import torch
    import gmbe_b200 as gm

    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.int32, device=dev)
    out = torch.zeros(4, dtype=torch.int64, device=dev)
    f = _lib(gm)
    # Sizes far beyond the pool: rejected before anything is queued, so the
    # (too small) buffers are never read.
    rc = f(buf.data_ptr(), buf.data_ptr(), 400000, buf.data_ptr(), buf.data_ptr(), 100000,
           2000000, 0, None, out.data_ptr(), None)
    assert rc == -8  # MBE_ERR_CAPACITY
    assert "pool" in gm.last_error()
