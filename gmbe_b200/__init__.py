"""Python binding of the B200 maximal biclique enumeration engine.

Thin ctypes layer over the C ABI in ``include/mbe.h`` (``libgmbe.so``, built
in-tree by ``gmbe_b200/csrc/Makefile``).  The reference's own surface is C++
(``CSRBiGraph``, ``IterFinderGpu6``; see ``include/mbe_finder.h``); this module
exists for tests, the benchmark and scripting.  There is no CPU fallback: if
the shared library is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgmbe.so")
CLI_PATH = os.path.join(_HERE, "MBE_GPU")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `make -C gmbe_b200/csrc` "
        "(or __graft_entry__.build()); the engine has no CPU fallback")
_lib = C.CDLL(LIB_PATH)

MBE_OK = 0
ERRORS = {
    -1: "MBE_ERR_INVALID", -2: "MBE_ERR_IO", -3: "MBE_ERR_FORMAT", -4: "MBE_ERR_CUDA",
    -5: "MBE_ERR_NOMEM", -6: "MBE_ERR_TIMEOUT", -7: "MBE_ERR_QUEUE_FULL",
    -8: "MBE_ERR_CAPACITY", -9: "MBE_ERR_ADMISSION", -10: "MBE_ERR_CANCELLED",
    -11: "MBE_ERR_NOT_FOUND", -12: "MBE_ERR_AGAIN",
}


class MBEError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code
        self.name = ERRORS.get(code, str(code))


class Opts(C.Structure):
    _fields_ = [("uvtrans", C.c_int32), ("order", C.c_int32), ("fast_mode", C.c_int32),
                ("device", C.c_int32)]


class GraphInfo(C.Structure):
    _fields_ = [("U_size", C.c_int32), ("V_size", C.c_int32), ("edge_size", C.c_int64),
                ("U_degree", C.c_int32), ("V_degree", C.c_int32), ("U_2degree", C.c_int32),
                ("V_2degree", C.c_int32), ("swapped", C.c_int32)]


class Params(C.Structure):
    _fields_ = [("bound_height", C.c_int32), ("bound_size", C.c_int32), ("prune", C.c_int32),
                ("blocks", C.c_int32), ("queue_capacity", C.c_int32),
                ("bitmap_max_l", C.c_int32), ("wait_limit_ns", C.c_int64),
                ("sm_timing", C.c_int32), ("root_begin", C.c_int32), ("root_end", C.c_int32),
                ("shard_count", C.c_int32), ("shard_index", C.c_int32),
                ("split_mode", C.c_int32), ("direct_max_c", C.c_int32),
                ("root_split_size", C.c_int32), ("share_min_work", C.c_int32),
                ("range_split_work", C.c_int32), ("range_chunk", C.c_int32),
                ("eager_share", C.c_int32), ("big_two_hop", C.c_int32),
                ("big_warps", C.c_int32), ("l2_window", C.c_int32),
                ("time_limit_ns", C.c_int64), ("touch_scan", C.c_int32),
                ("slot_records", C.c_int32),
                ("share_counts", C.c_int32), ("reserved_r", C.c_int32)]


class Result(C.Structure):
    _fields_ = [("count", C.c_uint64), ("set_hash", C.c_uint64), ("non_maximal", C.c_uint64),
                ("tasks_split", C.c_uint64), ("enum_seconds", C.c_double),
                ("kernel_ms", C.c_float), ("status", C.c_int32),
                ("sm_exit_max_ms", C.c_double), ("sm_exit_min_ms", C.c_double),
                ("warp_busy_frac", C.c_double), ("setup_ms", C.c_double),
                ("tier1_ms", C.c_double), ("tier2_ms", C.c_double), ("idle_ms", C.c_double),
                ("max_task_ms", C.c_double), ("max_task_root", C.c_int32),
                ("max_task_degree", C.c_int32), ("n_tasks", C.c_uint64),
                ("n_subproblems", C.c_uint64), ("max_task_tier1_ms", C.c_double),
                ("max_task_tier2_ms", C.c_double), ("max_task_graph", C.c_int32),
                ("reserved", C.c_int32), ("max_task_pushes1", C.c_uint64),
                ("max_task_pushes2", C.c_uint64), ("max_task_cands", C.c_int32),
                ("max_task_part", C.c_int32), ("max_task_parts", C.c_int32),
                ("reserved2", C.c_int32)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class GenSpec(C.Structure):
    _fields_ = [("nU", C.c_int64), ("nV", C.c_int64), ("n_edges", C.c_int64),
                ("gamma_u", C.c_double), ("gamma_v", C.c_double),
                ("max_deg_u", C.c_int64), ("max_deg_v", C.c_int64), ("seed", C.c_uint64),
                ("n_blocks", C.c_int32), ("block_u", C.c_int32), ("block_v", C.c_int32),
                ("reserved", C.c_int32), ("block_p", C.c_double), ("pair_p_max", C.c_double)]


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("max_graphs", C.c_int32), ("arena_bytes", C.c_int64),
                ("max_v", C.c_int32), ("max_degree", C.c_int32), ("max_two_hop", C.c_int32),
                ("prep_threads", C.c_int32), ("idle_exit_ns", C.c_int64)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("admitted", C.c_uint64), ("completed", C.c_uint64),
                ("rejected", C.c_uint64), ("cancelled", C.c_uint64), ("launches", C.c_uint64),
                ("arena_resets", C.c_uint64), ("resident", C.c_int64), ("waiting", C.c_int64),
                ("arena_used", C.c_int64), ("arena_bytes", C.c_int64),
                ("published", C.c_uint64), ("collected", C.c_uint64),
                ("launch_running", C.c_int64), ("dev_head", C.c_uint64), ("dev_tail", C.c_uint64),
                ("dev_done", C.c_uint64), ("dev_pending", C.c_uint64)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_P32 = C.POINTER(C.c_int32)
_sig = {
    "mbe_params_default": (None, [C.POINTER(Params)]),
    "mbe_opts_default": (None, [C.POINTER(Opts)]),
    "mbe_graph_from_adj": (C.c_int, [C.c_char_p, C.POINTER(Opts), C.POINTER(C.c_void_p)]),
    "mbe_graph_from_csr": (C.c_int, [_P32, _P32, C.c_int32, C.c_int32, C.c_int64,
                                     C.POINTER(Opts), C.POINTER(C.c_void_p)]),
    "mbe_graph_build_on_device": (C.c_int, [_P32, _P32, C.c_int32, C.c_int32, C.c_int64,
                                            C.POINTER(Opts), C.POINTER(C.c_void_p)]),
    "mbe_graph_get_info": (C.c_int, [C.c_void_p, C.POINTER(GraphInfo)]),
    "mbe_graph_free": (C.c_int, [C.c_void_p]),
    "mbe_device_release": (C.c_int, [C.c_int32]),
    "mbe_enumerate": (C.c_int, [C.c_void_p, C.POINTER(Params), C.POINTER(Result)]),
    "mbe_enumerate_emit_stream": (C.c_int, [C.c_void_p, C.POINTER(Params), C.POINTER(Result),
                                            C.c_int64, C.c_void_p, C.c_void_p]),
    "mbe_enumerate_emit": (C.c_int, [C.c_void_p, C.POINTER(Params), C.POINTER(Result), _P32,
                                     C.c_int64, C.POINTER(C.c_int64)]),
    "mbe_last_error_string": (C.c_char_p, []),
    "mbe_gen_chung_lu": (C.c_int, [C.POINTER(GenSpec), C.POINTER(_P32), C.POINTER(_P32),
                                   _P32, _P32, C.POINTER(C.c_int64)]),
    "mbe_gen_batch_spec": (C.c_int, [C.c_uint64, C.POINTER(GenSpec)]),
    "mbe_write_adj": (C.c_int, [C.c_char_p, _P32, _P32, C.c_int32]),
    "mbe_write_graph": (C.c_int, [C.c_char_p, _P32, _P32, C.c_int32]),
    "mbe_read_adj": (C.c_int, [C.c_char_p, C.POINTER(_P32), C.POINTER(_P32), _P32, _P32,
                               C.POINTER(C.c_int64)]),
    "mbe_free": (None, [C.c_void_p]),
    "mbe_batch_from_csr": (C.c_int, [C.c_int32, C.POINTER(_P32), C.POINTER(_P32), _P32, _P32,
                                     C.POINTER(C.c_int64), C.POINTER(Opts),
                                     C.POINTER(C.c_void_p)]),
    "mbe_batch_size": (C.c_int, [C.c_void_p]),
    "mbe_batch_set_tuning": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(Params)]),
    "mbe_batch_get_tuning": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(Params)]),
    "mbe_batch_run": (C.c_int, [C.c_void_p, C.POINTER(Params), C.POINTER(Result),
                                C.POINTER(Result)]),
    "mbe_batch_autotune": (C.c_int, [C.c_void_p, C.POINTER(Params), C.c_int32, _P32]),
    "mbe_batch_free": (C.c_int, [C.c_void_p]),
    "mbe_server_config_default": (None, [C.POINTER(ServerConfig)]),
    "mbe_server_create": (C.c_int, [C.POINTER(ServerConfig), C.POINTER(Params),
                                    C.POINTER(C.c_void_p)]),
    "mbe_server_submit": (C.c_int, [C.c_void_p, _P32, _P32, C.c_int32, C.c_int32, C.c_int64,
                                    C.POINTER(Opts), C.POINTER(C.c_uint64)]),
    "mbe_server_poll": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(Result)]),
    "mbe_server_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.c_int64, C.POINTER(Result)]),
    "mbe_server_cancel": (C.c_int, [C.c_void_p, C.c_uint64]),
    "mbe_server_get_stats": (C.c_int, [C.c_void_p, C.POINTER(ServerStats)]),
    "mbe_server_destroy": (C.c_int, [C.c_void_p]),
    "mbe_server_set_emit": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]),
    "mbe_measure_l2_read": (C.c_int, [C.c_int32, C.c_int64, C.c_int32, C.POINTER(C.c_double)]),
    "mbe_server_debug_request": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
}
for _name, (_res, _args) in _sig.items():
    _f = getattr(_lib, _name)
    _f.restype = _res
    _f.argtypes = _args


def last_error() -> str:
    s = _lib.mbe_last_error_string()
    return s.decode() if s else ""


def _check(rc: int):
    if rc != MBE_OK:
        raise MBEError(rc, last_error())


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_P32)


def release_device(device: int = 0):
    """mbe_device_release: hands back the device memory cached between calls."""
    _check(_lib.mbe_device_release(int(device)))


def default_params(**kw) -> Params:
    p = Params()
    _lib.mbe_params_default(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise TypeError(f"unknown parameter {k}")
        setattr(p, k, v)
    return p


def make_opts(uvtrans=0, order=1, fast_mode=1, device=0) -> Opts:
    return Opts(uvtrans, order, fast_mode, device)


_EMIT_FN = C.CFUNCTYPE(C.c_int, C.POINTER(C.c_int32), C.c_int32, C.POINTER(C.c_int32), C.c_int32,
                       C.c_void_p)
_SERVER_EMIT_FN = C.CFUNCTYPE(C.c_int, C.c_uint64, C.POINTER(C.c_int32), C.c_int32,
                              C.POINTER(C.c_int32), C.c_int32, C.c_void_p)


class Graph:
    """A bipartite graph resident on the GPU (reference CSRBiGraph after
    Read + CopyToGpu).  V rows are .adj lines, entries U ids."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle)

    @classmethod
    def from_csr(cls, row_off, col, nU: int = 0, uvtrans=0, order=1, fast_mode=1, device=0):
        ro, co = _i32(row_off), _i32(col)
        h = C.c_void_p()
        opts = make_opts(uvtrans, order, fast_mode, device)
        _check(_lib.mbe_graph_from_csr(_ptr(ro), _ptr(co), len(ro) - 1, int(nU), len(co),
                                       C.byref(opts), C.byref(h)))
        return cls(h.value)

    @classmethod
    def build_on_device(cls, row_off, col, nU: int = 0, uvtrans=0, order=1, fast_mode=1,
                        device=0):
        """from_csr with the transposes, ordering, keys and capacities computed
        on the GPU (mbe_graph_build_on_device); rows of equal degree keep their
        input order, which leaves the enumerated set unchanged."""
        ro, co = _i32(row_off), _i32(col)
        h = C.c_void_p()
        opts = make_opts(uvtrans, order, fast_mode, device)
        _check(_lib.mbe_graph_build_on_device(_ptr(ro), _ptr(co), len(ro) - 1, int(nU), len(co),
                                              C.byref(opts), C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_adj(cls, path: str, uvtrans=0, order=1, fast_mode=1, device=0):
        h = C.c_void_p()
        opts = make_opts(uvtrans, order, fast_mode, device)
        _check(_lib.mbe_graph_from_adj(os.fsencode(path), C.byref(opts), C.byref(h)))
        return cls(h.value)

    def info(self) -> GraphInfo:
        i = GraphInfo()
        _check(_lib.mbe_graph_get_info(self._h, C.byref(i)))
        return i

    def enumerate(self, **params) -> Result:
        p = default_params(**params)
        r = Result()
        _check(_lib.mbe_enumerate(self._h, C.byref(p), C.byref(r)))
        return r

    def enumerate_emit(self, buf_words: int = 1 << 22, **params):
        """mbe_enumerate_emit: (Result, [(U ids, V ids), ...]) in original ids."""
        p = default_params(**params)
        r = Result()
        buf = np.zeros(max(buf_words, 2), np.int32)
        used = C.c_int64()
        _check(_lib.mbe_enumerate_emit(self._h, C.byref(p), C.byref(r), _ptr(buf), buf_words,
                                       C.byref(used)))
        out, pos, n = [], 0, used.value
        while pos < n:
            nu, nv = int(buf[pos]), int(buf[pos + 1])
            us = tuple(int(x) for x in buf[pos + 2:pos + 2 + nu])
            vs = tuple(int(x) for x in buf[pos + 2 + nu:pos + 2 + nu + nv])
            out.append((us, vs))
            pos += 2 + nu + nv
        return r, out

    def enumerate_stream(self, on_biclique, ring_words: int = 1 << 22, **params) -> Result:
        """mbe_enumerate_emit_stream: calls on_biclique(U ids, V ids) (tuples,
        original ids) for every maximal biclique while the launch runs; a true
        return value stops the calls.  Returns the Result."""
        p = default_params(**params)
        r = Result()
        err = []

        def cb(u, nu, v, nv, _user):
            try:
                return 1 if on_biclique(tuple(u[:nu]), tuple(v[:nv])) else 0
            except Exception as e:  # noqa: BLE001 - surfaced after the call
                err.append(e)
                return 1

        f = _EMIT_FN(cb)
        rc = _lib.mbe_enumerate_emit_stream(self._h, C.byref(p), C.byref(r), int(ring_words),
                                            C.cast(f, C.c_void_p), None)
        if err:
            raise err[0]
        _check(rc)
        return r

    def free(self):
        if self._h and self._h.value:
            _lib.mbe_graph_free(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.free()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Batch:
    """Many graphs in one device arena, enumerated in one persistent launch
    (captured in a CUDA graph on the first run, replayed after that)."""

    def __init__(self, graphs, uvtrans=1, order=1, fast_mode=1, device=0):
        self._keep = [(_i32(g.row_off), _i32(g.col)) for g in graphs]
        n = len(graphs)
        ros = (_P32 * n)(*[_ptr(r) for r, _ in self._keep])
        cos = (_P32 * n)(*[_ptr(c) for _, c in self._keep])
        nvs = (C.c_int32 * n)(*[g.nV for g in graphs])
        nus = (C.c_int32 * n)(*[g.nU for g in graphs])
        nes = (C.c_int64 * n)(*[g.nE for g in graphs])
        opts = make_opts(uvtrans, order, fast_mode, device)
        h = C.c_void_p()
        _check(_lib.mbe_batch_from_csr(n, ros, cos, nvs, nus, nes, C.byref(opts), C.byref(h)))
        self._h = h
        self.n = n
        self._keep = None

    def run(self, **params):
        """Returns (per-graph results, totals)."""
        p = default_params(**params)
        per = (Result * self.n)()
        tot = Result()
        _check(_lib.mbe_batch_run(self._h, C.byref(p), per, C.byref(tot)))
        return list(per), tot

    def set_tuning(self, index=-1, **params):
        p = default_params(**params)
        _check(_lib.mbe_batch_set_tuning(self._h, index, C.byref(p)))

    def get_tuning(self, index):
        p = Params()
        _check(_lib.mbe_batch_get_tuning(self._h, index, C.byref(p)))
        return p

    def autotune(self, n_classes=4, **params):
        p = default_params(**params)
        chosen = (C.c_int32 * n_classes)()
        _check(_lib.mbe_batch_autotune(self._h, C.byref(p), n_classes, chosen))
        return list(chosen)

    def free(self):
        if self._h and self._h.value:
            _lib.mbe_batch_free(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.free()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Server:
    """Continuous-batching server on one GPU (mbe_server_* in include/mbe.h):
    graphs submitted at any time share one persistent launch."""

    def __init__(self, device=0, max_graphs=0, arena_bytes=0, max_v=0, max_degree=0,
                 max_two_hop=0, idle_exit_ns=0, prep_threads=0, **params):
        self._h = C.c_void_p()
        cfg = ServerConfig()
        _lib.mbe_server_config_default(C.byref(cfg))
        cfg.device = device
        for k, v in dict(max_graphs=max_graphs, arena_bytes=arena_bytes, max_v=max_v,
                         max_degree=max_degree, max_two_hop=max_two_hop,
                         idle_exit_ns=idle_exit_ns, prep_threads=prep_threads).items():
            if v:
                setattr(cfg, k, v)
        p = default_params(**params)
        h = C.c_void_p()
        _check(_lib.mbe_server_create(C.byref(cfg), C.byref(p), C.byref(h)))
        self._h = h

    def submit(self, row_off, col, nU=0, uvtrans=1, order=1, fast_mode=1) -> int:
        ro, co = _i32(row_off), _i32(col)
        rid = C.c_uint64()
        opts = make_opts(uvtrans, order, fast_mode)
        _check(_lib.mbe_server_submit(self._h, _ptr(ro), _ptr(co), len(ro) - 1, int(nU),
                                      len(co), C.byref(opts), C.byref(rid)))
        return rid.value

    def poll(self, rid: int):
        """The finished request's Result, or None while it runs."""
        r = Result()
        rc = _lib.mbe_server_poll(self._h, rid, C.byref(r))
        if rc == -12:  # MBE_ERR_AGAIN
            return None
        _check(rc)
        return r

    def wait(self, rid: int, timeout: float | None = None) -> Result:
        r = Result()
        ns = -1 if timeout is None else int(timeout * 1e9)
        _check(_lib.mbe_server_wait(self._h, rid, ns, C.byref(r)))
        if getattr(self, "_emit_err", None):
            raise self._emit_err.pop(0)
        return r

    def cancel(self, rid: int):
        _check(_lib.mbe_server_cancel(self._h, rid))

    def stats(self) -> dict:
        st = ServerStats()
        _check(_lib.mbe_server_get_stats(self._h, C.byref(st)))
        return st.as_dict()

    def set_emit(self, on_biclique, ring_words: int = 0):
        """mbe_server_set_emit: on_biclique(request id, U ids, V ids) (tuples,
        original ids) is called on the server's thread for every maximal
        biclique of every request submitted afterwards; a request's result is
        reported only after all its bicliques have been passed.  Call before
        the first submit.  An exception in on_biclique is kept and raised by
        the next wait()."""
        errs = []

        def cb(rid, u, nu, v, nv, _user):
            try:
                on_biclique(rid, tuple(u[:nu]), tuple(v[:nv]))
            except Exception as e:  # noqa: BLE001 - surfaced by wait()
                errs.append(e)
            return 0

        f = _SERVER_EMIT_FN(cb)
        _check(_lib.mbe_server_set_emit(self._h, int(ring_words), C.cast(f, C.c_void_p), None))
        # Only a callback the server took is kept (alive as long as the server);
        # a refused call leaves the one in use untouched.
        self._emit_cb = f
        self._emit_err = errs

    def debug_request(self, rid: int) -> dict:
        """A resident request's device counters (diagnosis)."""
        out = (C.c_uint64 * 4)()
        _check(_lib.mbe_server_debug_request(self._h, rid, out))
        return dict(roots_claimed=out[0], pending=out[1], n_roots=out[2], block=out[3])

    def close(self):
        if self._h and self._h.value:
            _lib.mbe_server_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Synthetic inputs.

@dataclass
class BipartiteCSR:
    row_off: np.ndarray  # int32 [nV+1]
    col: np.ndarray      # int32 [nE]
    nU: int

    @property
    def nV(self) -> int:
        return len(self.row_off) - 1

    @property
    def nE(self) -> int:
        return len(self.col)


def generate(spec: GenSpec) -> BipartiteCSR:
    ro, co = _P32(), _P32()
    nV, nU, nE = C.c_int32(), C.c_int32(), C.c_int64()
    _check(_lib.mbe_gen_chung_lu(C.byref(spec), C.byref(ro), C.byref(co), C.byref(nV),
                                 C.byref(nU), C.byref(nE)))
    try:
        r = np.ctypeslib.as_array(ro, (nV.value + 1,)).copy()
        c = (np.ctypeslib.as_array(co, (nE.value,)).copy() if nE.value
             else np.zeros(0, np.int32))
    finally:
        _lib.mbe_free(ro)
        _lib.mbe_free(co)
    return BipartiteCSR(r, c, nU.value)


def batch_spec(seed: int) -> GenSpec:
    s = GenSpec()
    _check(_lib.mbe_gen_batch_spec(C.c_uint64(seed), C.byref(s)))
    return s


def write_adj(path: str, g: BipartiteCSR):
    ro, co = _i32(g.row_off), _i32(g.col)
    _check(_lib.mbe_write_adj(os.fsencode(path), _ptr(ro), _ptr(co), g.nV))


def write_graph(path: str, g: BipartiteCSR):
    """Edge-pair .graph file for the CPU peers (mbe_write_graph)."""
    ro, co = _i32(g.row_off), _i32(g.col)
    _check(_lib.mbe_write_graph(os.fsencode(path), _ptr(ro), _ptr(co), g.nV))


def read_adj(path: str) -> BipartiteCSR:
    ro, co = _P32(), _P32()
    nV, nU, nE = C.c_int32(), C.c_int32(), C.c_int64()
    _check(_lib.mbe_read_adj(os.fsencode(path), C.byref(ro), C.byref(co), C.byref(nV),
                             C.byref(nU), C.byref(nE)))
    try:
        r = np.ctypeslib.as_array(ro, (nV.value + 1,)).copy()
        c = (np.ctypeslib.as_array(co, (nE.value,)).copy() if nE.value
             else np.zeros(0, np.int32))
    finally:
        _lib.mbe_free(ro)
        _lib.mbe_free(co)
    return BipartiteCSR(r, c, nU.value)


from .configs import CONFIGS, DESCRIPTIONS, batch_graph, config_graph  # noqa: E402,F401


def measure_l2_read(device: int = 0, nbytes: int = 32 << 20, passes: int = 100) -> float:
    """mbe_measure_l2_read: GB/s of L2-resident reads (one launch, `passes`
    sweeps over an `nbytes` buffer with L1-bypassing loads)."""
    out = C.c_double()
    _check(_lib.mbe_measure_l2_read(device, nbytes, passes, C.byref(out)))
    return out.value
