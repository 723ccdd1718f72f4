"""Generates tests/golden/large_ranges.json: the CPU oracle's maximal-biclique
count and set hash on root ranges of the large configuration (2M x 8M
Chung-Lu, exponents 2.1/2.2, cap 50,000, seed 3, ~60M edges; flags -t 1 -o 1
-f, bounds 20/1500).

The whole graph is far beyond what the oracle enumerates in minutes (roots at
the top of the degree order take minutes each), so parity on this
configuration is pinned on ranges of the internal root order that the oracle
finishes in seconds.  Each range also records the largest two-hop multiset
(sum of the root's neighbours' degrees) among its roots, the quantity that
sizes a launch's per-warp scratch, and a checksum of the generated CSR so a
test can tell a changed generator from a changed enumerator.

usage: python tests/golden/make_large_ranges.py
"""
import ctypes as C
import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import gmbe_b200 as gm  # noqa: E402
import oracle  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "large_ranges.json")
RANGES = [(0, 20000), (1000000, 1005000), (1500000, 1502000), (1700000, 1700500),
          (1800000, 1800200)]


def digest(ro, co):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(ro, np.int32).tobytes())
    h.update(np.ascontiguousarray(co, np.int32).tobytes())
    return h.hexdigest()[:16]


def internal_two_hop(ro, co, nU, degrees=False):
    """Two-hop multiset size of every internal root, in the oracle's internal
    order (-t 1 -o 1), and with degrees=True each root's degree as well."""
    ro = np.ascontiguousarray(ro, np.int32)
    co = np.ascontiguousarray(co, np.int32)
    nV = len(ro) - 1
    P = C.POINTER(C.c_int32)
    v_orig = np.zeros(max(nV, nU), np.int32)
    n_int = C.c_int32()
    oracle.lib().orc_internal_order(nV, nU, ro.ctypes.data_as(P), co.ctypes.data_as(P), 1, 1,
                                    v_orig.ctypes.data_as(P), C.byref(n_int))
    dv = np.diff(ro.astype(np.int64))
    du = np.bincount(co, minlength=nU).astype(np.int64)
    if n_int.value == nV:  # V rows stay the roots
        s = np.add.reduceat(du[co], ro[:-1].astype(np.int64))
        d = dv
    else:  # -t swapped the sides: U vertices are the roots
        s = np.bincount(co, weights=dv[np.repeat(np.arange(nV), dv)], minlength=nU)
        d = du
    order = v_orig[: n_int.value]
    if degrees:
        return s.astype(np.int64)[order], d.astype(np.int32)[order], n_int.value
    return s.astype(np.int64)[order], n_int.value


def main():
    t = time.time()
    g = gm.config_graph("large")
    print(f"generated in {time.time() - t:.1f} s: {len(g.row_off) - 1} rows, {len(g.col)} edges",
          flush=True)
    s_int, n_int = internal_two_hop(g.row_off, g.col, g.nU)
    ranges = []
    for a, b in RANGES:
        t = time.perf_counter()
        o = oracle.gmbe_range(g.row_off, g.col, g.nU, a, b, uvtrans=1)
        dt = time.perf_counter() - t
        ranges.append({"root_begin": a, "root_end": b, "count": int(o.count),
                       "set_hash": f"{o.set_hash:#018x}", "max_two_hop": int(s_int[a:b].max()),
                       "alg_bytes": int(o.alg_bytes), "oracle_seconds": round(dt, 1)})
        print(ranges[-1], flush=True)
    with open(OUT, "w") as f:
        json.dump({"generator": "tests/golden/make_large_ranges.py", "config": "large",
                   "flags": "-t 1 -o 1 -f, bounds 20/1500, pruning on",
                   "csr_sha256_16": digest(g.row_off, g.col), "internal_nV": int(n_int),
                   "ranges": ranges}, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
