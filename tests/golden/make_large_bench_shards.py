"""Generates tests/golden/large_bench_shards.json: the count and set hash of
each interleaved root shard (positions p = s mod 512 of the internal degree
order) of the large configuration that the benchmark enumerates (2M x 8M
Chung-Lu, exponents 2.1/2.2, cap 50,000, seed 3; flags -t 1 -o 1 -f, bounds
20/1500, pruning on).  Needs a GPU.

A 1/512 shard holds about 24 million bicliques: beyond the CPU oracle (its
1/20000 shards take 4-17 minutes on 8 cores, tests/golden/large_shards.json).
So these pins come from the engine run under a second schedule whose
push, pop and maximality code differs from the default one's for almost
every task: every task in the counts tier (bitmap_max_l = -1, the bitmap tier
off), GMBE's vertex-tuple children for sharing (split_mode = 1).  The
benchmark's default schedule (bitmap tier, sub-problem sharing) must agree
with them on every step.  Both schedules agree with the oracle on the
pinned 1/20000 shards and root ranges (tests/test_gpu_large.py).

usage: python tests/golden/make_large_bench_shards.py [first] [last]
       (shards first..last inclusive; default 0..39 and 492..511, the shards a
       default benchmark run takes; results are merged into the file)
"""
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import gmbe_b200 as gm  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "large_bench_shards.json")
SHARDS = 512
SCHEDULE = dict(bitmap_max_l=-1, split_mode=1)


def main():
    if len(sys.argv) == 3:
        todo = list(range(int(sys.argv[1]), int(sys.argv[2]) + 1))
    else:
        todo = list(range(0, 40)) + list(range(SHARDS - 20, SHARDS))
    d = {"generator": "tests/golden/make_large_bench_shards.py", "config": "large",
         "flags": "-t 1 -o 1 -f, bounds 20/1500, pruning on", "shard_count": SHARDS,
         "schedule": SCHEDULE, "shards": {}}
    if os.path.exists(OUT):
        with open(OUT) as f:
            d["shards"] = json.load(f).get("shards", {})
    g = gm.config_graph("large")
    with gm.Graph.from_csr(g.row_off, g.col, g.nU, uvtrans=1, order=1) as G:
        for s in todo:
            t = time.perf_counter()
            r = G.enumerate(shard_count=SHARDS, shard_index=s, **SCHEDULE)
            d["shards"][str(s)] = {"count": int(r.count), "set_hash": f"{r.set_hash:#018x}",
                                   "kernel_ms": round(r.kernel_ms, 1)}
            print(s, d["shards"][str(s)], f"{time.perf_counter() - t:.1f} s", flush=True)
            with open(OUT, "w") as f:
                json.dump(d, f, indent=1)


if __name__ == "__main__":
    main()
