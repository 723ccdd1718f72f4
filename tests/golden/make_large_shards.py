"""Generates tests/golden/large_shards.json: the CPU oracle's maximal-biclique
count and set hash on interleaved root shards of the large configuration
(2M x 8M Chung-Lu, exponents 2.1/2.2, cap 50,000, seed 3, ~60M edges; flags
-t 1 -o 1 -f, bounds 20/1500, pruning on).

A shard (offset o, stride s) is the roots at positions o, o + s, o + 2s, ...
from the top of the internal degree order, the same positions the engine
enumerates with shard_count = s, shard_index = o.  Unlike a contiguous range,
a shard samples every part of the degree order, the heaviest roots at the top
included, so it pins the roots whose subtrees dominate a whole-graph launch.
The whole graph is far beyond the oracle (a 1-in-20,000 shard takes 3-6
minutes on 8 cores: roughly 10^5-10^6 CPU-seconds for all roots).

usage: python tests/golden/make_large_shards.py [--threads N] [--offsets a,b,...]
       (new shards are merged into the existing file)
"""
import argparse
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import gmbe_b200 as gm  # noqa: E402
import oracle  # noqa: E402
from make_large_ranges import digest  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "large_shards.json")
STRIDE = 20000
OFFSETS = [0, 7, 9999]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--offsets", default=",".join(str(o) for o in OFFSETS))
    a = ap.parse_args()
    offsets = [int(x) for x in a.offsets.split(",") if x]
    t = time.time()
    g = gm.config_graph("large")
    print(f"generated in {time.time() - t:.1f} s", flush=True)
    shards = []
    if os.path.exists(OUT):
        with open(OUT) as f:
            shards = [x for x in json.load(f)["shards"] if x["shard_index"] not in offsets]
    for off in offsets:
        t = time.perf_counter()
        o = oracle.gmbe_strided(g.row_off, g.col, g.nU, off, STRIDE, uvtrans=1, threads=a.threads)
        dt = time.perf_counter() - t
        shards.append({"shard_index": off, "shard_count": STRIDE, "count": int(o.count),
                       "set_hash": f"{o.set_hash:#018x}", "non_maximal": int(o.non_maximal),
                       "alg_bytes": int(o.alg_bytes), "oracle_seconds": round(dt, 1)})
        print(shards[-1], flush=True)
        # merge with what other runs wrote meanwhile
        if os.path.exists(OUT):
            with open(OUT) as f:
                have = {x["shard_index"]: x for x in json.load(f)["shards"]}
            for x in shards:
                have[x["shard_index"]] = x
            shards = sorted(have.values(), key=lambda x: x["shard_index"])
        with open(OUT, "w") as f:
            json.dump({"generator": "tests/golden/make_large_shards.py", "config": "large",
                       "flags": "-t 1 -o 1 -f, bounds 20/1500, pruning on",
                       "csr_sha256_16": digest(g.row_off, g.col), "shards": shards}, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
