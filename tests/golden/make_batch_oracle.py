"""Generates tests/golden/batch_oracle.json: the CPU oracle's maximal-biclique
count and set hash for every graph of the batched workload (4,096 Chung-Lu
graphs, seeds 1000..5095, exponent 2.2, |U| log-uniform in [50, 5000],
|V|/|U| log-uniform in [0.5, 4], average degree uniform in [3, 30]; flags
-t 1 -o 1 -f, bounds 20/1500, pruning on).  Graph i is seed 1000 + i.

The benchmark's batched leg and tests/test_gpu_batch.py compare every
per-graph result of the batched launch with these.

usage: python tests/golden/make_batch_oracle.py [--threads N] [--n 4096]
"""
import argparse
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import gmbe_b200 as gm  # noqa: E402
import oracle  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "batch_oracle.json")
FIRST_SEED = 1000


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--n", type=int, default=4096)
    a = ap.parse_args()
    counts, hashes = [], []
    t0 = time.time()
    for i in range(a.n):
        g = gm.batch_graph(FIRST_SEED + i)
        o = oracle.gmbe(g.row_off, g.col, g.nU, uvtrans=1, order=1, threads=a.threads)
        counts.append(int(o.count))
        hashes.append(f"{o.set_hash:#018x}")
        if i % 256 == 255:
            print(f"{i + 1} graphs, {sum(counts)} bicliques, {time.time() - t0:.0f} s", flush=True)
    with open(OUT, "w") as f:
        json.dump({"generator": "tests/golden/make_batch_oracle.py", "first_seed": FIRST_SEED,
                   "n": a.n, "flags": "-t 1 -o 1 -f, bounds 20/1500, pruning on",
                   "total_count": sum(counts), "oracle_seconds": round(time.time() - t0, 1),
                   "count": counts, "set_hash": hashes}, f, separators=(",", ":"))
    print("wrote", OUT, sum(counts))


if __name__ == "__main__":
    main()
