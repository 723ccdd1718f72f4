"""Pins the batched workload's oracle fixture against the reference's own CPU
enumerator: writes each graph of tests/golden/batch_oracle.json (seeds
1000..5095) as an .adj file and runs MbeaFinderBitset on it
(src/BicliqueFinder.cu:59-197, built from the reference's sources into
oracle/_ref/ref_mbea by `make -C oracle ref`; selector 1, -t 1 -o 1), reading
the reference's own result line "maximal nodes:<n>".  The counts are stored
beside the oracle's as `reference_count` (the reference reports counts only,
so the set hashes rest on the oracle).

usage: python tests/golden/pin_batch_reference.py [--procs N]
"""
import argparse
import json
import multiprocessing as mp
import os
import re
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
FIXTURE = os.path.join(ROOT, "tests", "golden", "batch_oracle.json")
REF = os.path.join(ROOT, "oracle", "_ref", "ref_mbea")


def _count(args):
    seed, d = args
    sys.path.insert(0, ROOT)
    import gmbe_b200 as gm
    path = os.path.join(d, f"g{seed}.adj")
    gm.write_adj(path, gm.batch_graph(seed))
    out = subprocess.run([REF, path, "1", "1", "1"], check=True, capture_output=True,
                         text=True).stdout
    os.remove(path)
    return int(re.search(r"^maximal nodes:(\d+)$", out, re.M).group(1))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--procs", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    with open(FIXTURE) as f:
        fx = json.load(f)
    seeds = [fx["first_seed"] + i for i in range(fx["n"])]
    t0 = time.time()
    with tempfile.TemporaryDirectory() as d:
        with mp.get_context("spawn").Pool(args.procs) as pool:
            counts = pool.map(_count, [(s, d) for s in seeds], chunksize=8)
    fx["reference_count"] = counts
    fx["reference_tool"] = ("MbeaFinderBitset (oracle/_ref/ref_mbea, built from the reference's "
                            "sources), whole graph, -t 1 -o 1")
    fx["reference_seconds"] = round(time.time() - t0, 1)
    with open(FIXTURE, "w") as f:
        json.dump(fx, f, separators=(",", ":"))
    bad = [i for i, (a, b) in enumerate(zip(counts, fx["count"])) if a != b]
    print(f"{len(counts)} graphs, {sum(counts)} bicliques, {len(bad)} differ from the oracle "
          f"({fx['reference_seconds']} s)")


if __name__ == "__main__":
    main()
