"""Pins the oracle's large-configuration shard counts against the reference's
own CPU enumerator: runs MbeaFinderBitset (src/BicliqueFinder.cu:59-197,
built from the reference's sources into oracle/_ref/ref_mbea by
`make -C oracle ref`) on every root of each shard in
tests/golden/large_shards.json and records its count beside the oracle's as
`reference_count` (with `reference_seconds` and the thread count).

The .adj it reads is the large workload written by the stand-alone generator
(gmbe_b200/mbe_gen), so the reference parses, swaps and orders it itself
(-t 1 -o 1 -f).  Shard s is the roots at positions s, s + 20000, ... from the
top of the internal order; in the reference's order counted from the lowest
degree, that is offset (nV - 1 - s) mod 20000.  The reference's count covers
the count only (its enumerators do not report bicliques).

usage: python tests/golden/pin_large_shards_reference.py [--threads N] [--shards a,b,...]
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
FIXTURE = os.path.join(ROOT, "tests", "golden", "large_shards.json")
RANGES = os.path.join(ROOT, "tests", "golden", "large_ranges.json")
REF = os.path.join(ROOT, "oracle", "_ref", "ref_mbea")
GEN = os.path.join(ROOT, "gmbe_b200", "mbe_gen")
WORKLOADS = os.path.join(ROOT, "gmbe_b200", "workloads.json")
STRIDE = 20000


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--shards", default="")
    args = ap.parse_args()
    with open(FIXTURE) as f:
        fx = json.load(f)
    with open(RANGES) as f:
        nv = json.load(f)["internal_nV"]
    shards = [int(x) for x in args.shards.split(",") if x] or \
        [sh["shard_index"] for sh in fx["shards"]]
    offsets = [(nv - 1 - s) % STRIDE for s in shards]
    with open(WORKLOADS) as f:
        w = json.load(f)
    spec = w["workloads"]["large"]["spec"]
    with tempfile.TemporaryDirectory() as d:
        adj = os.path.join(d, "large.adj")
        subprocess.run([GEN, adj] + [str(spec[k]) for k in w["fields"]], check=True,
                       capture_output=True)
        # One run over all shards (the graph is read once); a line per shard.
        p = subprocess.Popen([REF, adj, "2", "1", "1", str(STRIDE),
                              ",".join(str(o) for o in offsets) + ",", "0", str(args.threads),
                              "0"], stdout=subprocess.PIPE, text=True)
        done = 0
        for line in p.stdout:
            f = line.split()
            if not f or f[0] != "sample":
                continue
            off, roots, count, secs = int(f[1]), int(f[3]), int(f[5]), float(f[7])
            s = shards[offsets.index(off)]
            for sh in fx["shards"]:
                if sh["shard_index"] == s:
                    sh["reference_count"] = count
                    sh["reference_seconds"] = round(secs, 1)
                    sh["reference_threads"] = args.threads
                    print(f"shard {s}: {roots} roots, reference {count}, oracle {sh['count']}, "
                          f"{secs:.1f} s", flush=True)
            fx["reference_tool"] = ("MbeaFinderBitset (oracle/_ref/ref_mbea, built from the "
                                    "reference's sources), every root of the shard")
            with open(FIXTURE, "w") as f2:  # after every shard: a stopped run keeps its pins
                json.dump(fx, f2, indent=1)
                f2.write("\n")
            done += 1
        if p.wait() != 0:
            sys.exit(f"ref_mbea exited with status {p.returncode} after {done} shards")


if __name__ == "__main__":
    t0 = time.time()
    main()
    print(f"done in {time.time() - t0:.0f} s")
