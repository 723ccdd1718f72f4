"""Generates tests/golden/golden.json: reference results on seeded graphs.

Runs the reference's own CPU enumerators, built from the reference sources by
`make -C oracle ref` (oracle/_ref/ref_mbea: MbeaFinder and MbeaFinderBitset
from src/BicliqueFinder.cu; oracle/_ref/MBE: MBEA/iMBEA/PMBE from
baselines/MBE.zip), on .adj files written from the seeded generator, and
records their maximal-biclique counts.  The set hash is recorded from the
CPU oracle (the reference prints counts only); on graphs with |U| <= 64 the
brute-force closure pins it independently.

Each case also records a checksum of the generated CSR so a test can tell a
changed generator from a changed enumerator.

usage: python tests/golden/make_golden.py [--with-medium]
"""
import argparse
import hashlib
import json
import os
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import gmbe_b200 as gm  # noqa: E402
import oracle  # noqa: E402
from util import planted, random_bipartite  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")
CONSTS = os.path.join(ROOT, "gmbe_b200", "workload_constants.json")


def csr_digest(ro, co):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(ro, np.int32).tobytes())
    h.update(np.ascontiguousarray(co, np.int32).tobytes())
    return h.hexdigest()[:16]


def run_ref(args, timeout):
    t = time.time()
    out = subprocess.run(args, capture_output=True, text=True, timeout=timeout).stdout
    m = re.search(r"maximal nodes:(-?\d+)", out) or re.search(r"maximal nodes/processing nodes : (\d+)/", out)
    return (int(m.group(1)) if m else None), time.time() - t


def case(name, ro, co, nU, ref_timeout=600, uvtrans=1, refs_to_run=None):
    entry = {"name": name, "nV": int(len(ro) - 1), "nU": int(nU), "nE": int(len(co)),
             "csr_sha256_16": csr_digest(ro, co)}
    t = time.time()
    o = oracle.gmbe(ro, co, nU, uvtrans=uvtrans)
    entry["oracle_seconds"] = round(time.time() - t, 3)
    entry["oracle_count"] = int(o.count)
    entry["oracle_set_hash"] = f"{o.set_hash:#018x}"
    entry["oracle_alg_bytes"] = int(o.alg_bytes)
    if nU <= 64:
        bf = oracle.brute_force(ro, co, nU)
        entry["brute_force_count"] = int(bf.count)
        entry["brute_force_set_hash"] = f"{bf.set_hash:#018x}"
    refs = {}
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, f"{name}.adj")
        gm.write_adj(path, gm.BipartiteCSR(np.asarray(ro), np.asarray(co), nU))
        mbea = oracle.ref_binary("ref_mbea")
        mbe = oracle.ref_binary("MBE")
        want = refs_to_run or ("MbeaFinderBitset", "MbeaFinder", "PMBE", "iMBEA", "MBEA")
        if mbea:
            for sel, label in ((1, "MbeaFinderBitset"), (0, "MbeaFinder")):
                if label not in want:
                    continue
                try:
                    c, t = run_ref([mbea, path, str(sel), str(uvtrans), "1"], ref_timeout)
                    refs[label] = {"count": c, "seconds": round(t, 3)}
                except subprocess.TimeoutExpired:
                    refs[label] = {"count": None, "timeout_s": ref_timeout}
        if mbe:
            for sel, label in ((2, "PMBE"), (1, "iMBEA"), (0, "MBEA")):
                if label not in want:
                    continue
                try:
                    c, t = run_ref([mbe, "-i", path, "-s", str(sel)], ref_timeout)
                    refs[label] = {"count": c, "seconds": round(t, 3)}
                except subprocess.TimeoutExpired:
                    refs[label] = {"count": None, "timeout_s": ref_timeout}
    entry["reference"] = refs
    print(json.dumps(entry), flush=True)
    return entry


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--with-medium", action="store_true")
    a = ap.parse_args()
    cases = []
    for seed in range(4):
        ro, co, nU = random_bipartite(40, 48, 0.25, seed)
        cases.append(case(f"tiny_random_{seed}", ro, co, nU, ref_timeout=120))
    ro, co, nU = planted(300, 200, blocks=6, seed=3, bsize=14)
    cases.append(case("planted_300x200", ro, co, nU))
    g = gm.config_graph("small")
    cases.append(case("config_small", g.row_off, g.col, g.nU))
    for seed in (1000, 1001, 1002):
        b = gm.batch_graph(seed)
        cases.append(case(f"batch_{seed}", b.row_off, b.col, b.nU))
    if a.with_medium:
        g = gm.config_graph("medium")
        c = case("config_medium", g.row_off, g.col, g.nU, ref_timeout=2400,
                 refs_to_run=("MbeaFinderBitset", "PMBE"))
        cases.append(c)
        consts = {"medium": {"count": c["oracle_count"], "set_hash": c["oracle_set_hash"],
                             "alg_bytes": c["oracle_alg_bytes"],
                             "csr_sha256_16": c["csr_sha256_16"],
                             "flags": "-t 1 -o 1 -f, pruning on",
                             "source": "tests/golden/make_golden.py --with-medium (CPU oracle)"}}
        if os.path.exists(CONSTS):  # keep the measured (ncu) figures
            with open(CONSTS) as f:
                old = json.load(f).get("medium", {})
            consts["medium"].update({k: v for k, v in old.items() if k.startswith("traffic")})
        with open(CONSTS, "w") as f:
            json.dump(consts, f, indent=1)
        print("wrote", CONSTS)
    elif os.path.exists(OUT):
        # The medium case takes minutes (and the reference's CPU enumerators
        # longer): keep the recorded one unless asked to recompute it.
        with open(OUT) as f:
            old = [c for c in json.load(f)["cases"] if c["name"] == "config_medium"]
        cases.extend(old)
    with open(OUT, "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": cases}, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
