"""Batched enumeration: one persistent launch over many graphs.

Per-graph count and set hash must equal the single-graph path and the CPU
oracle, on every replay of the captured launch and after autotuning.
"""
import numpy as np
import pytest

import oracle
from util import planted, random_bipartite

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gm():
    import gmbe_b200
    return gmbe_b200


def _graphs(gm, n):
    # batched-workload graphs, the lighter ones (a few seconds of oracle time)
    gs = []
    seed = 1000
    while len(gs) < n:
        g = gm.batch_graph(seed)
        seed += 1
        if g.nE <= 20000:
            gs.append(g)
    for seed in range(3):  # a few dense ones with heavy subtrees
        ro, co, nU = planted(200, 150, blocks=4, seed=seed, bsize=12)
        gs.append(gm.BipartiteCSR(ro, co, nU))
    ro, co, nU = random_bipartite(30, 40, 0.3, 7)
    gs.append(gm.BipartiteCSR(ro, co, nU))
    return gs


def test_batch_matches_oracle_and_single_path(gm):
    gs = _graphs(gm, 24)
    want = [oracle.gmbe(g.row_off, g.col, g.nU) for g in gs]
    with gm.Batch(gs) as B:
        for rep in range(3):  # first run captures, later runs replay
            per, tot = B.run()
            for i, (r, w) in enumerate(zip(per, want)):
                assert (r.count, r.set_hash) == (w.count, w.set_hash), (rep, i)
            assert tot.count == sum(w.count for w in want)
    for i in (0, 5, len(gs) - 1):
        g = gs[i]
        with gm.Graph.from_csr(g.row_off, g.col, g.nU, uvtrans=1) as G:
            r = G.enumerate()
        assert (r.count, r.set_hash) == (want[i].count, want[i].set_hash)


def test_batch_autotune_keeps_results(gm):
    gs = _graphs(gm, 40)
    with gm.Batch(gs) as B:
        before, _ = B.run()
        chosen = B.autotune(n_classes=4)
        assert len(chosen) == 4
        after, _ = B.run()
        for a, b in zip(before, after):
            assert (a.count, a.set_hash) == (b.count, b.set_hash)
        # tuning of one graph can be read back
        t = B.get_tuning(0)
        assert t.bound_height > 0


@pytest.mark.parametrize("split_mode", [0, 1])
def test_batch_split_modes(gm, split_mode):
    gs = _graphs(gm, 12)
    want = [oracle.gmbe(g.row_off, g.col, g.nU) for g in gs]
    with gm.Batch(gs) as B:
        B.set_tuning(-1, bound_height=2, bound_size=10)
        per, _ = B.run(split_mode=split_mode)
    for r, w in zip(per, want):
        assert (r.count, r.set_hash) == (w.count, w.set_hash)


@pytest.mark.last
def test_full_batched_workload_matches_oracle_fixture(gm):
    # The whole batched workload (4,096 graphs, seeds 1000..5095) in one
    # launch: every per-graph count and set hash on two replays equals the
    # CPU oracle's, committed in tests/golden/batch_oracle.json
    # (tests/golden/make_batch_oracle.py).
    import json
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "batch_oracle.json")
    with open(path) as f:
        orc = json.load(f)
    want = list(zip(orc["count"], (int(h, 16) for h in orc["set_hash"])))
    gs = [gm.batch_graph(orc["first_seed"] + i) for i in range(orc["n"])]
    with gm.Batch(gs) as B:
        for rep in range(2):
            per, tot = B.run()
            bad = [i for i, r in enumerate(per) if (r.count, r.set_hash) != want[i]]
            assert not bad, (rep, bad[:10])
            assert tot.count == orc["total_count"]
