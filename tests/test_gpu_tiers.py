"""Two scratch tiers (mbe_params.big_two_hop / big_warps): roots whose two-hop
multiset exceeds the bound run on a pool of warps sized for the largest root,
every other warp is sized for the bound.  Which warp runs a root must not
change the enumerated set: count and set hash equal the oracle's, bit for bit.

The bound is forced low here so that small graphs take the two-tier path;
without it the path is taken only when one layout for every warp does not fit
the device.  Device waits are bounded at 30 s so that a scheduling error shows
as a failed status, not a stall.
"""
import numpy as np
import pytest

import oracle
from util import hub_graph, planted, random_bipartite

pytestmark = [pytest.mark.gpu, pytest.mark.last]
WAIT = 30 * 10**9


@pytest.fixture(scope="module")
def gm():
    import gmbe_b200
    return gmbe_b200


def two_hop(ro, co, nU):
    """Two-hop multiset size of every V row (sum of its neighbours' degrees)."""
    du = np.bincount(co, minlength=nU)
    return np.add.reduceat(du[co], ro[:-1])


CASES = [("planted", lambda: planted(300, 200, blocks=6, seed=3, bsize=14)),
         ("hub", lambda: hub_graph(1)),
         ("dense", lambda: random_bipartite(40, 60, 0.3, 2))]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("big_warps", [0, 1, 5])
def test_two_tiers_match_oracle(gm, name, make, big_warps):
    ro, co, nU = make()
    want = oracle.gmbe(ro, co, nU)
    for uvtrans in (0, 1):
        with gm.Graph.from_csr(ro, co, nU, uvtrans=uvtrans) as G:
            s = two_hop(ro, co, nU) if uvtrans == 0 else None
            # a bound below the median root: most roots go to the big warps
            bound = int(np.median(s)) if s is not None else 64
            r = G.enumerate(big_two_hop=max(bound, 1), big_warps=big_warps, wait_limit_ns=WAIT)
        assert r.status == 0
        assert (r.count, r.set_hash) == (want.count, want.set_hash)


def test_two_tiers_every_root_big_and_none_big(gm):
    ro, co, nU = planted(200, 150, blocks=5, seed=17, bsize=12)
    want = oracle.gmbe(ro, co, nU)
    with gm.Graph.from_csr(ro, co, nU, uvtrans=1) as G:
        for bound in (1, 1 << 30):  # every root above the bound / none
            r = G.enumerate(big_two_hop=bound, wait_limit_ns=WAIT)
            assert (r.count, r.set_hash) == (want.count, want.set_hash)
        # one tier again on the same workspace afterwards
        r = G.enumerate(wait_limit_ns=WAIT)
        assert (r.count, r.set_hash) == (want.count, want.set_hash)


def test_two_tiers_shards_and_ranges_add_up(gm):
    ro, co, nU = hub_graph(2)
    want = oracle.gmbe(ro, co, nU)
    M = (1 << 64) - 1
    with gm.Graph.from_csr(ro, co, nU, uvtrans=1) as G:
        nV = G.info().V_size
        tot, h = 0, 0
        for si in range(3):
            r = G.enumerate(shard_count=3, shard_index=si, big_two_hop=200, big_warps=2,
                            wait_limit_ns=WAIT)
            tot, h = tot + r.count, (h + r.set_hash) & M
        assert (tot, h) == (want.count, want.set_hash)
        tot, h = 0, 0
        for a, b in ((0, nV // 3), (nV // 3, nV)):
            r = G.enumerate(root_begin=a, root_end=b, big_two_hop=200, wait_limit_ns=WAIT)
            tot, h = tot + r.count, (h + r.set_hash) & M
        assert (tot, h) == (want.count, want.set_hash)


def test_two_tiers_emit_the_same_set(gm):
    ro, co, nU = planted(200, 150, blocks=5, seed=17, bsize=12)
    with gm.Graph.from_csr(ro, co, nU, uvtrans=1) as G:
        r1, one = G.enumerate_emit(buf_words=1 << 24, wait_limit_ns=WAIT)
        r2, two = G.enumerate_emit(buf_words=1 << 24, big_two_hop=100, wait_limit_ns=WAIT)
    assert (r2.count, r2.set_hash) == (r1.count, r1.set_hash)
    assert len(two) == len(set(two)) == r2.count
    assert set(two) == set(one)


def test_two_tiers_need_split_mode_0(gm):
    ro, co, nU = planted(100, 80, blocks=2, seed=5)
    with gm.Graph.from_csr(ro, co, nU) as G:
        with pytest.raises(gm.MBEError) as ei:
            G.enumerate(big_two_hop=10, split_mode=1)
    assert ei.value.name == "MBE_ERR_INVALID"


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("work,chunk", [(1, 1), (50, 4), (400, 64)])
def test_two_tiers_with_root_parts(gm, name, make, work, chunk):
    # Roots split into parts: a listed big root's parts go through the part
    # records that only big warps claim, the other roots' parts through the
    # common queue.  Thresholds this low split nearly every root.
    ro, co, nU = make()
    want = oracle.gmbe(ro, co, nU)
    with gm.Graph.from_csr(ro, co, nU, uvtrans=1) as G:
        for big_warps in (0, 2):
            r = G.enumerate(big_two_hop=64, big_warps=big_warps, range_split_work=work,
                            range_chunk=chunk, wait_limit_ns=WAIT)
            assert r.status == 0
            assert (r.count, r.set_hash) == (want.count, want.set_hash)
            if chunk == 1:
                assert r.tasks_split > 0
