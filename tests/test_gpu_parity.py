"""GPU parity: the engine (through the C ABI) against the CPU oracle.

The bar is bit-exact equality of the maximal-biclique count and of the
canonical set hash.  Oracle sizes are kept to seconds.
"""
import numpy as np
import pytest

import oracle
from util import hub_graph, planted, random_bipartite

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gm():
    import gmbe_b200
    return gmbe_b200


def run(gm, ro, co, nU, opts=None, **params):
    opts = opts or {}
    with gm.Graph.from_csr(ro, co, nU, **opts) as g:
        return g.enumerate(**params)


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("shape", [(12, 10, 0.4), (30, 40, 0.25), (40, 60, 0.15), (64, 48, 0.3)])
def test_tiny_vs_brute_force(gm, seed, shape):
    nV, nU, p = shape
    ro, co, nU = random_bipartite(nV, nU, p, seed)
    bf = oracle.brute_force(ro, co, nU)
    r = run(gm, ro, co, nU)
    assert (r.count, r.set_hash) == (bf.count, bf.set_hash)


@pytest.mark.parametrize("bitmap", [-1, 32, 64, 0])
@pytest.mark.parametrize("prune", [1, 0])
@pytest.mark.parametrize("split", [(20, 1500), (1, 1), (1 << 30, 1 << 30)])
@pytest.mark.parametrize("touch_scan", [0, 1])
def test_params_do_not_change_result(gm, bitmap, prune, split, touch_scan):
    # touch_scan 1: every counting pass collects its first touches from the
    # global bitmap (the path graphs with |V| above ~114k take).
    ro, co, nU = planted(300, 200, blocks=6, seed=3, bsize=14)
    want = oracle.gmbe(ro, co, nU)
    r = run(gm, ro, co, nU, bitmap_max_l=bitmap, prune=prune, bound_height=split[0],
            bound_size=split[1], touch_scan=touch_scan)
    assert r.status == 0
    assert (r.count, r.set_hash) == (want.count, want.set_hash)


@pytest.mark.parametrize("seed", range(4))
def test_touch_scan_on_hub_graphs(gm, seed):
    # Counts-tier roots (|L| = 300) with every first touch from the global bitmap.
    ro, co, nU = hub_graph(seed)
    want = oracle.gmbe(ro, co, nU)
    for ts in (1, -1):
        r = run(gm, ro, co, nU, touch_scan=ts)
        assert (r.count, r.set_hash) == (want.count, want.set_hash)


@pytest.mark.parametrize("uvtrans,order", [(0, 0), (0, 1), (0, 2), (1, 1), (2, 2), (1, 3)])
def test_side_swap_and_order(gm, uvtrans, order):
    ro, co, nU = planted(200, 150, blocks=4, seed=11)
    want = oracle.brute_force(ro, co, nU) if nU <= 64 else oracle.mbea(ro, co, nU)
    r = run(gm, ro, co, nU, opts=dict(uvtrans=uvtrans, order=order, fast_mode=int(order != 3)))
    assert (r.count, r.set_hash) == (want.count, want.set_hash)


def test_small_config(gm):
    g = gm.config_graph("small")
    want = oracle.gmbe(g.row_off, g.col, g.nU)
    for uvtrans in (0, 1):
        r = run(gm, g.row_off, g.col, g.nU, opts=dict(uvtrans=uvtrans))
        assert (r.count, r.set_hash) == (want.count, want.set_hash)


@pytest.mark.parametrize("seed", range(3))
def test_wide_l_uses_counts_tier(gm, seed):
    # Roots with |L| well above the bitmap limit (128) exercise tier 1 and
    # its hand-off to tier 2, with and without splitting.
    ro, co, nU = hub_graph(seed)
    want = oracle.gmbe(ro, co, nU)
    for uvtrans in (0, 2):
        for bitmap in (-1, 0):
            r = run(gm, ro, co, nU, opts=dict(uvtrans=uvtrans), bitmap_max_l=bitmap,
                    bound_height=1 << 30, bound_size=1 << 30)
            assert (r.count, r.set_hash) == (want.count, want.set_hash)
            r = run(gm, ro, co, nU, opts=dict(uvtrans=uvtrans), bitmap_max_l=bitmap)
            assert (r.count, r.set_hash) == (want.count, want.set_hash)


def test_root_ranges_add_up(gm):
    g = gm.config_graph("small")
    with gm.Graph.from_csr(g.row_off, g.col, g.nU, uvtrans=1) as G:
        nV = G.info().V_size
        cuts = [0, nV // 3, nV // 2, nV]
        tot_c, tot_h = 0, 0
        for a, b in zip(cuts, cuts[1:]):
            r = G.enumerate(root_begin=a, root_end=b)
            o = oracle.gmbe_range(g.row_off, g.col, g.nU, a, b, uvtrans=1)
            assert (r.count, r.set_hash) == (o.count, o.set_hash)
            tot_c += r.count
            tot_h = (tot_h + r.set_hash) % (1 << 64)
        full = G.enumerate()
        assert (full.count, full.set_hash) == (tot_c, tot_h)


def test_tiny_queue_falls_back_inline(gm):
    ro, co, nU = planted(300, 200, blocks=6, seed=9, bsize=14)
    want = oracle.gmbe(ro, co, nU)
    r = run(gm, ro, co, nU, bound_height=1, bound_size=1, queue_capacity=8)
    assert (r.count, r.set_hash) == (want.count, want.set_hash)


def test_repeat_calls_identical(gm):
    g = gm.config_graph("small")
    with gm.Graph.from_csr(g.row_off, g.col, g.nU) as G:
        a = G.enumerate()
        b = G.enumerate(blocks=7)
        c = G.enumerate()
    assert (a.count, a.set_hash) == (b.count, b.set_hash) == (c.count, c.set_hash)


def test_idle_wait_limit_reports_timeout_then_recovers(gm):
    # Many trivial roots, then (input order, roots are taken from the last
    # row backwards) the rows of a dense block: the warps that find no more
    # roots idle while the block is still pending and give up after the
    # (tiny) idle limit.  The call must return MBE_ERR_TIMEOUT, not hang, and
    # the next call on the same graph must be exact.
    rng = np.random.default_rng(0)
    rows = []
    blk = rng.random((22, 22)) < 0.7
    for i in range(22):
        r = np.nonzero(blk[i])[0]
        rows.append(r if len(r) else np.array([0]))
    for i in range(3000):
        rows.append(np.array([22 + i]))
    ro = np.zeros(len(rows) + 1, np.int32)
    ro[1:] = np.cumsum([len(r) for r in rows])
    co = np.concatenate(rows).astype(np.int32)
    nU = int(co.max()) + 1
    want = oracle.gmbe(ro, co, nU)
    with gm.Graph.from_csr(ro, co, nU, order=0) as G:
        with pytest.raises(gm.MBEError) as ei:
            G.enumerate(wait_limit_ns=1, blocks=1, bound_height=1 << 30, bound_size=1 << 30)
        assert ei.value.name == "MBE_ERR_TIMEOUT"
        r = G.enumerate()
        assert (r.count, r.set_hash) == (want.count, want.set_hash)


@pytest.mark.parametrize("shape", [(24, 36, 0.85), (26, 40, 0.88)])
def test_dense_small_graph_is_shared_out(gm, shape):
    # A few dozen vertices at high density hold 10^5 - 10^6 bicliques under a
    # handful of roots: exact results, and the work must be spread over warps
    # (the split test by |P| * |L| alone would keep each root in one warp).
    nV, nU, p = shape
    ro, co, nU = random_bipartite(nV, nU, p, 1)
    want = oracle.gmbe(ro, co, nU)
    with gm.Graph.from_csr(ro, co, nU) as G:
        r = G.enumerate(sm_timing=1)
    assert (r.count, r.set_hash) == (want.count, want.set_hash)
    assert r.n_subproblems > 4 * nV


@pytest.mark.parametrize("root_split", [0, 1, 64, 1 << 20])
def test_root_split_threshold_does_not_change_result(gm, root_split):
    # Heavy roots split into vertex-tuple child tasks (GMBE's own split) while
    # deeper levels share out sub-problems: any threshold gives the same set.
    for ro, co, nU in (planted(300, 200, blocks=6, seed=3, bsize=14), hub_graph(1)):
        want = oracle.gmbe(ro, co, nU)
        r = run(gm, ro, co, nU, root_split_size=root_split)
        assert r.status == 0
        assert (r.count, r.set_hash) == (want.count, want.set_hash)
        if root_split == 1:
            assert r.tasks_split > 0


def test_slot_reuse_across_graphs_is_exact(gm):
    # Small dense graphs keep most warps idle, so nearly every child is shared
    # out and the sub-problem slots are freed and reused constantly, by warps
    # on different SMs and across launches on different graphs.  Alternating
    # graphs back to back, every run must still be exact.
    shapes = [(24, 36, 0.85, 1), (26, 40, 0.8, 2), (30, 30, 0.75, 3), (20, 44, 0.85, 4)]
    graphs = []
    for nV, nU, p, seed in shapes:
        ro, co, nU = random_bipartite(nV, nU, p, seed)
        want = oracle.gmbe(ro, co, nU)
        graphs.append((gm.Graph.from_csr(ro, co, nU), (want.count, want.set_hash)))
    try:
        for rep in range(25):
            for i, (G, want) in enumerate(graphs):
                r = G.enumerate()
                assert (r.count, r.set_hash) == want, f"graph {i} repeat {rep}"
    finally:
        for G, _ in graphs:
            G.free()


@pytest.mark.parametrize("work,chunk", [(1, 2), (1, 64), (1 << 10, 8), (1 << 22, 0), (0, 0)])
def test_root_parts_do_not_change_result(gm, work, chunk):
    # A heavy root split into parts by a hash of the candidate id: each part
    # pushes its own first-level candidates, earlier parts act as Q, later
    # ones stay candidates of the children.  Any split gives the same set.
    cases = [planted(300, 200, blocks=6, seed=3, bsize=14), hub_graph(1),
             random_bipartite(24, 36, 0.85, 1), random_bipartite(120, 90, 0.08, 4)]
    for ro, co, nU in cases:
        want = oracle.gmbe(ro, co, nU)
        for bitmap in (0, -1):  # bitmap tier from set-up, or counts tier only
            r = run(gm, ro, co, nU, range_split_work=work, range_chunk=chunk,
                    bitmap_max_l=bitmap)
            assert r.status == 0
            assert (r.count, r.set_hash) == (want.count, want.set_hash)
            if work == 1 and chunk == 2:
                assert r.tasks_split > 0


@pytest.mark.parametrize("world", [2, 3, 8])
def test_shards_match_oracle_and_add_up(gm, world):
    # The N>1 path: rank r enumerates the roots at positions p = r mod world
    # from the top of the internal order; each share matches the oracle's and
    # the shares sum (mod 2^64) to the whole graph.
    from gmbe_b200.dist import shard_params
    g = gm.config_graph("small")
    with gm.Graph.from_csr(g.row_off, g.col, g.nU, uvtrans=1) as G:
        full = G.enumerate()
        tot_c, tot_h = 0, 0
        for rank in range(world):
            r = G.enumerate(**shard_params(rank, world))
            o = oracle.gmbe_strided(g.row_off, g.col, g.nU, rank, world, uvtrans=1)
            assert (r.count, r.set_hash) == (o.count, o.set_hash)
            tot_c += r.count
            tot_h = (tot_h + r.set_hash) % (1 << 64)
    assert (full.count, full.set_hash) == (tot_c, tot_h)


@pytest.mark.parametrize("slot_records", [8, 64])
@pytest.mark.parametrize("case", ["planted", "hub", "dense"])
def test_large_export_slots(gm, slot_records, case):
    # Shared-out children with more than slot_records candidates go through
    # the 4 MiB slots (on the large graph, children of hundreds of thousands
    # of candidates do); share_min_work 1 shares nearly every child.
    ro, co, nU = {"planted": lambda: planted(300, 200, blocks=6, seed=3, bsize=14),
                  "hub": lambda: hub_graph(3),
                  "dense": lambda: random_bipartite(40, 60, 0.35, 9)}[case]()
    want = oracle.gmbe(ro, co, nU)
    for params in (dict(), dict(bitmap_max_l=64), dict(big_two_hop=64)):
        r = run(gm, ro, co, nU, slot_records=slot_records, share_min_work=1, **params)
        assert r.status == 0
        assert (r.count, r.set_hash) == (want.count, want.set_hash), params


def test_share_counts_switch_and_device_release(gm):
    # Counts-tier children shared out or kept (results equal), and the
    # device's cached workspace handed back between calls.
    ro, co, nU = hub_graph(4)
    want = oracle.gmbe(ro, co, nU)
    with gm.Graph.from_csr(ro, co, nU, uvtrans=1) as G:
        for sc in (0, -1, 0):
            r = G.enumerate(share_counts=sc, share_min_work=1)
            assert (r.count, r.set_hash) == (want.count, want.set_hash)
            gm.release_device(0)
        r = G.enumerate()
        assert (r.count, r.set_hash) == (want.count, want.set_hash)


def test_l2_read_measurement(gm):
    # The benchmark's L2 roofline denominator: reads of an L2-resident buffer
    # run well above HBM speed (B200: HBM ~6.5 TB/s measured by copy).
    gbs = gm.measure_l2_read(0, 32 << 20, 50)
    assert 5000 < gbs < 200000
    with pytest.raises(gm.MBEError):
        gm.measure_l2_read(0, 1 << 10, 50)
