"""Serving (mbe_server_*): continuous batching on one GPU.

Every request's count and set hash must equal the CPU oracle's, whether it
ran alone or in a mix that shared the persistent launch with others (integer
results: the tolerance is zero).  Also: admission limits, arena rewinds,
launches ending when idle and restarting, and the request life cycle.
"""
import threading
import time

import pytest

import oracle
from util import hub_graph, planted, random_bipartite

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gm():
    import gmbe_b200
    return gmbe_b200


def _mix(gm):
    graphs = []
    for i, (nV, nU, p) in enumerate([(30, 40, 0.25), (64, 48, 0.3), (120, 90, 0.08),
                                     (40, 60, 0.15), (200, 150, 0.05)]):
        graphs.append(random_bipartite(nV, nU, p, 100 + i))
    graphs.append(planted(300, 200, blocks=6, seed=3, bsize=14))
    graphs.append(planted(400, 300, blocks=8, seed=5, bsize=12))
    graphs.append(hub_graph(2))
    graphs.append(random_bipartite(24, 36, 0.85, 1))  # dense: ~250k bicliques
    for seed in (1000, 1001, 1007, 1013):
        g = gm.batch_graph(seed)
        graphs.append((g.row_off, g.col, g.nU))
    want = [oracle.gmbe(ro, co, nU) for ro, co, nU in graphs]
    return graphs, [(w.count, w.set_hash) for w in want]


def test_results_same_alone_and_in_the_mix(gm):
    graphs, want = _mix(gm)
    with gm.Server(max_v=8192, max_degree=2048, max_two_hop=1 << 17) as srv:
        # The mix: submitted from two threads at once, collected afterwards.
        ids = [None] * len(graphs)

        def submit(idx):
            for i in idx:
                ro, co, nU = graphs[i]
                ids[i] = srv.submit(ro, co, nU)

        ts = [threading.Thread(target=submit, args=(range(k, len(graphs), 2),)) for k in (0, 1)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        mixed = [srv.wait(rid, timeout=120) for rid in ids]
        # Each alone: submitted only after the previous one finished.
        alone = []
        for ro, co, nU in graphs:
            alone.append(srv.wait(srv.submit(ro, co, nU), timeout=120))
        st = srv.stats()
    for i, w in enumerate(want):
        assert (mixed[i].count, mixed[i].set_hash) == w, f"graph {i} in the mix"
        assert (alone[i].count, alone[i].set_hash) == w, f"graph {i} alone"
        assert mixed[i].enum_seconds > 0
    assert st["completed"] == 2 * len(graphs) and st["resident"] == 0


def test_admission_rejects_graph_beyond_capacity(gm):
    ro, co, nU = random_bipartite(200, 150, 0.05, 7)
    with gm.Server(max_v=64, max_degree=64, max_two_hop=4096) as srv:
        with pytest.raises(gm.MBEError) as ei:
            srv.submit(ro, co, nU)
        assert ei.value.name == "MBE_ERR_ADMISSION"
        small = random_bipartite(30, 40, 0.25, 9)
        w = oracle.gmbe(*small)
        r = srv.wait(srv.submit(*small), timeout=60)
        assert (r.count, r.set_hash) == (w.count, w.set_hash)
        assert srv.stats()["rejected"] == 1


def test_small_arena_rewinds_and_stays_exact(gm):
    graphs = [random_bipartite(40 + 3 * i, 50, 0.2, 200 + i) for i in range(24)]
    want = [oracle.gmbe(*g) for g in graphs]
    # 64 KiB of arena holds a few of these graphs at a time: admission waits
    # until the resident ones finish, the launch ends and the arena rewinds.
    with gm.Server(arena_bytes=64 << 10, max_v=1024, max_degree=1024,
                   max_two_hop=1 << 16) as srv:
        ids = [srv.submit(*g) for g in graphs]
        got = [srv.wait(rid, timeout=120) for rid in ids]
        st = srv.stats()
    for g, w in zip(got, want):
        assert (g.count, g.set_hash) == (w.count, w.set_hash)
    assert st["arena_resets"] >= 1


def test_idle_launch_ends_and_a_new_one_starts(gm):
    a = random_bipartite(64, 48, 0.3, 11)
    b = planted(300, 200, blocks=6, seed=13, bsize=14)
    wa, wb = oracle.gmbe(*a), oracle.gmbe(*b)
    with gm.Server(idle_exit_ns=50_000, max_v=1024, max_degree=1024,
                   max_two_hop=1 << 16) as srv:
        ra = srv.wait(srv.submit(*a), timeout=60)
        time.sleep(0.05)  # far beyond the idle limit: the launch has ended
        rb = srv.wait(srv.submit(*b), timeout=60)
        st = srv.stats()
    assert (ra.count, ra.set_hash) == (wa.count, wa.set_hash)
    assert (rb.count, rb.set_hash) == (wb.count, wb.set_hash)
    assert st["launches"] >= 2


def test_request_life_cycle(gm):
    heavy = random_bipartite(26, 40, 0.8, 2)  # ~400k bicliques: milliseconds on the GPU
    light = random_bipartite(30, 40, 0.25, 3)
    wh = oracle.gmbe(*heavy)
    with gm.Server(max_graphs=1, max_v=1024, max_degree=1024, max_two_hop=1 << 16) as srv:
        rh = srv.submit(*heavy)
        rl = srv.submit(*light)  # waits: one graph at a time
        srv.cancel(rl)
        with pytest.raises(gm.MBEError) as ei:
            srv.poll(rl)
        assert ei.value.name == "MBE_ERR_CANCELLED"
        r = srv.wait(rh, timeout=120)
        assert (r.count, r.set_hash) == (wh.count, wh.set_hash)
        with pytest.raises(gm.MBEError) as ei:
            srv.poll(rh)  # collected already
        assert ei.value.name == "MBE_ERR_NOT_FOUND"
        with pytest.raises(gm.MBEError) as ei:
            srv.cancel(10 ** 9)
        assert ei.value.name == "MBE_ERR_NOT_FOUND"
        assert srv.stats()["cancelled"] == 1


def test_preparation_pool_keeps_submission_order_and_exact_results(gm):
    # Graphs are prepared on the server's own threads (-t/-o build, keys,
    # arena image) after submit returns; admission still follows submission
    # order, and every result equals the oracle's, for one preparation thread
    # and for several.
    graphs, want = _mix(gm)
    for threads in (1, 4):
        with gm.Server(max_v=8192, max_degree=2048, max_two_hop=1 << 17,
                       prep_threads=threads) as srv:
            ids = [srv.submit(ro, co, nU) for ro, co, nU in graphs]
            got = [srv.wait(rid, timeout=120) for rid in ids]
            st = srv.stats()
        for i, w in enumerate(want):
            assert (got[i].count, got[i].set_hash) == w, f"graph {i}, {threads} threads"
        assert st["completed"] == len(graphs) and st["waiting"] == 0


def test_cancel_while_preparing_and_forget_while_held(gm):
    # A request cancelled before its preparation finished never runs; one
    # forgotten (polled after cancel) while a preparation thread still holds
    # it is freed by that thread.  The server stays exact afterwards.
    big = gm.batch_graph(1007)
    small = random_bipartite(30, 40, 0.25, 9)
    w = oracle.gmbe(*small)
    with gm.Server(max_v=8192, max_degree=2048, max_two_hop=1 << 17, prep_threads=1) as srv:
        cancelled = 0
        for _ in range(8):
            rid = srv.submit(big.row_off, big.col, big.nU)
            try:
                srv.cancel(rid)
                cancelled += 1
                with pytest.raises(gm.MBEError) as ei:
                    srv.poll(rid)
                assert ei.value.name == "MBE_ERR_CANCELLED"
            except gm.MBEError as e:  # it reached the GPU first
                assert e.name == "MBE_ERR_INVALID"
                srv.wait(rid, timeout=120)
        r = srv.wait(srv.submit(*small), timeout=60)
        st = srv.stats()
    assert (r.count, r.set_hash) == (w.count, w.set_hash)
    assert cancelled >= 1 and st["cancelled"] == cancelled


def test_server_emission_gives_every_biclique_before_the_result(gm):
    # mbe_server_set_emit: the bicliques of every request, drained from the
    # launch's ring by the server thread, equal mbe_enumerate_emit_stream's
    # for the same graph (as sets; each once), and all of a request's have
    # been delivered when its result comes back.  A ring of 4,096 words is
    # far smaller than the output, so the launch waits for the drain.
    graphs = [random_bipartite(64, 48, 0.3, 11), planted(300, 200, blocks=6, seed=13, bsize=14),
              hub_graph(3), random_bipartite(120, 90, 0.08, 102)]
    for seed in (1000, 1002, 1004, 1007):
        g = gm.batch_graph(seed)
        graphs.append((g.row_off, g.col, g.nU))
    want = []
    for ro, co, nU in graphs:
        got = []
        with gm.Graph.from_csr(ro, co, nU, uvtrans=1, order=1, fast_mode=1) as G:
            r = G.enumerate_stream(lambda u, v: got.append((u, v)) and False)
        want.append((sorted(got), r.count, r.set_hash))
    for ring in (4096, 0):
        with gm.Server(max_v=8192, max_degree=2048, max_two_hop=1 << 17) as srv:
            recs = {}
            seen_at_result = {}
            srv.set_emit(lambda rid, u, v: recs.setdefault(rid, []).append((u, v)),
                         ring_words=ring)
            ids = [srv.submit(ro, co, nU) for ro, co, nU in graphs]
            res = []
            for rid in ids:
                res.append(srv.wait(rid, timeout=120))
                seen_at_result[rid] = len(recs.get(rid, []))
            with pytest.raises(gm.MBEError) as ei:
                srv.set_emit(lambda *a: None)  # only before the first submit
            assert ei.value.name == "MBE_ERR_INVALID"
        for i, rid in enumerate(ids):
            bic, count, h = want[i]
            assert (res[i].count, res[i].set_hash) == (count, h), (ring, i)
            assert seen_at_result[rid] == count, (ring, i)
            assert sorted(recs[rid]) == bic, (ring, i)
