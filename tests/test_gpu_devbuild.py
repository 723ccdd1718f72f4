"""Graph build on the device (mbe_graph_build_on_device) against the host build
and the oracle.

The device build orders rows exactly as the host build does (size, then
content, then original id), so both have the same internal ids: root shards
and ranges enumerate the same roots.  The bar is bit-exact equality of count
and set hash with the oracle and the golden fixtures, per shard with the host
build, equal graph summaries, equal emitted sets, and the host build's error
codes on malformed input.
"""
import numpy as np
import pytest

import oracle
from test_cpu import _case_graph, _golden_cases
from util import hub_graph, planted, random_bipartite

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gm():
    import gmbe_b200
    return gmbe_b200


def info_tuple(G):
    i = G.info()
    return (i.U_size, i.V_size, i.edge_size, i.U_degree, i.V_degree, i.U_2degree, i.V_2degree,
            i.swapped)


@pytest.mark.parametrize("name", list(_golden_cases()))
def test_golden_cases(gm, name):
    c = _golden_cases()[name]
    ro, co, nU = _case_graph(gm, name)
    for uvtrans in (0, 1):
        with gm.Graph.build_on_device(ro, co, nU, uvtrans=uvtrans) as G:
            r = G.enumerate()
        assert r.status == 0
        assert r.count == c["oracle_count"]
        assert f"{r.set_hash:#018x}" == c["oracle_set_hash"]


@pytest.mark.parametrize("uvtrans,order", [(0, 0), (0, 1), (0, 2), (1, 1), (2, 2), (1, 3), (2, 0)])
def test_summary_and_result_equal_host_build(gm, uvtrans, order):
    for ro, co, nU in (planted(200, 150, blocks=4, seed=11), hub_graph(2),
                       random_bipartite(50, 30, 0.3, 5)):
        opts = dict(uvtrans=uvtrans, order=order, fast_mode=1)
        with gm.Graph.from_csr(ro, co, nU, **opts) as H, \
                gm.Graph.build_on_device(ro, co, nU, **opts) as D:
            assert info_tuple(D) == info_tuple(H)
            rh, rd = H.enumerate(), D.enumerate()
            assert (rd.count, rd.set_hash) == (rh.count, rh.set_hash)
            # same internal order: every shard holds the same roots
            for si in range(5):
                a = H.enumerate(shard_count=5, shard_index=si)
                b = D.enumerate(shard_count=5, shard_index=si)
                assert (b.count, b.set_hash) == (a.count, a.set_hash), si


def test_equal_degrees_follow_the_host_order(gm):
    # Every row of degree 3 (identical rows included): the order is decided
    # by row content and original id alone, as in the host build.
    rng = np.random.default_rng(4)
    nV, nU = 120, 40
    rows = [np.sort(rng.choice(nU, 3, replace=False)).astype(np.int32) for _ in range(nV)]
    rows[7] = rows[3]
    rows[50] = rows[3]
    ro = np.zeros(nV + 1, np.int32)
    ro[1:] = np.cumsum([3] * nV)
    co = np.concatenate(rows)
    want = oracle.gmbe(ro, co, nU)
    for order in (0, 1, 2):
        with gm.Graph.from_csr(ro, co, nU, uvtrans=0, order=order) as H, \
                gm.Graph.build_on_device(ro, co, nU, uvtrans=0, order=order) as D:
            r = D.enumerate()
            assert (r.count, r.set_hash) == (want.count, want.set_hash)
            for si in range(7):
                a = H.enumerate(shard_count=7, shard_index=si)
                b = D.enumerate(shard_count=7, shard_index=si)
                assert (b.count, b.set_hash) == (a.count, a.set_hash), (order, si)


def test_wide_id_range(gm):
    # U ids spread over 2^21: most U rows of the transpose are empty and the
    # radix sort runs over all 21 key bits.
    rng = np.random.default_rng(9)
    nV, nU = 300, 1 << 21
    pool = np.sort(rng.choice(nU, 400, replace=False)).astype(np.int32)
    rows = [np.sort(rng.choice(pool, rng.integers(1, 12), replace=False)) for _ in range(nV)]
    ro = np.zeros(nV + 1, np.int32)
    ro[1:] = np.cumsum([len(r) for r in rows])
    co = np.concatenate(rows).astype(np.int32)
    want = oracle.gmbe(ro, co, nU)
    for uvtrans in (0, 1):
        with gm.Graph.build_on_device(ro, co, nU, uvtrans=uvtrans) as D:
            r = D.enumerate()
        assert (r.count, r.set_hash) == (want.count, want.set_hash)
    with gm.Graph.build_on_device(ro, co, 0) as D:  # nU = max id + 1
        assert D.info().U_size == int(co.max()) + 1
        r = D.enumerate()
    assert (r.count, r.set_hash) == (want.count, want.set_hash)


def test_params_and_shards_on_device_built_graph(gm):
    ro, co, nU = planted(300, 200, blocks=6, seed=3, bsize=14)
    want = oracle.gmbe(ro, co, nU)
    with gm.Graph.build_on_device(ro, co, nU, uvtrans=1) as D:
        for params in (dict(), dict(bitmap_max_l=-1), dict(prune=0),
                       dict(bound_height=1, bound_size=1), dict(split_mode=1)):
            r = D.enumerate(**params)
            assert (r.count, r.set_hash) == (want.count, want.set_hash)
        total, h = 0, 0
        for si in range(3):
            r = D.enumerate(shard_count=3, shard_index=si)
            total += r.count
            h = (h + r.set_hash) & ((1 << 64) - 1)
        assert (total, h) == (want.count, want.set_hash)


def test_emission_on_device_built_graph(gm):
    for ro, co, nU in (planted(200, 150, blocks=5, seed=17, bsize=12), hub_graph(1)):
        with gm.Graph.from_csr(ro, co, nU, uvtrans=1) as H:
            rh, got_h = H.enumerate_emit(buf_words=1 << 24)
        with gm.Graph.build_on_device(ro, co, nU, uvtrans=1) as D:
            rd, got_d = D.enumerate_emit(buf_words=1 << 24)
        assert (rd.count, rd.set_hash) == (rh.count, rh.set_hash)
        assert len(got_d) == len(set(got_d)) == rd.count
        assert set(got_d) == set(got_h)


def test_without_fast_mode_builds_as_host(gm):
    ro, co, nU = planted(200, 150, blocks=4, seed=11)
    for order in (1, 3):
        opts = dict(uvtrans=1, order=order, fast_mode=0)
        with gm.Graph.from_csr(ro, co, nU, **opts) as H, \
                gm.Graph.build_on_device(ro, co, nU, **opts) as D:
            assert info_tuple(D) == info_tuple(H)
            assert D.info().U_2degree > 0
            rh, rd = H.enumerate(), D.enumerate()
        assert (rd.count, rd.set_hash) == (rh.count, rh.set_hash)


def _bad_inputs():
    ro = np.array([0, 2, 4, 5], np.int32)
    co = np.array([0, 3, 1, 2, 4], np.int32)
    yield "empty row", np.array([0, 2, 2, 5], np.int32), co, 5, "MBE_ERR_FORMAT"
    yield "not ascending", ro, np.array([3, 0, 1, 2, 4], np.int32), 5, "MBE_ERR_FORMAT"
    yield "duplicate id", ro, np.array([0, 0, 1, 2, 4], np.int32), 5, "MBE_ERR_FORMAT"
    yield "id >= nU", ro, co, 4, "MBE_ERR_FORMAT"
    yield "negative id", ro, np.array([-1, 3, 1, 2, 4], np.int32), 5, "MBE_ERR_FORMAT"
    yield "row_off[0] != 0", np.array([1, 2, 4, 5], np.int32), co, 5, "MBE_ERR_FORMAT"
    yield "row_off[nV] != nE", np.array([0, 2, 4, 4], np.int32), co, 5, "MBE_ERR_FORMAT"
    yield "decreasing offsets", np.array([0, 3, 2, 5], np.int32), co, 5, "MBE_ERR_FORMAT"


@pytest.mark.parametrize("case", list(_bad_inputs()), ids=lambda c: c[0])
def test_malformed_input_rejected_like_host_build(gm, case):
    _, ro, co, nU, code = case
    with pytest.raises(gm.MBEError) as eh:
        gm.Graph.from_csr(ro, co, nU, uvtrans=1)
    with pytest.raises(gm.MBEError) as ed:
        gm.Graph.build_on_device(ro, co, nU, uvtrans=1)
    assert eh.value.name == ed.value.name == code
    # The device stays usable after a rejected build.
    ro2, co2, nU2 = random_bipartite(12, 10, 0.4, 0)
    with gm.Graph.build_on_device(ro2, co2, nU2) as D:
        r = D.enumerate()
    want = oracle.brute_force(ro2, co2, nU2)
    assert (r.count, r.set_hash) == (want.count, want.set_hash)


def test_empty_graph_is_invalid_on_device(gm):
    with pytest.raises(gm.MBEError) as ed:
        gm.Graph.build_on_device(np.zeros(1, np.int32), np.zeros(0, np.int32), 0)
    assert ed.value.name == "MBE_ERR_INVALID"
