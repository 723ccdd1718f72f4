"""Biclique emission (mbe_enumerate_emit): every maximal biclique itself.

Counts and set hashes compare whole sets indirectly; here the emitted sets
are compared directly: with a brute-force closure enumeration on graphs small
enough for it, and elsewhere by count, absence of duplicates and the set hash
recomputed from the records (integers: the tolerance is zero).
"""
import itertools

import numpy as np
import pytest

import oracle
from util import hub_graph, planted, random_bipartite

pytestmark = pytest.mark.gpu
M64 = (1 << 64) - 1


@pytest.fixture(scope="module")
def gm():
    import gmbe_b200
    return gmbe_b200


def fmix64(k):
    k ^= k >> 33
    k = (k * 0xff51afd7ed558ccd) & M64
    k ^= k >> 33
    k = (k * 0xc4ceb9fe1a85ec53) & M64
    k ^= k >> 33
    return k


def set_hash(bicliques):
    # The canonical set hash of include/mbe.h, from (U ids, V ids) pairs.
    total = 0
    for us, vs in bicliques:
        sl = sum(fmix64(2 * u) for u in us) & M64
        sr = sum(fmix64(2 * v + 1) for v in vs) & M64
        rot = ((sr << 29) | (sr >> 35)) & M64
        total = (total + fmix64(sl ^ rot ^ ((len(us) << 32) | len(vs)))) & M64
    return total


def closure_bicliques(ro, co):
    # Every maximal biclique of a tiny graph: close each non-empty set of V rows.
    nV = len(ro) - 1
    rows = [set(int(x) for x in co[ro[v]:ro[v + 1]]) for v in range(nV)]
    found = set()
    for k in range(1, nV + 1):
        for sub in itertools.combinations(range(nV), k):
            us = set.intersection(*(rows[v] for v in sub))
            if not us:
                continue
            vs = tuple(v for v in range(nV) if us <= rows[v])
            found.add((tuple(sorted(us)), vs))
    return found


def emit(gm, ro, co, nU, opts=None, **params):
    with gm.Graph.from_csr(ro, co, nU, **(opts or {})) as G:
        return G.enumerate_emit(**params)


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.parametrize("shape", [(10, 12, 0.4), (12, 9, 0.5), (14, 16, 0.3)])
def test_emitted_set_equals_brute_force(gm, seed, shape):
    nV, nU, p = shape
    ro, co, nU = random_bipartite(nV, nU, p, seed)
    want = closure_bicliques(ro, co)
    for opts in ({"uvtrans": 0, "order": 0}, {"uvtrans": 1, "order": 1}):
        r, got = emit(gm, ro, co, nU, opts)
        assert len(got) == len(set(got)) == r.count
        assert set(got) == want
        assert set_hash(got) == r.set_hash


def test_emitted_records_match_oracle_on_larger_graphs(gm):
    cases = [planted(300, 200, blocks=6, seed=3, bsize=14), hub_graph(1),
             random_bipartite(24, 36, 0.85, 1)]
    for ro, co, nU in cases:
        want = oracle.gmbe(ro, co, nU)
        r, got = emit(gm, ro, co, nU, {"uvtrans": 1}, buf_words=1 << 25)
        assert (r.count, r.set_hash) == (want.count, want.set_hash)
        assert len(got) == len(set(got)) == want.count
        assert set_hash(got) == want.set_hash


def test_emitted_set_does_not_depend_on_parameters(gm):
    ro, co, nU = planted(200, 150, blocks=5, seed=17, bsize=12)
    base = None
    for params in (dict(), dict(bitmap_max_l=-1), dict(prune=0), dict(bound_height=1, bound_size=1),
                   dict(split_mode=1), dict(range_split_work=1, range_chunk=2)):
        r, got = emit(gm, ro, co, nU, {"uvtrans": 1}, **params)
        s = set(got)
        assert len(s) == len(got) == r.count
        if base is None:
            base = s
        assert s == base


def test_emit_buffer_too_small(gm):
    ro, co, nU = planted(200, 150, blocks=5, seed=17, bsize=12)
    with gm.Graph.from_csr(ro, co, nU) as G:
        with pytest.raises(gm.MBEError) as ei:
            G.enumerate_emit(buf_words=64)
        assert ei.value.name == "MBE_ERR_CAPACITY"


@pytest.mark.last
@pytest.mark.parametrize("ring_words", [64, 1000, 4096])
def test_stream_through_a_ring_smaller_than_the_output(gm, ring_words):
    # The kernel writes into a ring the host drains while the launch runs;
    # with 64 words the ring holds a handful of records at a time, so the
    # producers wait on the host again and again.  Every biclique arrives
    # once, and the set equals the buffered emission's and the oracle's.
    ro, co, nU = planted(300, 200, blocks=6, seed=3, bsize=14)
    want = oracle.gmbe(ro, co, nU)
    with gm.Graph.from_csr(ro, co, nU, uvtrans=1) as G:
        got = []
        r = G.enumerate_stream(lambda u, v: got.append((u, v)), ring_words=ring_words)
        rb, buffered = G.enumerate_emit(buf_words=1 << 24)
    assert (r.count, r.set_hash) == (want.count, want.set_hash)
    assert len(got) == len(set(got)) == want.count
    assert set(got) == set(buffered)
    assert set_hash(got) == want.set_hash
    assert sum(2 + len(u) + len(v) for u, v in got) > 4 * ring_words


@pytest.mark.last
def test_stream_stops_delivering_but_counts_exactly(gm):
    ro, co, nU = hub_graph(2)
    want = oracle.gmbe(ro, co, nU)
    with gm.Graph.from_csr(ro, co, nU, uvtrans=1) as G:
        got = []
        r = G.enumerate_stream(lambda u, v: got.append((u, v)) or len(got) >= 10, ring_words=256)
    assert len(got) == 10
    assert (r.count, r.set_hash) == (want.count, want.set_hash)


@pytest.mark.last
def test_stream_with_two_tiers_and_exported_children(gm):
    # Records written by warps running exported children and big-root parts.
    ro, co, nU = planted(300, 200, blocks=6, seed=3, bsize=14)
    want = oracle.gmbe(ro, co, nU)
    with gm.Graph.from_csr(ro, co, nU, uvtrans=1) as G:
        got = []
        r = G.enumerate_stream(lambda u, v: got.append((u, v)), ring_words=512, big_two_hop=64,
                               range_split_work=1, range_chunk=2, share_min_work=1)
    assert (r.count, r.set_hash) == (want.count, want.set_hash)
    assert len(got) == len(set(got)) == want.count and set_hash(got) == want.set_hash
