"""Parity on the large configuration (2M x 8M Chung-Lu, ~60M edges, -t 1 -o 1
-f): root ranges of the internal order against the CPU oracle's results in
tests/golden/large_ranges.json (made by tests/golden/make_large_ranges.py).

The oracle cannot enumerate the whole graph in reasonable time, so the ranges
are ones it finishes in seconds, spread over the degree order.  An explicit
root range sizes its launch from its own roots, so each range runs in one
scratch tier; the grid is held at 32 blocks to keep the scratch near 14 GB.
"""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.last]
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "large_ranges.json")


@pytest.fixture(scope="module")
def gm():
    import gmbe_b200
    return gmbe_b200


def test_large_config_root_ranges_match_oracle(gm):
    with open(GOLDEN) as f:
        d = json.load(f)
    g = gm.config_graph("large")
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(g.row_off, np.int32).tobytes())
    h.update(np.ascontiguousarray(g.col, np.int32).tobytes())
    assert h.hexdigest()[:16] == d["csr_sha256_16"], "generator output changed"
    with gm.Graph.from_csr(g.row_off, g.col, g.nU, uvtrans=1, order=1, fast_mode=1) as G:
        assert G.info().V_size == d["internal_nV"]
        for rg in d["ranges"]:
            r = G.enumerate(root_begin=rg["root_begin"], root_end=rg["root_end"], blocks=32,
                            wait_limit_ns=60 * 10**9)
            assert r.status == 0
            assert (r.count, f"{r.set_hash:#018x}") == (rg["count"], rg["set_hash"]), rg


SHARDS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "large_shards.json")


def test_large_config_root_shards_match_oracle(gm):
    # Interleaved 1/20000 root shards of the large graph (the heaviest roots
    # at the top of the degree order included) against the oracle's count
    # and set hash in tests/golden/large_shards.json
    # (tests/golden/make_large_shards.py).  The whole launch plan runs: two
    # scratch tiers, big-root parts.  The device build orders roots exactly as
    # the host build does, so the same shards hold the same roots.
    with open(SHARDS) as f:
        d = json.load(f)
    g = gm.config_graph("large")
    with gm.Graph.build_on_device(g.row_off, g.col, g.nU, uvtrans=1, order=1) as G:
        for sh in d["shards"]:
            r = G.enumerate(shard_count=sh["shard_count"], shard_index=sh["shard_index"],
                            wait_limit_ns=600 * 10**9, time_limit_ns=900 * 10**9)
            assert r.status == 0
            assert (r.count, f"{r.set_hash:#018x}") == (sh["count"], sh["set_hash"]), sh
