"""The benchmark workloads as seeded generator specs.

The specs live in workloads.json beside this file (one source for this module
and for the stand-alone mbe_gen program, which the timed CPU runs of the
reference's own enumerators use to make the same inputs without loading the
engine).  Each configuration is a Chung-Lu bipartite graph (see
``mbe_gen_chung_lu`` in include/mbe.h) with the shape the workload names.
All of them cap the probability of any single (u, v) pair at 0.1: with hub
weights whose product exceeds the edge count, plain Chung-Lu saturates a
block of hubs to a near-complete bipartite graph, and the few missing edges
of such a block give 2^k maximal bicliques for k hubs (measured: the top
roots of the uncapped medium graph hold 1, 2, 4, ..., 128 bicliques each),
which no enumerator can finish.  The cap keeps every marginal named by the
workload (sizes, edge count, exponents, degree caps as expected-degree caps)
and removes only that saturation.
"""
from __future__ import annotations

import json
import os

from . import GenSpec, batch_spec, generate

WORKLOADS_JSON = os.path.join(os.path.dirname(os.path.abspath(__file__)), "workloads.json")

with open(WORKLOADS_JSON) as _f:
    _W = json.load(_f)

PAIR_P_MAX = 0.1
FIELDS = _W["fields"]


def _spec(nU, nV, nE, gu, gv, mu, mv, seed, n_blocks=0, bu=0, bv=0, bp=0.0):
    return GenSpec(nU=nU, nV=nV, n_edges=nE, gamma_u=gu, gamma_v=gv, max_deg_u=mu,
                   max_deg_v=mv, seed=seed, n_blocks=n_blocks, block_u=bu, block_v=bv,
                   reserved=0, block_p=bp, pair_p_max=PAIR_P_MAX)


def _from_json(d):
    return GenSpec(reserved=0, **d)


# small: 2,000 x 3,000, ~20,000 edges, exponent 2.1 both sides, degree cap 200
# medium skewed: 100,000 x 400,000, ~2,000,000 edges, exponents 2.0 / 2.4,
#   degree cap 5,000, plus 64 planted 24 x 24 blocks at edge probability 0.7
# large: 2,000,000 x 8,000,000, ~60,000,000 edges, exponents 2.1 / 2.2, cap 50,000
# serving mix, medium requests: 20,000 x 80,000, ~300,000 edges, exponent 2.1
CONFIGS = {name: (lambda d=w["spec"]: _from_json(d)) for name, w in _W["workloads"].items()}

# Workload names as the benchmark reports them.
DESCRIPTIONS = {name: w["description"] for name, w in _W["workloads"].items()}


def config_graph(name: str):
    """Generates the named workload graph (host CSR, .adj-shaped)."""
    return generate(CONFIGS[name]())


def batch_graph(seed: int):
    """One graph of the batched workload (seeds 1000..5095)."""
    return generate(batch_spec(seed))


def serve_mix(n: int, seed: int = 7, medium_share: float = 0.05, medium_pool: int = 4):
    """The serving request stream: n graphs, each a medium serving graph
    (20,000 x 80,000, ~300,000 edges, exponent 2.1) with probability
    medium_share, else a graph of the batched distribution (seed 1000 + i).
    The medium requests cycle through medium_pool seeded graphs.  Returns
    (graphs, is_medium)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    med = [generate(_spec(20000, 80000, 300000, 2.1, 2.1, 2000, 2000, seed * 1000 + k))
           for k in range(medium_pool)]
    is_med = rng.random(n) < medium_share
    graphs = [med[i % medium_pool] if is_med[i] else batch_graph(1000 + i) for i in range(n)]
    return graphs, is_med
