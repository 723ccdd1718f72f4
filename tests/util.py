"""Small graph helpers shared by the tests."""
import numpy as np


def random_bipartite(nV, nU, p, seed):
    """Dense random bipartite graph, .adj-shaped, every V row non-empty and
    every U id used (so no side has isolated vertices)."""
    rng = np.random.default_rng(seed)
    A = rng.random((nV, nU)) < p
    for v in range(nV):
        if not A[v].any():
            A[v, rng.integers(nU)] = True
    for u in range(nU):
        if not A[:, u].any():
            A[rng.integers(nV), u] = True
    rows = [np.nonzero(A[v])[0].astype(np.int32) for v in range(nV)]
    ro = np.zeros(nV + 1, np.int32)
    ro[1:] = np.cumsum([len(r) for r in rows])
    return ro, np.concatenate(rows).astype(np.int32), nU


def planted(nV, nU, blocks, seed, p_bg=0.02, p_blk=0.8, bsize=12):
    """Sparse background plus dense planted blocks (heavy subtrees)."""
    rng = np.random.default_rng(seed)
    A = rng.random((nV, nU)) < p_bg
    for _ in range(blocks):
        vs = rng.choice(nV, size=min(bsize, nV), replace=False)
        us = rng.choice(nU, size=min(bsize, nU), replace=False)
        A[np.ix_(vs, us)] |= rng.random((len(vs), len(us))) < p_blk
    for v in range(nV):
        if not A[v].any():
            A[v, rng.integers(nU)] = True
    for u in range(nU):
        if not A[:, u].any():
            A[rng.integers(nV), u] = True
    rows = [np.nonzero(A[v])[0].astype(np.int32) for v in range(nV)]
    ro = np.zeros(nV + 1, np.int32)
    ro[1:] = np.cumsum([len(r) for r in rows])
    return ro, np.concatenate(rows).astype(np.int32), nU





def hub_graph(seed, nV=600, nU=1200, hubs=10, hub_deg=300, p_bg=0.004):
    """Sparse background plus a few V rows of degree ~hub_deg (|L| > 128)."""
    rng = np.random.default_rng(seed)
    A = rng.random((nV, nU)) < p_bg
    for h in rng.choice(nV, size=hubs, replace=False):
        A[h, rng.choice(nU, size=hub_deg, replace=False)] = True
    for v in range(nV):
        if not A[v].any():
            A[v, rng.integers(nU)] = True
    for u in range(nU):
        if not A[:, u].any():
            A[rng.integers(nV), u] = True
    rows = [np.nonzero(A[v])[0].astype(np.int32) for v in range(nV)]
    ro = np.zeros(nV + 1, np.int32)
    ro[1:] = np.cumsum([len(r) for r in rows])
    return ro, np.concatenate(rows).astype(np.int32), nU
