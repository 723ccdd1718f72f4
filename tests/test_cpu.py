"""CPU-only tests: the oracle against the reference's golden results, host
logic (generator, .adj I/O, input validation) and the C-ABI library's
exports.  No compute call here needs a GPU."""
import ctypes
import hashlib
import json
import os
import re
import subprocess

import numpy as np
import pytest

import oracle
from util import planted, random_bipartite

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "golden.json")


@pytest.fixture(scope="module")
def gm():
    import gmbe_b200
    return gmbe_b200


def _digest(ro, co):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(ro, np.int32).tobytes())
    h.update(np.ascontiguousarray(co, np.int32).tobytes())
    return h.hexdigest()[:16]


# ---------------------------------------------------------------------------
# The C ABI library exports every function the headers declare.

def _declared_functions():
    names = []
    hdr = open(os.path.join(ROOT, "include", "mbe.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(mbe_\w+)\s*\(", hdr, flags=re.M):
        names.append(m.group(1))
    return sorted(set(names))


def test_library_exports_every_declared_symbol(gm):
    names = _declared_functions()
    assert len(names) >= 12
    lib = ctypes.CDLL(gm.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_cpp_classes_exported(gm):
    out = subprocess.run(["nm", "-DC", gm.LIB_PATH], capture_output=True, text=True).stdout
    for sym in ("CSRBiGraph::Read", "IterFinderGpu6::Execute", "BicliqueFinder::PrintResult",
                "IterFinderGpu6::IterFinderGpu6"):
        assert sym in out, sym


def test_cli_built(gm):
    assert os.access(gm.CLI_PATH, os.X_OK)


# ---------------------------------------------------------------------------
# Oracle pinned against the reference's own enumerators (golden fixtures).

def _golden_cases():
    with open(GOLDEN) as f:
        return {c["name"]: c for c in json.load(f)["cases"]}


def _case_graph(gm, name):
    if name.startswith("tiny_random_"):
        return random_bipartite(40, 48, 0.25, int(name.rsplit("_", 1)[1]))
    if name == "planted_300x200":
        return planted(300, 200, blocks=6, seed=3, bsize=14)
    if name == "config_small":
        g = gm.config_graph("small")
        return g.row_off, g.col, g.nU
    if name.startswith("batch_"):
        g = gm.batch_graph(int(name.split("_")[1]))
        return g.row_off, g.col, g.nU
    if name == "config_medium":
        g = gm.config_graph("medium")
        return g.row_off, g.col, g.nU
    raise KeyError(name)


@pytest.mark.parametrize("name", [n for n in _golden_cases() if n != "config_medium"])
def test_oracle_matches_reference_golden(gm, name):
    c = _golden_cases()[name]
    ro, co, nU = _case_graph(gm, name)
    assert _digest(ro, co) == c["csr_sha256_16"], "generator output changed"
    o = oracle.gmbe(ro, co, nU)
    for label, ref in c["reference"].items():
        if ref.get("count") is not None:
            assert o.count == ref["count"], label
    assert f"{o.set_hash:#018x}" == c["oracle_set_hash"]
    if "brute_force_set_hash" in c:
        bf = oracle.brute_force(ro, co, nU)
        assert f"{bf.set_hash:#018x}" == c["brute_force_set_hash"] == c["oracle_set_hash"]


@pytest.mark.parametrize("seed", range(8))
def test_three_oracles_agree(seed):
    ro, co, nU = random_bipartite(30 + seed, 24 + 4 * seed, 0.3, seed)
    bf = oracle.brute_force(ro, co, nU)
    mb = oracle.mbea(ro, co, nU)
    for uvtrans, order, prune in ((0, 0, 1), (1, 1, 1), (2, 2, 0), (0, 1, 0)):
        gmr = oracle.gmbe(ro, co, nU, uvtrans=uvtrans, order=order, prune=prune, threads=2)
        assert (gmr.count, gmr.set_hash) == (bf.count, bf.set_hash)
    assert (mb.count, mb.set_hash) == (bf.count, bf.set_hash)


def test_oracle_root_ranges_are_additive():
    ro, co, nU = planted(200, 150, blocks=4, seed=2)
    full = oracle.gmbe(ro, co, nU)
    nV_int = min(len(ro) - 1, nU)  # uvtrans=1: the smaller side holds the roots
    a = oracle.gmbe_range(ro, co, nU, 0, nV_int // 2)
    b = oracle.gmbe_range(ro, co, nU, nV_int // 2, nV_int)
    assert a.count + b.count == full.count
    assert (a.set_hash + b.set_hash) % (1 << 64) == full.set_hash


def test_hash_detects_a_planted_mistake():
    # Dropping one edge changes the set of maximal bicliques, and the hash
    # must see it even when the count happens to stay the same.
    ro, co, nU = random_bipartite(20, 20, 0.4, 1)
    base = oracle.brute_force(ro, co, nU)
    co2 = co.copy()
    row = 3
    keep = np.ones(len(co2), bool)
    keep[ro[row]] = False
    if ro[row + 1] - ro[row] == 1:
        pytest.skip("row has one edge")
    ro2 = ro.copy()
    ro2[row + 1:] -= 1
    mut = oracle.brute_force(ro2, co2[keep], nU)
    assert mut.set_hash != base.set_hash


# ---------------------------------------------------------------------------
# Host logic: generator, .adj I/O, validation.

def test_generator_is_deterministic_and_clean(gm):
    a = gm.config_graph("small")
    b = gm.config_graph("small")
    assert np.array_equal(a.row_off, b.row_off) and np.array_equal(a.col, b.col)
    deg = np.diff(a.row_off)
    assert deg.min() >= 1  # no empty .adj line
    assert deg.max() <= 400
    for v in range(a.nV):
        r = a.col[a.row_off[v]:a.row_off[v + 1]]
        assert np.all(np.diff(r) > 0)
    assert np.array_equal(np.unique(a.col), np.arange(a.nU))  # dense U ids
    assert abs(a.nE - 20000) < 1000


def test_batch_spec_ranges(gm):
    for s in range(1000, 1040):
        sp = gm.batch_spec(s)
        assert 50 <= sp.nU <= 5000
        assert 0.5 * sp.nU - 1 <= sp.nV <= 4 * sp.nU + 1
        assert 3 * sp.nU - 1 <= sp.n_edges <= 30 * sp.nU + 1
        assert sp.gamma_u == sp.gamma_v == 2.2


def test_adj_roundtrip(gm, tmp_path):
    g = gm.config_graph("small")
    p = str(tmp_path / "g.adj")
    gm.write_adj(p, g)
    h = gm.read_adj(p)
    assert np.array_equal(g.row_off, h.row_off) and np.array_equal(g.col, h.col)
    assert h.nU == g.nU
    lines = open(p).read().split("\n")
    assert lines[-1] == "" and all(lines[:-1])


@pytest.mark.parametrize("text,code", [
    ("1 2 3\n3 2\n", "MBE_ERR_FORMAT"),      # row not ascending
    ("1 2 3\n\n4\n", "MBE_ERR_FORMAT"),      # empty row
    ("1 1\n", "MBE_ERR_FORMAT"),             # duplicate id
    ("1 2 x\n", "MBE_ERR_FORMAT"),           # bad token
    ("1 99999999999\n", "MBE_ERR_FORMAT"),   # id >= 2^31
])
def test_adj_rejects_bad_input(gm, tmp_path, text, code):
    p = tmp_path / "bad.adj"
    p.write_text(text)
    with pytest.raises(gm.MBEError) as ei:
        gm.Graph.from_adj(str(p))
    assert ei.value.name == code


def test_missing_file_is_io_error(gm, tmp_path):
    with pytest.raises(gm.MBEError) as ei:
        gm.Graph.from_adj(str(tmp_path / "nope.adj"))
    assert ei.value.name == "MBE_ERR_IO"


def test_truncated_file_reads_partial_last_line(gm, tmp_path):
    p = tmp_path / "t.adj"
    p.write_text("0 1\n1 2")  # no trailing newline: still two rows
    g = gm.read_adj(str(p))
    assert g.nV == 2 and g.nE == 4


def test_csr_validation_runs_before_any_device_call(gm):
    ro = np.array([0, 2, 2], np.int32)  # second row empty
    co = np.array([0, 1], np.int32)
    with pytest.raises(gm.MBEError) as ei:
        gm.Graph.from_csr(ro, co, 2)
    assert ei.value.name == "MBE_ERR_FORMAT"


@pytest.mark.parametrize("ro,code", [
    ([0, 2, 2, 3], "MBE_ERR_FORMAT"),   # empty row
    ([1, 2, 3, 3], "MBE_ERR_FORMAT"),   # row_off[0] != 0
    ([0, 2, 3, 4], "MBE_ERR_FORMAT"),   # row_off[nV] != nE
    ([0, 3, 2, 3], "MBE_ERR_FORMAT"),   # decreasing offsets
    ([0], "MBE_ERR_INVALID"),           # no rows
])
def test_device_build_checks_offsets_before_any_device_call(gm, ro, code):
    # mbe_graph_build_on_device reads through the row offsets only after the
    # host has checked them; malformed offsets never reach a kernel.
    co = np.array([0, 1, 2], np.int32)
    with pytest.raises(gm.MBEError) as ei:
        gm.Graph.build_on_device(np.array(ro, np.int32), co, 3)
    assert ei.value.name == code


def test_bench_serving_leg_reports_instead_of_hanging():
    # The serving leg runs in a child process under a hard limit: a child that
    # outlives the limit, or fails, becomes an error entry of the bench line.
    import bench
    out = bench.serving_leg_isolated(limit_s=1)
    assert out == {"error": "serving leg did not finish within 1 s"}
    import torch
    if not torch.cuda.is_available():
        out = bench.serving_leg_isolated(limit_s=300)
        assert set(out) == {"error"} and "exited with status" in out["error"]


def test_params_defaults(gm):
    p = gm.default_params()
    assert (p.bound_height, p.bound_size, p.prune) == (20, 1500, 1)


def test_ctypes_mirrors_match_the_c_header(gm, tmp_path):
    # The Python binding mirrors the C structs field by field; a field added
    # on one side only would make the library write past the caller's struct.
    # gcc compiles a probe against include/mbe.h that prints each struct's
    # size and every field's offset.
    mirrors = {"mbe_opts": gm.Opts, "mbe_graph_info": gm.GraphInfo, "mbe_params": gm.Params,
               "mbe_result": gm.Result, "mbe_gen_spec": gm.GenSpec,
               "mbe_server_config": gm.ServerConfig, "mbe_server_stats": gm.ServerStats}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "mbe.h"', 'int main(void) {']
    for cname, py in mirrors.items():
        lines.append(f'  printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'  printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines += ['  return 0;', '}']
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    subprocess.run(["gcc", "-I", inc, "-o", str(exe), str(src)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], check=True, capture_output=True,
                                                 text=True).stdout.splitlines())
    for cname, py in mirrors.items():
        assert int(got[cname]) == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(got[f"{cname}.{f}"]) == getattr(py, f).offset, f"{cname}.{f}"


def test_server_needs_a_device(gm):
    # Without a usable GPU the server reports a CUDA error instead of crashing.
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(gm.MBEError) as ei:
        gm.Server()
    assert ei.value.name == "MBE_ERR_CUDA"


def test_new_entry_points_check_arguments_before_any_device_call(gm):
    # mbe_measure_l2_read refuses sizes outside 1-96 MiB and passes outside
    # 1-1000; mbe_server_set_emit refuses a null server or callback.  Both
    # before touching a device.
    for nbytes, passes in ((1 << 10, 10), (1 << 30, 10), (32 << 20, 0), (32 << 20, 5000)):
        with pytest.raises(gm.MBEError) as ei:
            gm.measure_l2_read(0, nbytes, passes)
        assert ei.value.name == "MBE_ERR_INVALID"
    import ctypes as C
    lib = C.CDLL(gm.LIB_PATH)
    lib.mbe_server_set_emit.restype = C.c_int
    lib.mbe_server_set_emit.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    assert lib.mbe_server_set_emit(None, 0, None, None) == -1  # MBE_ERR_INVALID


def test_large_shard_pins_agree_with_the_reference():
    # tests/golden/pin_large_shards_reference.py ran the reference's own
    # MbeaFinderBitset on every root of the pinned large-graph shards; its
    # counts must equal the oracle's (the reference reports counts only).
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "large_shards.json")) as f:
        d = json.load(f)
    pinned = [sh for sh in d["shards"] if "reference_count" in sh]
    assert pinned, "no shard carries the reference's count"
    for sh in pinned:
        assert sh["reference_count"] == sh["count"], sh["shard_index"]


def test_batch_fixture_agrees_with_the_reference():
    # tests/golden/pin_batch_reference.py ran the reference's own
    # MbeaFinderBitset on all 4,096 graphs of the batched workload; every
    # count must equal the oracle's.
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "batch_oracle.json")) as f:
        d = json.load(f)
    assert len(d["reference_count"]) == d["n"] == len(d["count"])
    assert d["reference_count"] == d["count"]


def test_graph_writer_matches_reference_converter(gm, tmp_path):
    # The edge-pair .graph file the CPU peers read.  Where the reference's own
    # converter (preprocess/adj_to_graph.cpp) is built into oracle/_ref, both
    # files must be identical byte for byte; otherwise the format is checked.
    ro, co, nU = planted(60, 40, blocks=2, seed=21)
    g = gm.BipartiteCSR(ro, co, nU)
    adj, ours = tmp_path / "g.adj", tmp_path / "ours.graph"
    gm.write_adj(str(adj), g)
    gm.write_graph(str(ours), g)
    lines = ours.read_text().splitlines()
    assert lines[0] == f"{g.nV} {int(co.max()) + 1}"
    pairs = [tuple(map(int, l.split())) for l in lines[1:]]
    want = [(v, int(u)) for v in range(g.nV) for u in co[ro[v]:ro[v + 1]]]
    assert pairs == want
    conv = oracle.ref_binary("adj_to_graph")
    if conv:
        theirs = tmp_path / "theirs.graph"
        subprocess.run([conv, str(adj), str(theirs)], check=True, capture_output=True)
        assert ours.read_bytes() == theirs.read_bytes()


def _shard_rank(rank, world, port, graph, out):
    # One rank of the N>1 path, the CPU oracle standing in for its GPU: its
    # share of the roots (the strided positions mbe_params shard_* selects),
    # then the same reduction bench.py uses.
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from gmbe_b200.dist import shard_params, sum_results
        ro, co, nU = graph
        p = shard_params(rank, world)
        r = oracle.gmbe_strided(ro, co, nU, p["shard_index"], p["shard_count"], threads=1)
        out[rank] = sum_results(r.count, r.set_hash)
    finally:
        dist.destroy_process_group()


def test_sharded_ranks_sum_to_the_whole_graph():
    import socket
    import torch.multiprocessing as mp
    graph = planted(300, 200, blocks=6, seed=3, bsize=14)
    want = oracle.gmbe(*graph)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_shard_rank, args=(r, 2, port, graph, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == out[1] == (want.count, want.set_hash)
    # each share alone is a strict part of the whole
    half = oracle.gmbe_strided(*graph, 0, 2)
    assert 0 < half.count < want.count


def test_batch_oracle_fixture_reproduces(gm):
    # tests/golden/batch_oracle.json (all 4,096 batched graphs) agrees with
    # the reference-pinned golden cases for seeds 1000..1002 and with the
    # oracle rerun on a spread of its graphs.
    with open(os.path.join(ROOT, "tests", "golden", "batch_oracle.json")) as f:
        d = json.load(f)
    assert d["n"] == len(d["count"]) == len(d["set_hash"]) == 4096
    assert sum(d["count"]) == d["total_count"]
    gold = _golden_cases()
    for i in range(3):
        c = gold[f"batch_{1000 + i}"]
        assert (d["count"][i], d["set_hash"][i]) == (c["oracle_count"], c["oracle_set_hash"])
    for i in (5, 777, 2048, 4095):
        g = gm.batch_graph(d["first_seed"] + i)
        o = oracle.gmbe(g.row_off, g.col, g.nU, uvtrans=1, order=1)
        assert (o.count, f"{o.set_hash:#018x}") == (d["count"][i], d["set_hash"][i])


@pytest.fixture(scope="module")
def large_graph(gm):
    return gm.config_graph("large")


def test_large_range_fixture_reproduces(gm, large_graph):
    # The large configuration's parity fixtures (tests/golden/large_ranges.json)
    # come from the oracle on this generator's graph: regenerate it and the
    # cheapest range.
    with open(os.path.join(ROOT, "tests", "golden", "large_ranges.json")) as f:
        d = json.load(f)
    g = large_graph
    assert _digest(g.row_off, g.col) == d["csr_sha256_16"]
    rg = d["ranges"][0]
    o = oracle.gmbe_range(g.row_off, g.col, g.nU, rg["root_begin"], rg["root_end"], uvtrans=1)
    assert (o.count, f"{o.set_hash:#018x}") == (rg["count"], rg["set_hash"])


# ---------------------------------------------------------------------------
# Scratch-tier plan (gmbe::choose_tiers, through a probe linked to the
# library; host arithmetic only).

MBE_ERR_NOMEM, MBE_ERR_CAPACITY = -5, -8


@pytest.fixture(scope="module")
def tiers(gm, tmp_path_factory):
    d = tmp_path_factory.mktemp("tiers")
    exe = d / "tiers_probe"
    libdir = os.path.dirname(gm.LIB_PATH)
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "gmbe_b200", "csrc"),
                    "-o", str(exe), os.path.join(ROOT, "tests", "probes", "tiers_probe.cpp"),
                    "-L", libdir, "-lgmbe", f"-Wl,-rpath,{libdir}"], check=True)

    def run(nV, S, D, roots, warps=2368, budget=1 << 50, force_bound=0, force_big=0):
        S, D, roots = (np.asarray(S, np.int64), np.asarray(D, np.int32),
                       np.asarray(roots, np.int32))
        req = d / "req.bin"
        with open(req, "wb") as f:
            f.write(np.array([nV, len(S), warps, force_big], np.int32).tobytes())
            f.write(np.array([budget], np.uint64).tobytes())
            f.write(np.array([force_bound], np.int64).tobytes())
            f.write(S.tobytes() + D.tobytes() + roots.tobytes())
        out = subprocess.run([str(exe), str(req)], check=True, capture_output=True,
                             text=True).stdout
        r = {}
        for line in out.splitlines():
            k, *v = line.split()
            r[k] = [int(x) for x in v] if len(v) > 1 else int(v[0])
        return r
    return run


def _roots(seed, n=500):
    rng = np.random.default_rng(seed)
    S = rng.integers(1, 20000, n)
    D = np.minimum(S, rng.integers(1, 300, n))
    return S, D, np.arange(n)[::-1]  # claim order: the top of the order first


def test_tiers_one_tier_when_it_fits(tiers):
    r = tiers(1000, [10, 50, 200], [2, 5, 9], [2, 1, 0])
    assert (r["rc"], r["n_big"], r["list"]) == (0, 0, 0)
    assert r["small"] == r["big"] == [200, 9, 200]  # |C| <= min(|V|, two-hop)


def test_tiers_forced_bound_lists_the_roots_above_it(tiers):
    S, D, roots = _roots(1)
    r = tiers(600, S, D, roots, force_bound=5000)
    above = S > 5000
    assert r["rc"] == 0 and r["mismatch"] == 0
    assert r["list"] == r["flagged"] == above.sum()
    assert r["first"] == roots[np.argmax(above)]
    assert r["last"] == roots[len(S) - 1 - np.argmax(above[::-1])]
    assert r["n_big"] == min(above.sum(), 2368 // 2) and r["bound"] == 5000
    assert r["big"] == [min(600, S.max()), D.max(), S.max()]
    # the small tier: the bound, the degrees below it, and room for any
    # exported sub-problem of a big warp (8,064 records)
    assert r["small"] == [max(min(min(600, S.max()), 8064), min(600, 5000)), D[~above].max(), 5000]


def test_tiers_forced_pool_and_bound_above_every_root(tiers):
    S, D, roots = _roots(2)
    assert tiers(600, S, D, roots, force_bound=1000, force_big=3)["n_big"] == 3
    r = tiers(600, S, D, roots, force_bound=int(S.max()))
    assert (r["rc"], r["n_big"], r["list"], r["flagged"]) == (0, 0, 0, 0)


def test_tiers_report_what_does_not_fit(tiers):
    S, D, roots = _roots(3)
    assert tiers(600, S, D, roots, budget=4096, force_bound=1000)["rc"] == MBE_ERR_NOMEM
    big = tiers(600, S, D, roots, force_bound=1000)
    # room for the small tier and less than one big warp more
    budget = big["small_bytes"] * 2368 + (big["big_bytes"] - big["small_bytes"]) // 2
    assert tiers(600, S, D, roots, budget=budget, force_bound=1000)["rc"] == MBE_ERR_NOMEM
    assert tiers(600, [1 << 31], [5], [0])["rc"] == MBE_ERR_CAPACITY
    # Every root below the smallest two-hop bound, yet one layout for every
    # warp (the count map over 10^7 vertices is 40 MB a warp) is above the
    # budget: a second tier cannot help, and the plan says so.
    r = tiers(10**7, [900, 1000], [3, 4], [1, 0], budget=10 * 10**9)
    assert (r["rc"], r["n_big"], r["list"]) == (MBE_ERR_NOMEM, 0, 0)


def test_tiers_plan_of_the_large_configuration(tiers, large_graph):
    # The whole large graph on 148 x 16 warps with 185 GB for scratch: one
    # layout for the worst root does not fit, so two tiers are planned.
    sys_path = os.path.join(ROOT, "tests", "golden")
    import sys
    if sys_path not in sys.path:
        sys.path.insert(0, sys_path)
    from make_large_ranges import internal_two_hop
    g = large_graph
    S, D, n = internal_two_hop(g.row_off, g.col, g.nU, degrees=True)
    roots = np.arange(n)[::-1]
    warps, budget = 148 * 16, 185 * 10**9
    r = tiers(n, S[roots], D[roots], roots, warps=warps, budget=budget)
    assert r["rc"] == 0 and r["mismatch"] == 0 and r["n_big"] >= 1
    T = r["bound"]
    assert T >= 1 << 16 and T & (T - 1) == 0
    assert r["small_bytes"] * warps <= budget * 6 // 10
    assert r["list"] == (S > T).sum() == r["flagged"]
    fit = (budget - r["small_bytes"] * warps) // (r["big_bytes"] - r["small_bytes"])
    assert r["n_big"] == min(r["list"], fit, warps // 2)
    total = r["small_bytes"] * (warps - r["n_big"]) + r["big_bytes"] * r["n_big"]
    assert total <= budget
    print(f"large plan: bound {T}, {r['list']} listed roots, {r['n_big']} big warps, "
          f"small {r['small_bytes'] / 1e6:.1f} MB, big {r['big_bytes'] / 1e9:.3f} GB, "
          f"total {total / 1e9:.1f} GB")
