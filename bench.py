#!/usr/bin/env python
"""Benchmark: maximal-biclique enumeration of the large workload.

Workload: the large configuration, a 2M x 8M Chung-Lu bipartite graph (~60M
edges, exponents 2.1/2.2, expected-degree cap 50,000, seed 3; synthetic),
with the reference's flags -t 1 -o 1 -f and bounds 20/1500.  The whole graph
holds about 12 billion maximal bicliques, most of them under its few
thousand heaviest roots, far more than one timed step can enumerate.  One
step is one launch over one interleaved root shard: the roots at positions
p = s mod 20000 of the internal degree order (about 100 roots, spread over
the whole order, the heaviest included), for the shards s whose count, set
hash and algorithmic bytes the CPU oracle computed
(tests/golden/large_shards.json).  Steps cycle through those shards.  The
graph is resident in HBM before the timed region; every step's count and set
hash must equal the oracle's.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun: at step i rank r enumerates pinned shard number
i*N + r (mod the number of pinned shards), so the work per GPU is fixed as N
grows (weak scaling), with no data-path collective; value = all ranks'
bicliques / the slowest rank's device time.

Extra legs at N = 1: the medium configuration (whole graph per launch, its
count and hash pinned by the oracle), the 4,096-graph batched workload, the
serving workload, and the CPU baseline.  --impl reference times the
reference's own CPU enumerator (MbeaFinderBitset, built from the reference's
sources into oracle/_ref/) on root samples of the same graph.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

WORKLOAD = "large"
METRIC = "maximal bicliques/s"
UNIT = "bicliques/s"
FLAGS = dict(uvtrans=1, order=1, fast_mode=1)
CONSTS = os.path.join(ROOT, "gmbe_b200", "workload_constants.json")
WORKLOADS = os.path.join(ROOT, "gmbe_b200", "workloads.json")
LARGE_ORACLE = os.path.join(ROOT, "tests", "golden", "large_shards.json")
LARGE_ORACLE_RANGES = os.path.join(ROOT, "tests", "golden", "large_ranges.json")
FALLBACK_HBM_GBS = 6650.0
_T0 = time.time()


def log(msg):
    """Progress on stderr (the JSON line alone goes to stdout)."""
    print(f"[bench {time.time() - _T0:7.1f}s] {msg}", file=sys.stderr, flush=True)


def load_consts(name):
    with open(CONSTS) as f:
        return json.load(f)[name]


def load_json(path):
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(prefix=f"gmbe_clocks{self.index}_", suffix=".csv")
            self.f = os.fdopen(fd, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader",
                 "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        with open(self.path) as f:
            lines = f.readlines()
        os.unlink(self.path)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1].split()[0]))
                smax.append(float(parts[2].split()[0]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


REF_SAMPLER = os.path.join(ROOT, "oracle", "_ref", "ref_mbea")
MBE_GEN = os.path.join(ROOT, "gmbe_b200", "mbe_gen")
# The CPU sample of a step: the roots of the step's pinned shard that lie in
# the lowest CPU_MAX_ROOT of the reference's root order.  The reference's
# MbeaFinderBitset takes seconds to minutes per root above that (all 100
# roots of shard 0: 140 s on 8 host threads, against 1.7 s for the engine),
# so a bounded sample leaves them out; that overstates the CPU rate, the
# higher roots having far fewer bicliques per second.
CPU_MAX_ROOT = 0.9
SHARD_STRIDE = 20000


def write_workload_adj(name, path):
    """Writes a workload's .adj with the stand-alone generator (no engine)."""
    w = load_json(WORKLOADS)
    spec = w["workloads"][name]["spec"]
    out = subprocess.run([MBE_GEN, path] + [str(spec[f]) for f in w["fields"]], check=True,
                         capture_output=True, text=True).stdout.split()
    return int(out[0]), int(out[1])  # generated rows, U ids


def ref_samples(adj, offsets, threads, stride=SHARD_STRIDE, max_root=CPU_MAX_ROOT):
    """The reference's own CPU enumerator (MbeaFinderBitset, src/BicliqueFinder.cu:
    59-197, built from its sources into oracle/_ref/ref_mbea) on root samples of a
    workload: sample j = roots j, j + stride, ... (from the lowest degree up) of
    the lowest max_root of its root order, on `threads` OpenMP threads.  The
    graph is read once (untimed); returns [(bicliques, seconds), ...]."""
    if not os.path.exists(REF_SAMPLER):
        raise FileNotFoundError("oracle/_ref/ref_mbea is not built")
    p = subprocess.run([REF_SAMPLER, adj, "2", "1", "1", str(stride),
                        ",".join(str(j) for j in offsets) + ",", "0", str(threads),
                        str(max_root)], check=True, capture_output=True, text=True)
    out = []
    for line in p.stdout.splitlines():
        f = line.split()
        if f and f[0] == "sample":
            out.append((int(f[5]), float(f[7])))
    if len(out) != len(offsets):
        raise RuntimeError(f"reference sampler printed {len(out)} of {len(offsets)} samples")
    return out


def pinned_offsets(steps, warmup, internal_nv):
    """The reference-order sample offsets of the pinned shards the GPU steps
    enumerate (shard s = internal roots nV-1-s, nV-1-s-20000, ...), warm-up
    steps first, in step order."""
    pins = pinned_shards()
    idx = [len(pins) - 1 - (i % len(pins)) for i in range(warmup)] + \
          [i % len(pins) for i in range(steps)]
    return [(internal_nv - 1 - pins[k]["shard_index"]) % SHARD_STRIDE for k in idx], \
        [pins[k]["shard_index"] for k in idx]


def sample_text(shards):
    return (f"reference MbeaFinderBitset (oracle/_ref, built from the reference's sources) on "
            f"the roots of the pinned shards {','.join(str(s) for s in sorted(set(shards)))} "
            f"(1/{SHARD_STRIDE} of the roots each, the GPU steps' shards) that lie in the lowest "
            f"{CPU_MAX_ROOT:.0%} of the root order (higher roots take seconds to minutes each on "
            f"the CPU: all 100 roots of shard 0 took 140 s on 8 threads); OpenMP over roots; "
            f"graph read excluded")


def cpu_samples(warmup, steps):
    cores = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as d:
        adj = os.path.join(d, f"{WORKLOAD}.adj")
        write_workload_adj(WORKLOAD, adj)
        internal_nv = load_json(LARGE_ORACLE_RANGES)["internal_nV"]
        offs, shards = pinned_offsets(steps, warmup, internal_nv)
        res = ref_samples(adj, offs, cores)[warmup:]
    return res, shards[warmup:], cores


def cpu_baseline_leg(warmup, steps):
    """The same samples the reference arm times at this --steps/--warmup."""
    res, shards, cores = cpu_samples(warmup, steps)
    cnt = sum(c for c, _ in res)
    sec = sum(t for _, t in res)
    return {"value": cnt / sec, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": sample_text(shards) + f": {cnt} bicliques in {sec:.2f} s"}


def run_reference(args):
    """The reference arm: the reference's own CPU enumerator on all host
    cores, timed per step on the CPU sample of the step's shard (warm-up
    steps are untimed samples first).  Loads nothing from the engine: the
    workload's .adj comes from the stand-alone generator.  Rank 0 alone runs."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    res, shards, cores = cpu_samples(args.warmup, args.steps)
    cnt = sum(c for c, _ in res)
    sec = sum(t for _, t in res)
    value = cnt / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * sec / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic", "config": workload_config(args.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": sample_text(shards)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_profile_case():
    """A reduced launch of the enumeration kernel on the large graph for ncu
    captures: 16 blocks over the roots [1000000, 1005000) of the internal
    order (two-hop multisets up to 18,495, so the scratch is a few GB), one
    warm-up and one profiled enumeration, both checked against the oracle's
    count and set hash (tests/golden/large_ranges.json)."""
    import gmbe_b200 as gm
    rg = [r for r in load_json(os.path.join(ROOT, "tests", "golden", "large_ranges.json"))["ranges"]
          if r["root_begin"] == 1000000][0]
    g = gm.config_graph(WORKLOAD)
    with gm.Graph.build_on_device(g.row_off, g.col, g.nU, **FLAGS) as G:
        kw = dict(blocks=16, root_begin=rg["root_begin"], root_end=rg["root_end"])
        rs = [G.enumerate(**kw) for _ in range(2)]
    for r in rs:
        if (r.count, f"{r.set_hash:#018x}") != (rg["count"], rg["set_hash"]):
            raise SystemExit(f"profile case mismatch: {r.count} {r.set_hash:#x}")
    print(json.dumps({"profile_case": "large, 16 blocks, roots [1000000, 1005000)",
                      "count": rs[1].count, "set_hash": f"{rs[1].set_hash:#x}",
                      "kernel_ms": rs[1].kernel_ms}), flush=True)


BATCH_ORACLE = os.path.join(ROOT, "tests", "golden", "batch_oracle.json")


def run_profile_batch(n=512):
    """A reduced batched launch for ncu captures: the first n graphs of the
    batched workload (seeds 1000..1000+n-1) in one launch, captured and
    replayed twice, every per-graph count and set hash checked against the
    oracle's (tests/golden/batch_oracle.json)."""
    import gmbe_b200 as gm
    orc = load_json(BATCH_ORACLE)
    want = list(zip(orc["count"], (int(h, 16) for h in orc["set_hash"])))[:n]
    B = gm.Batch([gm.batch_graph(1000 + i) for i in range(n)])
    runs = [B.run() for _ in range(2)]
    B.free()
    for per, _ in runs:
        if [(r.count, r.set_hash) for r in per] != want:
            raise SystemExit("batch profile case: results differ from the oracle's")
    tot = runs[-1][1]
    print(json.dumps({"profile_case": f"batched, graphs 0..{n - 1}", "bicliques": tot.count,
                      "kernel_ms": tot.kernel_ms}), flush=True)


def batched_leg(n=4096, replays=3):
    """Batched workload: n graphs of the batched distribution (seeds 1000..)
    in one persistent launch replayed from a CUDA graph, against one plain
    launch per graph over all n graphs (graphs resident on the device in
    both arms).  Every per-graph count and set hash of every replay is
    compared with the plain launches and with the CPU oracle's values
    (tests/golden/batch_oracle.json)."""
    import gmbe_b200 as gm
    with open(BATCH_ORACLE) as f:
        orc = json.load(f)
    want = list(zip(orc["count"], (int(h, 16) for h in orc["set_hash"])))[:n]
    log("batched: generating")
    gs = [gm.batch_graph(1000 + i) for i in range(n)]
    log("batched: building")
    B = gm.Batch(gs)
    per, tot = B.run()  # capture + warm-up
    equal_oracle = [(r.count, r.set_hash) for r in per] == want
    walls = []
    for _ in range(replays):
        t = time.perf_counter()
        per, tot = B.run()
        walls.append(time.perf_counter() - t)
        equal_oracle &= [(r.count, r.set_hash) for r in per] == want
    wall = statistics.median(walls)
    B.free()
    log("batched: plain arm")
    Gs = [gm.Graph.from_csr(g.row_off, g.col, g.nU, **FLAGS) for g in gs]
    Gs[0].enumerate()
    t = time.perf_counter()
    plain = [G.enumerate() for G in Gs]
    plain_wall = time.perf_counter() - t
    equal_plain = [(r.count, r.set_hash) for r in plain] == [(r.count, r.set_hash) for r in per]
    for G in Gs:
        G.free()
    return {"graphs": n, "graphs_per_s": n / wall, "replay_ms": wall * 1e3,
            "kernel_ms": tot.kernel_ms, "bicliques": tot.count,
            "plain_graphs_per_s": n / plain_wall,
            "plain_sample": f"all {n} graphs, one mbe_enumerate each",
            "speedup_vs_plain": (n / wall) / (n / plain_wall),
            "results_equal_plain": equal_plain, "results_equal_oracle": equal_oracle}


def serving_leg(n=1000, rates=(100, 200, 300, 1000, 5000, 20000)):
    """Serving: n requests (95 % batched-distribution graphs, 5 % medium
    serving graphs; stream seed 7) submitted at Poisson arrival times for each
    offered load, through mbe_server_*; latency from arrival to result.  The
    plain arm runs each request through mbe_graph_from_csr + mbe_enumerate
    (measured service times) and its latencies are those of a FIFO server at
    the same arrival process."""
    import numpy as np
    import gmbe_b200 as gm
    from gmbe_b200.configs import serve_mix
    log("serving: generating")
    reqs, is_med = serve_mix(n)
    rng = np.random.default_rng(7)
    pct = lambda x, q: float(np.percentile(x, q)) * 1e3
    srv = gm.Server(max_v=32768, max_degree=4096, max_two_hop=1 << 17, arena_bytes=8 << 30,
                    max_graphs=4096)
    log("serving: warm-up")
    for g in reqs[:20]:
        srv.wait(srv.submit(g.row_off, g.col, g.nU), timeout=60)
    loads, outs = {}, []
    arrivals = {}
    for rate in rates:
        log(f"serving: offered load {rate}/s")
        arr = np.cumsum(rng.exponential(1.0 / rate, n))
        arrivals[rate] = arr
        t0 = time.perf_counter()
        sub = []
        for i, g in enumerate(reqs):
            while time.perf_counter() - t0 < arr[i]:
                pass
            sub.append((srv.submit(g.row_off, g.col, g.nU), time.perf_counter() - t0))
        lat, fin, out = [], [], []
        for (rid, ts), a in zip(sub, arr):
            r = srv.wait(rid, timeout=120)
            out.append((r.count, r.set_hash))
            lat.append(ts + r.enum_seconds - a)
            fin.append(ts + r.enum_seconds)
        outs.append(out)
        loads[str(rate)] = {"graphs_per_s": n / max(fin), "p50_ms": pct(lat, 50),
                            "p95_ms": pct(lat, 95), "p99_ms": pct(lat, 99)}
    st = srv.stats()
    srv.close()
    log("serving: plain arm")
    svc, plain = [], []
    for g in reqs:
        t = time.perf_counter()
        with gm.Graph.from_csr(g.row_off, g.col, g.nU, **FLAGS) as G:
            r = G.enumerate()
        svc.append(time.perf_counter() - t)
        plain.append((r.count, r.set_hash))
    for rate in rates:
        fin, lat = 0.0, []
        for a, s in zip(arrivals[rate], svc):
            fin = max(fin, a) + s
            lat.append(fin - a)
        loads[str(rate)]["plain_fifo"] = {"graphs_per_s": n / fin, "p50_ms": pct(lat, 50),
                                          "p95_ms": pct(lat, 95), "p99_ms": pct(lat, 99)}
    plain_gps = n / sum(svc)
    best = max(v["graphs_per_s"] for v in loads.values())
    return {"requests": n, "medium_requests": int(is_med.sum()),
            "mix": "95% batched-distribution graphs, 5% 20k x 80k ~300k-edge graphs; Poisson arrivals, seed 7",
            "loads_per_s": loads, "plain_graphs_per_s": plain_gps,
            "speedup_vs_plain": best / plain_gps, "launches": st["launches"],
            "results_equal_plain": all(o == plain for o in outs)}


SERVING_LIMIT_S = 420


def serving_leg_isolated(limit_s=SERVING_LIMIT_S):
    """serving_leg in a child process (its own CUDA context) under a hard time
    limit: a server that stalls cannot keep this run from printing its line.
    The child's progress goes to stderr as usual; its result is the last line
    of its stdout."""
    cmd = [sys.executable, os.path.abspath(__file__), "--serving-leg"]
    try:
        p = subprocess.run(cmd, stdout=subprocess.PIPE, text=True, timeout=limit_s)
    except subprocess.TimeoutExpired:
        log(f"serving: no result within {limit_s} s; child stopped")
        return {"error": f"serving leg did not finish within {limit_s} s"}
    lines = [x for x in (p.stdout or "").splitlines() if x.strip()]
    if p.returncode != 0 or not lines:
        return {"error": f"serving leg exited with status {p.returncode}"}
    try:
        return json.loads(lines[-1])
    except ValueError:
        return {"error": "serving leg printed no result"}


def workload_config(world):
    w = load_json(WORKLOADS)["workloads"][WORKLOAD]
    pins = pinned_shards()
    return {"workload": w["description"], "flags": "-t 1 -o 1 -f", "bound_height": 20,
            "bound_size": 1500,
            "step": "one launch over one interleaved root shard of the large graph: roots at "
                    "positions p = s mod 20000 of the internal degree order, s cycling through "
                    "the oracle-pinned shards " + ",".join(str(x["shard_index"]) for x in pins),
            "parallelism": f"{world} GPU(s), one shard each per step" if world > 1 else "1 GPU",
            "l2": "inputs (CSR ~0.5 GB, scratch tens of GB) larger than the 126 MB L2"}


def pinned_shards():
    """The oracle's pinned root shards of the large graph, by shard index."""
    d = load_json(LARGE_ORACLE)
    return sorted(d["shards"], key=lambda x: x["shard_index"]) if d else []


def medium_leg(steps=5, warmup=2):
    """The medium configuration, whole graph per launch (the previous
    headline): count and hash pinned by the oracle on every launch."""
    import torch
    import gmbe_b200 as gm
    consts = load_consts("medium")
    g = gm.config_graph("medium")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    with gm.Graph.build_on_device(g.row_off, g.col, g.nU, **FLAGS) as G:
        for _ in range(warmup):
            G.enumerate()
        ms, skew, busy = [], [], []
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            r = G.enumerate(sm_timing=1)
            if (r.count, f"{r.set_hash:#x}") != (consts["count"], consts["set_hash"]):
                raise RuntimeError(f"medium mismatch: {r.count} {r.set_hash:#x}")
            ms.append(r.kernel_ms)
            skew.append(r.sm_exit_max_ms - r.sm_exit_min_ms)
            busy.append(r.warp_busy_frac)
    peak, kind = peaks()
    kern = statistics.mean(ms)
    ach = consts["alg_bytes"] / (kern / 1e3) / 1e9
    # The medium graph's CSR (~24 MB) stays in the 126 MB L2 during a launch,
    # so its roofline is also given against L2 reads, measured here.
    l2 = max(gm.measure_l2_read(0, 32 << 20, 200) for _ in range(3))
    return {"workload": gm.DESCRIPTIONS["medium"], "bicliques_per_launch": consts["count"],
            "value": consts["count"] / (kern / 1e3), "unit": UNIT, "kernel_ms": kern,
            "kernel_ms_all": ms, "sm_last_task_skew_ms": statistics.median(skew),
            "warp_busy_frac": statistics.median(busy), "results_equal_oracle": True,
            "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak, "peak_kind": kind,
                         "algorithmic_bytes_per_launch": consts["alg_bytes"]},
            "roofline_l2": {"bound": "l2", "achieved": ach, "peak": l2, "unit": "GB/s",
                            "frac": ach / l2,
                            "peak_kind": "measured in this run: mbe_measure_l2_read, 32 MiB "
                                         "read 200 times with L1-bypassing loads, best of 3"}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the medium, batched and serving legs (they run at N=1 only)")
    ap.add_argument("--profile", action="store_true",
                    help="one reduced launch for ncu: 16 blocks, roots [1000000, 1005000) of the "
                         "large graph (a few GB)")
    ap.add_argument("--profile-batch", action="store_true",
                    help="one reduced batched launch for ncu: the first 512 graphs of the batch")
    ap.add_argument("--serving-leg", action="store_true",
                    help="run only the serving leg and print its result (used by the N=1 run)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.profile:
        run_profile_case()
        return
    if args.profile_batch:
        run_profile_batch()
        return
    if args.serving_leg:
        print(json.dumps(serving_leg()), flush=True)
        return

    import torch
    import torch.distributed as dist
    import gmbe_b200 as gm

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)
    if args.warmup < 1 or args.steps < 1:
        raise SystemExit("--steps and --warmup must be >= 1")
    pins = pinned_shards()
    if not pins:
        raise SystemExit("no pinned shards (tests/golden/large_shards.json)")

    log("generating the large graph")
    g = gm.config_graph(WORKLOAD)
    G = gm.Graph.build_on_device(g.row_off, g.col, g.nU, device=local, **FLAGS)

    def barrier():
        if world > 1:
            dist.barrier()

    # Step i of rank r takes pinned shard (i * N + r) mod n; warm-ups the
    # same way from the other end of the list.
    def pin_of(step, timed):
        k = step * world + rank
        return pins[k % len(pins)] if timed else pins[len(pins) - 1 - (k % len(pins))]

    mismatched = []

    def enum_pin(Gx, pin, **kw):
        r = Gx.enumerate(shard_count=pin["shard_count"], shard_index=pin["shard_index"], **kw)
        if (r.count, f"{r.set_hash:#018x}") != (pin["count"], pin["set_hash"]):
            mismatched.append(pin["shard_index"])
        return r

    log("warm-up")
    for i in range(args.warmup):
        enum_pin(G, pin_of(i, False))
    clocks = ClockSampler(local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    step_ms, kern_ms, skew, busy, results = [], [], [], [], []
    n_bic, alg = 0, 0
    log("timed steps")
    for i in range(args.steps):
        pin = pin_of(i, True)
        torch.cuda.synchronize()
        barrier()
        ev0.record()
        r = enum_pin(G, pin, sm_timing=1)
        ev1.record()
        torch.cuda.synchronize()
        barrier()
        step_ms.append(ev0.elapsed_time(ev1))
        kern_ms.append(r.kernel_ms)
        skew.append(r.sm_exit_max_ms - r.sm_exit_min_ms)
        busy.append(r.warp_busy_frac)
        n_bic += r.count
        alg += pin["alg_bytes"]
        results.append({"shard": pin["shard_index"], "count": r.count,
                        "set_hash": f"{r.set_hash:#018x}", "kernel_ms": round(r.kernel_ms, 2)})
    clk = clocks.stop()
    tot = torch.tensor([sum(step_ms), sum(kern_ms), float(n_bic), float(alg)],
                       dtype=torch.float64, device=dev)
    if world > 1:
        t_max = tot[:2].clone()
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
        n_all = tot[2:].clone()
        dist.all_reduce(n_all, op=dist.ReduceOp.SUM)
        tot = torch.cat([t_max, n_all])
    total_ms, kern_total, n_all_bic, alg_all = (float(x) for x in tot.tolist())
    value = n_all_bic / (total_ms / 1e3)

    # ---- end to end through the public API with host buffers ----
    # Each call uploads the .adj-shaped CSR, builds the graph on the device
    # (mbe_graph_build_on_device), enumerates the step's shard and reads the
    # result back.
    log("end-to-end calls")
    G.free()
    e2e_steps = max(1, min(args.steps, 3))
    h2d = 4 * ((g.nV + 1) + g.nE)
    iV = min(g.nV, g.nU)
    d2h = 8 + 24 + 4 * iV + 256 + 24
    secs, e2e_n = [], 0
    for i in range(e2e_steps):
        barrier()
        t = time.perf_counter()
        with gm.Graph.build_on_device(g.row_off, g.col, g.nU, device=local, **FLAGS) as G2:
            r = enum_pin(G2, pin_of(i, True))
        secs.append(time.perf_counter() - t)
        e2e_n += r.count
    e2e = torch.tensor([sum(secs), float(e2e_n)], dtype=torch.float64, device=dev)
    if world > 1:
        a = e2e[:1].clone()
        dist.all_reduce(a, op=dist.ReduceOp.MAX)
        b = e2e[1:].clone()
        dist.all_reduce(b, op=dist.ReduceOp.SUM)
        e2e = torch.cat([a, b])
    e2e_secs, e2e_bic = (float(x) for x in e2e.tolist())
    bad = torch.tensor([len(mismatched)], device=dev)
    if world > 1:
        dist.all_reduce(bad)

    if rank == 0:
        peak, peak_kind = peaks()
        kern_mean = kern_total / args.steps
        alg_step = alg_all / args.steps / world
        ach = alg_step / (kern_mean / 1e3) / 1e9
        tpb = (load_json(CONSTS) or {}).get(WORKLOAD, {}).get("traffic_bytes_per_biclique")
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": workload_config(world),
            "bicliques_per_step": n_all_bic / args.steps,
            "enum_ms_per_step": kern_mean,
            "sm_last_task_skew_ms": statistics.median(skew),
            "warp_busy_frac": statistics.median(busy),
            "steps_detail": results,
            "pins": {"fixture": os.path.relpath(LARGE_ORACLE, ROOT), "source": "CPU oracle",
                     "mismatches": int(bad.item())},
            "gpu_launches": args.steps,
            "clocks": clk,
            "e2e": {"value": e2e_bic / e2e_secs, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_steps,
                    "api": "mbe_graph_build_on_device + mbe_enumerate (one shard) from host arrays"},
            "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak, "peak_kind": peak_kind,
                         "traffic": (tpb * n_all_bic / args.steps / world) if tpb else None,
                         "algorithmic_bytes_per_launch": alg_step,
                         "algorithmic_bytes_source": "the oracle's GMBE-tree bytes of each step's "
                                                     "shard (tests/golden/large_shards.json)",
                         "kernel": "mbe_enum_kernel_tiers"},
        }
        # A leg that fails is reported in the line; the measured steps stand.
        if world == 1 and not args.no_extras:
            for name, fn in (("medium", medium_leg), ("batched", batched_leg)):
                log(f"{name} leg")
                try:
                    line[name] = fn()
                except Exception as e:  # noqa: BLE001
                    log(f"{name} leg failed: {e}")
                    line[name] = {"error": f"{type(e).__name__}: {e}"}
            # The serving leg's own process needs the memory this one caches.
            gm.release_device(local)
            torch.cuda.empty_cache()
            line["serving"] = serving_leg_isolated()
        if world == 1 and not args.no_cpu_baseline:
            log("CPU baseline")
            try:
                line["cpu_baseline"] = cpu_baseline_leg(args.warmup, args.steps)
            except Exception as e:  # noqa: BLE001
                log(f"CPU baseline failed: {e}")
                line["cpu_baseline"] = {"error": f"{type(e).__name__}: {e}"}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if int(bad.item()):
        raise SystemExit(f"{int(bad.item())} shard results differ from the pins")


if __name__ == "__main__":
    main()
