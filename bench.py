#!/usr/bin/env python
"""Benchmark: maximal-biclique enumeration of the medium skewed workload.

One step = one complete enumeration of the medium graph (100k x 400k Chung-Lu,
~2M edges, 64 planted 24x24 blocks; seeded, synthetic) through the engine,
with the reference's flags -t 1 -o 1 -f and bounds 20/1500.  The graph is
resident in HBM before the timed region; every step's count and set hash are
checked against the recorded oracle values.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun: each rank enumerates an interleaved share of the
roots (shard_index = rank) and one NCCL all-reduce sums (count, set hash) per
step; value = the graph's bicliques / the slowest rank's device time.

--impl reference times the CPU restatement of the same path (oracle/, the
GMBE per-root DFS with OpenMP over every host core) on a stratified sample of
the roots, because the reference has no CPU implementation of its GPU path.
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

WORKLOAD = "medium"
METRIC = "maximal bicliques/s"
UNIT = "bicliques/s"
FLAGS = dict(uvtrans=1, order=1, fast_mode=1)
CONSTS = os.path.join(ROOT, "gmbe_b200", "workload_constants.json")
FALLBACK_HBM_GBS = 6650.0
_T0 = time.time()


def log(msg):
    """Progress on stderr (the JSON line alone goes to stdout)."""
    print(f"[bench {time.time() - _T0:7.1f}s] {msg}", file=sys.stderr, flush=True)


def load_consts():
    with open(CONSTS) as f:
        return json.load(f)[WORKLOAD]


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


def cpu_sample(g, target_s=10.0):
    """Oracle (CPU port of the path, all host cores) on a stratified root
    sample sized to ~target_s; returns (bicliques/s, description, cores)."""
    import oracle
    cores = os.cpu_count() or 1
    t = time.perf_counter()
    oracle.gmbe_strided(g.row_off, g.col, g.nU, 1 << 30, 1, threads=cores)  # graph set-up only
    t_setup = time.perf_counter() - t
    stride = 512
    while True:
        t = time.perf_counter()
        r = oracle.gmbe_strided(g.row_off, g.col, g.nU, 0, stride, threads=cores)
        dt = max(time.perf_counter() - t - t_setup, 1e-6)
        if dt >= target_s / 4 or stride == 1:
            break
        stride = max(1, stride // 4)
    return r.count / dt, f"every {stride}th root of the {WORKLOAD} graph from the top of the " \
                         f"degree order: {r.count} bicliques in {dt:.2f} s (graph set-up excluded)", cores


def run_reference(args):
    """The reference arm: CPU restatement of the path on all host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import gmbe_b200 as gm
    import oracle
    g = gm.config_graph(WORKLOAD)
    cores = os.cpu_count() or 1
    t = time.perf_counter()
    oracle.gmbe_strided(g.row_off, g.col, g.nU, 1 << 30, 1, threads=cores)
    t_setup = time.perf_counter() - t
    # Sample size: ~20 s for the whole run.
    stride = 256
    t = time.perf_counter()
    oracle.gmbe_strided(g.row_off, g.col, g.nU, 0, stride, threads=cores)
    per = max(time.perf_counter() - t - t_setup, 1e-3)
    budget = 20.0 / max(1, args.steps + args.warmup)
    while per * 2 < budget and stride > 1:
        stride //= 2
        per *= 2
    for i in range(args.warmup):
        oracle.gmbe_strided(g.row_off, g.col, g.nU, i % stride, stride, threads=cores)
    tot, cnt = 0.0, 0
    for i in range(args.steps):
        t = time.perf_counter()
        r = oracle.gmbe_strided(g.row_off, g.col, g.nU, i % stride, stride, threads=cores)
        tot += max(time.perf_counter() - t - t_setup, 1e-9)
        cnt += r.count
    value = cnt / tot
    sample = (f"per step every {stride}th root of the {WORKLOAD} graph (offsets 0..{args.steps - 1}), "
              f"CPU restatement of the GMBE path, OpenMP over roots; graph set-up excluded")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * tot / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic", "config": {"workload": WORKLOAD_DESC(), "flags": "-t 1 -o 1 -f",
                                        "bound_height": 20, "bound_size": 1500},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_profile_case():
    """A reduced launch of the same kernel for ncu captures: 16 blocks and a
    stratified 1/64 share of the medium graph's roots, one warm-up and one
    profiled enumeration.  Sized so ncu's multi-pass replay stays within a
    few GB of device memory and a minute or two."""
    import gmbe_b200 as gm
    g = gm.config_graph(WORKLOAD)
    with gm.Graph.from_csr(g.row_off, g.col, g.nU, **FLAGS) as G:
        kw = dict(blocks=16, shard_count=64, shard_index=0)
        a = G.enumerate(**kw)
        b = G.enumerate(**kw)
    if (a.count, a.set_hash) != (b.count, b.set_hash):
        raise SystemExit("profile case not reproducible")
    print(json.dumps({"profile_case": "medium, 16 blocks, roots p = 0 mod 64", "count": b.count,
                      "set_hash": f"{b.set_hash:#x}", "kernel_ms": b.kernel_ms}), flush=True)


BATCH_ORACLE = os.path.join(ROOT, "tests", "golden", "batch_oracle.json")


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


def WORKLOAD_DESC():
    import gmbe_b200 as gm
    return gm.DESCRIPTIONS[WORKLOAD]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched and serving legs (they run at N=1 only)")
    ap.add_argument("--profile", action="store_true",
                    help="one reduced launch for ncu: 16 blocks, every 64th root (~1.6 GB scratch)")
    ap.add_argument("--serving-leg", action="store_true",
                    help="run only the serving leg and print its result (used by the N=1 run)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.profile:
        run_profile_case()
        return
    if args.serving_leg:
        print(json.dumps(serving_leg()), flush=True)
        return

    import numpy as np
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
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    consts = load_consts()
    g = gm.config_graph(WORKLOAD)
    G = gm.Graph.from_csr(g.row_off, g.col, g.nU, device=local, **FLAGS)
    from gmbe_b200.dist import shard_params, sum_results
    shard = shard_params(rank, world)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    def barrier():
        if world > 1:
            dist.barrier()

    def reduce_result(r):
        return sum_results(r.count, r.set_hash, device=dev)

    def check(c, h):
        if (c, h) != (consts["count"], int(consts["set_hash"], 16)):
            raise SystemExit(f"result mismatch: count {c} hash {h:#x}, expected "
                             f"{consts['count']} {consts['set_hash']}")

    for _ in range(args.warmup):
        check(*reduce_result(G.enumerate(**shard)))

    clocks = ClockSampler(local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    step_ms, kern_ms, exit_skew, busy = [], [], [], []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        barrier()
        ev0.record()
        r = G.enumerate(sm_timing=1, **shard)
        ev1.record()
        torch.cuda.synchronize()
        barrier()
        step_ms.append(ev0.elapsed_time(ev1))
        kern_ms.append(r.kernel_ms)
        exit_skew.append(r.sm_exit_max_ms - r.sm_exit_min_ms)
        busy.append(r.warp_busy_frac)
        check(*reduce_result(r))
    clk = clocks.stop()
    total_ms = torch.tensor([sum(step_ms)], dtype=torch.float64, device=dev)
    kern_total = torch.tensor([sum(kern_ms)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(total_ms, op=dist.ReduceOp.MAX)
        dist.all_reduce(kern_total, op=dist.ReduceOp.MAX)
    total_ms = float(total_ms.item())
    kern_mean_ms = float(kern_total.item()) / args.steps
    value = consts["count"] * args.steps / (total_ms / 1000.0)

    # ---- end to end through the public API with host buffers ----
    log("timed steps done; end-to-end calls")
    e2e_steps = max(1, min(args.steps, 3))
    # Each call uploads the .adj-shaped CSR once and builds the graph on the
    # device (mbe_graph_build_on_device), then enumerates; it reads back the
    # build's checks (8 B), its capacities (24 B), the internal row order
    # (4 B per internal V vertex), the launch's control block (208 B) and the
    # result (24 B).
    iV = min(g.nV, g.nU) if FLAGS["uvtrans"] == 1 else g.nV
    h2d = 4 * ((g.nV + 1) + g.nE)
    d2h = 8 + 24 + 4 * iV + 208 + 24
    G.free()

    def e2e_leg(build):
        secs = []
        for _ in range(e2e_steps):
            barrier()
            t = time.perf_counter()
            with build(g.row_off, g.col, g.nU, device=local, **FLAGS) as G2:
                r = G2.enumerate(**shard)
            secs.append(time.perf_counter() - t)
            check(*reduce_result(r))
        tot = torch.tensor([sum(secs)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(tot, op=dist.ReduceOp.MAX)
        return consts["count"] * e2e_steps / float(tot.item())

    e2e_value = e2e_leg(gm.Graph.build_on_device)
    # The same call with the graph built on the host (mbe_graph_from_csr),
    # which uploads the CSR, its transpose and the hash keys.
    e2e_host_value = e2e_leg(gm.Graph.from_csr)

    if rank == 0:
        peak, peak_kind = peaks()
        alg = consts["alg_bytes"] / max(world, 1)
        achieved = alg / (kern_mean_ms / 1000.0) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": WORKLOAD_DESC(), "flags": "-t 1 -o 1 -f", "bound_height": 20,
                       "bound_size": 1500, "bicliques_per_step": consts["count"],
                       "parallelism": f"roots interleaved over {world} GPU(s)" if world > 1 else "1 GPU",
                       "l2": "flushed (256 MB write) before every timed step"},
            "enum_ms_per_step": kern_mean_ms,
            "sm_last_task_skew_ms": statistics.median(exit_skew),
            "warp_busy_frac": statistics.median(busy),
            "gpu_launches": args.steps,
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_steps,
                    "api": "mbe_graph_build_on_device + mbe_enumerate",
                    "host_build_value": e2e_host_value},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": consts.get("traffic_bytes_per_launch"),
                         "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": alg,
                         "kernel": "mbe_enum_kernel"},
        }
        # A leg that fails is reported in the line; the measured steps stand.
        if world == 1 and not args.no_extras:
            try:
                line["batched"] = batched_leg()
            except Exception as e:  # noqa: BLE001
                log(f"batched leg failed: {e}")
                line["batched"] = {"error": f"{type(e).__name__}: {e}"}
            line["serving"] = serving_leg_isolated()
        if world == 1 and not args.no_cpu_baseline:
            log("CPU baseline")
            try:
                v, sample, cores = cpu_sample(g)
                line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                                        "sample": sample}
            except Exception as e:  # noqa: BLE001
                log(f"CPU baseline failed: {e}")
                line["cpu_baseline"] = {"error": f"{type(e).__name__}: {e}"}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
