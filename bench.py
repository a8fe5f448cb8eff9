#!/usr/bin/env python3
"""Benchmark of the tabu-search hot path on one B200 (per rank).

Workload (default): plain Max Bisection tabu search on the seeded
conflict-style graph -- n = 100,000 unit-square points joined within a radius
for mean degree ~60 plus 2,000 cliques of 8-32 vertices, node weights
U[1,1000], w(u,v) = nw_u + nw_v -- from a seeded balanced random partition,
tenure 50, Piter 500, gamma 150, with all six lookup structures side by side.
Every iteration evaluates all floor(n/2)*ceil(n/2) = 2.5e9 swap pairs.

One STEP = one tabu iteration (all-pairs sweep + argmax + move) on each of the
six structures.  Each iteration is timed on the device with CUDA events on the
library's stream; a 256 MiB buffer is written between timed iterations so no
iteration starts with a warm L2.  `value` is swap-gains/s of the whole job
(pairs evaluated / device time); `e2e` runs the same solves through the C-ABI
from pinned host edge lists (graph upload and build, start, iterations, result
read back) under a wall clock.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "graph-data-structures-local-search_b200")
sys.path.insert(0, PKG)
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "tabu iters/s & swap-gains/s (frac HBM roof); batched solves/s + p50/p99 vs plain"
UNIT = "swap-gains/s"
WORKLOAD = ("config2: plain Max Bisection tabu search, conflict-style graph n=100000 "
            "(radius for mean degree ~60 + 2000 cliques of 8-32), tenure 50, Piter 500, gamma 150, "
            "six lookup structures")


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx = float(r[1])
                for k, nm in enumerate(names):
                    if r[4 + k].lower().startswith("active"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


WORKLOADS = {
    "config2": ("maxbs", WORKLOAD),
    "config3": ("mdp", "config3: plain MDP, Chung-Lu n=200000 (exponent 2.3, mean degree 50, max 5000), "
                       "m=2000, tenure 100"),
    "config1": ("mdp", "config1: plain MDP, Erdos-Renyi n=2000 mean degree 20, m=200, tenure 20"),
    "config5": ("mixed", "config5: served"),
}


def build_workload(name: str = "config2", n: int = 0):
    from ts_b200 import gen
    wl = getattr(gen, name)(n) if n else getattr(gen, name)()
    wl["problem"], wl["desc"] = WORKLOADS[name]
    return wl


def algorithmic_bytes(kind: str, n: int, m: int, ldc: int, key_bytes: int, deg_in: np.ndarray,
                      cap_in: np.ndarray, wpr: int, w_bytes: int = 4) -> int:
    """Compulsory HBM bytes of one iteration of `kind`: the row and column
    state every structure reads (contributions, tabu stamps, vertex ids) plus
    what its lookups must touch once -- the inside rows' CSR entries, hash
    tables or bitmap rows, or the whole WSwap matrix."""
    delta = n - m
    base = m * (key_bytes + 8) + delta * (key_bytes + 4)  # row side: vg, tabu, id; columns: vg, tabu
    if kind == "csr":
        return base + 16 * m + 12 * int(deg_in.sum())  # rowptr pairs, (col, w) + pos per entry
    if kind == "csr-bb":
        return base + 4 * delta + 16 * m + 8 * int(deg_in.sum())
    if kind == "hash":
        return base + 4 * delta + 16 * m + 8 * int(cap_in.sum())
    if kind in ("csr-bitset", "csr-bitset-bb"):
        return base + 4 * delta + 8 * m * wpr
    if kind == "wswap":
        return base + w_bytes * m * ldc
    raise ValueError(kind)


def profile_entry(workload: str, kind: str, grid: int):
    """Counters of one launch of this structure's iteration kernel on this
    workload, from an ncu capture (profiles/dram_traffic.json: DRAM bytes,
    warp instructions, L2 hit rate, active threads per warp instruction).  An
    entry records the grid it was captured with; one captured with another
    grid (another tile shape) is not this kernel's, so it gives None."""
    p = os.path.join(ROOT, "profiles", "dram_traffic.json")
    try:
        with open(p) as f:
            d = json.load(f)
        v = d.get(workload, {}).get(kind)
        if not isinstance(v, dict) or int(v.get("grid", -1)) != int(grid):
            return None
        return v
    except Exception:
        return None


def issue_fraction(warp_inst: float, seconds: float, sm_mhz: float) -> float:
    """Warp instructions issued per second over the issue peak: 148 SMs x 4
    schedulers x one warp instruction per clock."""
    return warp_inst / seconds / (148 * 4 * sm_mhz * 1e6)


def oracle_iterations(wl, problem, m, warm: int, k: int, threads: int, tenure: int):
    """Seconds the oracle (the reference loop restated, int64) takes for k
    whole tabu iterations (sweep + ArgMax + move) after `warm` iterations from
    the seeded start: runs of warm and warm + k iterations, differenced, so
    the start state's cost cancels."""
    from oracle import oracle as O
    op = O.MDP if problem == 0 else O.MAXBS
    g = O.Graph(wl["n"], wl["u"], wl["v"], wl["w"], drop_self_loops=problem == 0)
    kw = dict(m=m if problem == 0 else 0, tenure_policy=O.TENURE_FIXED, tenure=tenure, piter=500, gamma=150,
              seed=1, threads=threads)
    t0 = time.time()
    O.run(g, op, max_iter=warm, **kw)
    t_w = time.time() - t0
    t0 = time.time()
    r = O.run(g, op, max_iter=warm + k, **kw)
    t_wk = time.time() - t0
    assert r.iterations == warm + k
    return max(t_wk - t_w, 1e-9)


def cpu_baseline_sample(wl, problem, m, iters: int = 12):
    """The oracle on all host cores: whole iterations of the same solve."""
    from oracle import oracle as O
    threads = O.max_threads()
    n = wl["n"]
    P = m * (n - m)
    dt = oracle_iterations(wl, problem, m, 2, iters, threads, wl["tenure"])
    return {"value": P * iters / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"oracle (OpenMP over row blocks): tabu iterations 3-{2 + iters} of the seeded solve, "
                      f"{P:.3g} pairs each ({dt:.1f} s)"}


def run_reference(args):
    """--impl reference: the reference loop restated on the host cores (the
    reference has no CPU implementation and its CUDA build cannot index this
    instance's 2.5e9 pairs in int32): each step one whole tabu iteration
    (all-pairs sweep, ArgMax, move) of the default workload's seeded solve,
    after `warmup` iterations, with all host threads."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import oracle as O
    wl = build_workload()
    n = wl["n"]
    m = n // 2
    P = m * (n - m)
    threads = O.max_threads()
    dt = oracle_iterations(wl, 1, m, args.warmup, args.steps, threads, wl["tenure"])
    value = P * args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic (seeded conflict-style graph)",
        "config": {"workload": WORKLOAD, "n": n, "m": m, "pairs_per_iter": P},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"tabu iterations {args.warmup + 1}-{args.warmup + args.steps} of the seeded "
                                   "solve, whole iterations"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def whole_job_value(local_ms: float, ws: int, pairs_per_rank: int, device):
    """Replicas: every rank evaluates the same number of pairs on its own GPU.
    The job's time is the slowest rank's device time (all-reduce MAX, the
    same collective on every rank) and its value all ranks' pairs over it.
    Returns (max_ms, pairs/s)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([local_ms], dtype=torch.float64, device=device)
    if ws > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    t_max_ms = float(t.item())
    return t_max_ms, ws * pairs_per_rank / (t_max_ms / 1e3)


def run_ours(args):
    import torch
    import torch.distributed as dist
    import ts_b200 as T

    ws, rank, local = dist_env()
    if ws > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    wl = build_workload(args.workload, args.n)
    n, u, v, w = wl["n"], wl["u"], wl["v"], wl["w"]
    mdp = wl["problem"] == "mdp"
    problem = T.PROBLEM_MDP if mdp else T.PROBLEM_MAXBS
    m = wl["m"] if mdp else n // 2
    P = m * (n - m)
    kinds = args.structures.split(",") if args.structures else list(T.STRUCT_NAMES)
    seed = 1 + rank  # replicas: one independent seeded start per rank

    graphs, solvers = {}, {}
    for k in kinds:
        g = T.Graph(n, u, v, w, k, drop_self_loops=mdp, stream=stream.cuda_stream)
        s = T.Solver(g, problem, m=m if mdp else 0, max_iter=10**9, tenure_policy=T.TENURE_FIXED,
                     tenure=wl["tenure"], piter=500, gamma=150, seed=seed,
                     sweep={"auto": T.PASS_AUTO, "tile": T.PASS_TILE, "rows": T.PASS_ROWS}[args.sweep])
        s.init(None)
        graphs[k], solvers[k] = g, s
    total = args.warmup + args.steps
    for k in kinds:
        adm = solvers[k].prepare(total)
        assert adm == total, (k, adm)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device=dev)

    # per-structure compulsory bytes, from the state at the start of the timed region
    gi = graphs[kinds[0]].info()
    solver_grid = {k: solvers[k].info().grid for k in kinds}
    w_bytes = max(1, solvers["wswap"].info().w_bytes) if "wswap" in kinds else 4
    words = (n + 63) // 64
    wpr = words + (words & 1)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            for k in kinds:
                flush.zero_()
                solvers[k].enqueue(1)
    torch.cuda.synchronize(dev)
    sol, _, _, _ = solvers[kinds[0]].state()
    rowptr = np.zeros(n + 1, np.int64)
    deg = np.bincount(np.concatenate([u, v]), minlength=n).astype(np.int64)
    inside = sol[:m]
    deg_in = deg[inside]
    cap_in = np.array([_hash_cap(int(d)) for d in deg_in], np.int64)
    ldc = (n - m + 3) // 4 * 4
    key_bytes = 4 if 4 * gi.max_weighted_degree < (1 << 30) else 8
    bytes_per_iter = {k: algorithmic_bytes(k, n, m, ldc, key_bytes, deg_in, cap_in, wpr, w_bytes) for k in kinds}
    del rowptr

    ev = {k: [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)] for k in kinds}
    clocks = ClockSampler(local)
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    wall0 = time.time()
    with torch.cuda.stream(stream):
        # The GPU sleeps first while the host enqueues every timed launch, so
        # no host launch latency falls between a launch's two events.
        gpu_head_start(torch, args.steps * len(kinds))
        for i in range(args.steps):
            for k in kinds:
                flush.zero_()
                a, b = ev[k][i]
                a.record(stream)
                solvers[k].enqueue(1)
                b.record(stream)
    torch.cuda.synchronize(dev)
    wall = time.time() - wall0
    if ws > 1:
        dist.barrier()
    clocks.stop()
    for k in kinds:
        it = solvers[k].sync()
        assert it == total, (k, it, total)
    # every structure ran the same search from the same start: same state
    ref_state = solvers[kinds[0]].state()
    for k in kinds[1:]:
        for a, b in zip(ref_state, solvers[k].state()):
            assert np.array_equal(a, b), f"{k} ended the timed steps in another state than {kinds[0]}"
    agree = {"structures_agree": True, "checked": "sol, pos, tabu and contributions after the timed steps"}
    per = {}
    tot_ms = 0.0
    for k in kinds:
        ts = [a.elapsed_time(b) for a, b in ev[k]]
        ms = float(sum(ts))
        tot_ms += ms
        avg_s = ms / 1e3 / args.steps
        per[k] = {"iters_per_s": 1.0 / avg_s, "swap_gains_per_s": P / avg_s, "ms_per_iter": ms / args.steps,
                  "bytes_per_iter": bytes_per_iter[k], "achieved_gbs": bytes_per_iter[k] / avg_s / 1e9,
                  "grid": solver_grid[k]}
    t_max_ms, value = whole_job_value(tot_ms, ws, P * len(kinds) * args.steps, dev)

    peak, peak_src = measured_peaks()
    dom = max(kinds, key=lambda k: per[k]["ms_per_iter"])
    achieved = per[dom]["achieved_gbs"]
    csum = clocks.summary()
    sm_mhz = csum["sm_mhz"] or csum["sm_max_mhz"] or 1965.0
    prof = {k: profile_entry(args.workload, k, solver_grid[k]) for k in kinds}
    for k in kinds:
        pe = prof[k]
        if pe and pe.get("warp_inst"):
            per[k]["int_issue_frac"] = issue_fraction(float(pe["warp_inst"]), per[k]["ms_per_iter"] / 1e3, sm_mhz)
            per[k]["dram_bytes_ncu"] = pe.get("bytes")
            per[k]["l2_hit_rate_ncu"] = pe.get("l2_hit_pct")
            per[k]["threads_per_warp_inst_ncu"] = pe.get("threads_per_inst")
    traffic = prof[dom]["bytes"] if prof[dom] else None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "kernel": f"iter_kernel[{dom}]",
                "peak_source": peak_src,
                "int_issue_frac": per[dom].get("int_issue_frac"),
                "note": "dominant kernel = slowest structure per iteration; int_issue_frac = its warp "
                        "instructions per launch (ncu capture of the same grid) / measured launch time / "
                        "(148 SMs x 4 schedulers x SM clock)"}
    if "wswap" in per:  # the structure whose sweep is HBM-bound: the matrix streams once per iteration
        roofline["hbm_bound_kernel"] = {"kernel": "iter_kernel[wswap]", "achieved": per["wswap"]["achieved_gbs"],
                                        "frac": per["wswap"]["achieved_gbs"] / peak}

    for k in kinds:
        solvers[k].close()
        graphs[k].close()
    del flush
    torch.cuda.empty_cache()

    line = None
    if rank == 0:
        configs = None if (args.no_extras or args.no_configs) else run_configs(T, torch, dev, stream, kinds)
        ref_cuda = None if (args.no_extras or args.no_configs) else run_reference_cuda(configs)
        e2e = None if args.no_extras else run_e2e(T, torch, wl, kinds, args, seed, problem, m)
        cpu = None if args.no_extras else cpu_baseline_sample(wl, problem, m)
        batched = None if (args.no_extras or args.no_batched) else run_batched(T, torch, dev, args)
        served = None if (args.no_extras or args.no_served) else run_served_sweep(T, torch, args)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded conflict-style graph; MWIS-VR instances are not available offline)",
            "config": {"workload": wl["desc"], "n": n, "m": m, "pairs_per_iter": P, "structures": kinds,
                       "l2": "256 MiB buffer written between timed iterations (outside the events)",
                       "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU"},
            "iters_per_s": len(kinds) * args.steps / (t_max_ms / 1e3),
            "per_structure": per,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "agreement": agree,
            "configs": configs,
            "reference_cuda": ref_cuda,
            "batched": batched,
            "served": served,
            "gpu_launches": len(kinds) * args.steps,
            "clocks": csum,
            "wall_s_timed_region": wall,
        }
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line))
    return 0


def _hash_cap(deg: int) -> int:
    """Slots of a vertex's hash table: power of two >= 2 * degree, at least 8."""
    cap = 8
    while cap < 2 * deg:
        cap <<= 1
    return cap


def gpu_head_start(torch, launches: int):
    """Keeps the current stream busy ~0.3 ms per upcoming launch (at least 50
    ms) so the host can enqueue them all before the device reaches them."""
    seconds = max(0.05, 3e-4 * launches)
    torch.cuda._sleep(int(seconds * 2.0e9))


def time_structures(T, torch, dev, stream, wl, problem, m, kinds, iters, warmup, flush_between, seed=1):
    """Plain solves of one workload, one structure at a time (built, started
    from the same seeded state, `warmup` untimed iterations, then `iters`
    timed ones).  flush_between: a 256 MiB buffer is written before every
    timed iteration (outside its events); otherwise the iterations run back
    to back between one pair of events, as a caller's loop runs them.
    Returns per structure it/s, swap-gains/s and the state reached."""
    n = wl["n"]
    P = m * (n - m)
    mdp = problem == T.PROBLEM_MDP
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device=dev) if flush_between else None
    out = {}
    for k in kinds:
        g = T.Graph(n, wl["u"], wl["v"], wl["w"], k, drop_self_loops=mdp, stream=stream.cuda_stream)
        s = T.Solver(g, problem, m=m if mdp else 0, max_iter=10**9, tenure_policy=T.TENURE_FIXED,
                     tenure=wl["tenure"], piter=500, gamma=150, seed=seed)
        try:
            s.init(None)
            assert s.prepare(warmup + iters) == warmup + iters
            with torch.cuda.stream(stream):
                s.enqueue(warmup)
            torch.cuda.synchronize(dev)
            evs = []
            with torch.cuda.stream(stream):
                gpu_head_start(torch, iters)
                if flush is None:
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                    s.enqueue(iters)
                    b.record(stream)
                    evs.append((a, b))
                else:
                    for _ in range(iters):
                        flush.zero_()
                        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        a.record(stream)
                        s.enqueue(1)
                        b.record(stream)
                        evs.append((a, b))
            torch.cuda.synchronize(dev)
            assert s.sync() == warmup + iters
            each = [a.elapsed_time(b) for a, b in evs]
            ms = sum(each)
            st = s.state()
            si = s.info()
        finally:
            s.close()
            g.close()
        sec = ms / 1e3 / iters
        out[k] = {"iters_per_s": 1.0 / sec, "swap_gains_per_s": P / sec, "ms_per_iter": ms / iters,
                  "grid": si.grid, "w_bytes": si.w_bytes, "_state": st}
        if len(each) > 1:
            out[k]["ms_first_last"] = [round(each[0], 4), round(each[-1], 4)]
    states = [out[k].pop("_state") for k in kinds]
    same = all(all(np.array_equal(a, b) for a, b in zip(states[0], st)) for st in states[1:])
    return out, same, states[0]


def run_configs(T, torch, dev, stream, kinds):
    """Config 1 (MDP ER n=2000, m=200, tenure 20) and config 3 (MDP Chung-Lu
    n=200000, m=2000, tenure 100) per structure, plus config 3's graph at
    m=1000 (the only m at which the reference's own loaders accept that
    graph, see run_reference_cuda).  Config 1's iterations run back to back
    (its whole state is a few hundred KB); config 3's are timed one at a time
    with L2 flushed between them and reported against the HBM roofline."""
    from ts_b200 import gen
    peak, peak_src = measured_peaks()
    res = {}
    c1 = gen.config1()
    per, same, _ = time_structures(T, torch, dev, stream, c1, T.PROBLEM_MDP, c1["m"], kinds, iters=3000,
                                   warmup=200, flush_between=False)
    res["config1"] = {"workload": WORKLOADS["config1"][1], "timed": "iterations 201-3200, back to back",
                      "per_structure": per, "structures_agree": same}
    c3 = gen.config3()
    n, m = c3["n"], c3["m"]
    per, same, st = time_structures(T, torch, dev, stream, c3, T.PROBLEM_MDP, m, kinds, iters=30, warmup=5,
                                    flush_between=True)
    deg = np.bincount(np.concatenate([c3["u"], c3["v"]]), minlength=n).astype(np.int64)
    sol = st[0]
    deg_in = deg[sol[:m]]
    cap_in = np.array([_hash_cap(int(d)) for d in deg_in], np.int64)
    words = (n + 63) // 64
    wpr = words + (words & 1)
    ldc = (n - m + 3) // 4 * 4
    for k in kinds:
        b = algorithmic_bytes(k, n, m, ldc, 4, deg_in, cap_in, wpr, w_bytes=max(1, per[k]["w_bytes"]))
        per[k]["bytes_per_iter"] = b
        per[k]["achieved_gbs"] = b * per[k]["iters_per_s"] / 1e9
        per[k]["hbm_frac"] = per[k]["achieved_gbs"] / peak
    res["config3"] = {"workload": WORKLOADS["config3"][1], "timed": "iterations 6-35, 256 MiB L2 flush before each",
                      "per_structure": per, "structures_agree": same, "peak_gbs": peak, "peak_source": peak_src}
    c3b = dict(c3, m=1000)
    per, same, _ = time_structures(T, torch, dev, stream, c3b, T.PROBLEM_MDP, 1000, kinds, iters=30, warmup=5,
                                   flush_between=True)
    res["config3_m1000"] = {"workload": "config3 graph with m=1000 (the reference's b2500 loader fixes m=1000)",
                            "timed": "iterations 6-35, 256 MiB L2 flush before each", "per_structure": per,
                            "structures_agree": same}
    return res


def _write_instance(path, n, u, v, w, header, one_based):
    import pandas as pd
    with open(path, "w") as f:
        f.write(header + "\n")
    off = 1 if one_based else 0
    pd.DataFrame({"a": u.astype(np.int64) + off, "b": v.astype(np.int64) + off, "w": w}).to_csv(
        path, sep=" ", header=False, index=False, mode="a")


REF_MDP_ALGS = ["csr", "csr-bb", "csr-bitset-bb", "hash", "wswap"]


def run_reference_cuda(configs):
    """The reference's own CUDA programs, built unmodified from its sources by
    oracle/build_ref.sh (linked with a shim that injects the seed, stamps
    every ArgMax copy with a monotonic clock and exits after a set number of
    them), timed on this GPU.  Iterations/s = ArgMax copies between the first
    and the last stamp / elapsed time of the first tabu call.
      config 1: MDG-a file "2000 200" (the exact config);
      config 3's graph: the MDG-a header computes n(n-1)/2 in int, which
        overflows at n = 200,000, and the other loaders fix m (sparse/nenad
        100, b2500 1000, p3000-5000 n/2 -- too many pairs for int indices),
        so the b2500 loader runs it, at m = 1000, beside this engine at m = 1000.
    GPU-MDP-CSR-Bitset.cu does not compile (syntax error); the Hash program
    packs (u<<16)|v into 32 bits, so its lookups alias above n = 65,536."""
    import tempfile
    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    if not all(os.path.exists(os.path.join(ref_dir, f"mdp_{a}")) for a in REF_MDP_ALGS):
        return {"unavailable": "reference programs not built (oracle/_ref); oracle/build_ref.sh builds them"}
    from ts_b200 import gen
    out = {"what": "the reference's own CUDA programs, unmodified, on this GPU; iterations/s of their first "
                   "tabu call (ArgMax copy stamps)",
           "csr-bitset": "not buildable (GPU-MDP-CSR-Bitset.cu does not compile)"}
    cases = [("config1", gen.config1(), "MDG-a", 3000, False),
             ("config3_m1000", gen.config3(), "b2500", 30, True)]
    with tempfile.TemporaryDirectory() as td:
        for name, wl, fmt, limit, one_based in cases:
            n = wl["n"]
            path = os.path.join(td, name + ".txt")
            if fmt == "MDG-a":
                _write_instance(path, n, wl["u"], wl["v"], wl["w"], f"{n} {wl['m']}", False)
            else:
                _write_instance(path, n, wl["u"], wl["v"], wl["w"], f"{n} {len(wl['u'])}", True)
            per = {}
            for alg in REF_MDP_ALGS:
                trace = os.path.join(td, f"{name}_{alg}.trace")
                env = dict(os.environ, TS_REF_TRACE=trace, TS_REF_N=str(n), TS_REF_SEED="1",
                           TS_REF_LIMIT=str(limit))
                cmd = f'ulimit -s unlimited; exec "{os.path.join(ref_dir, "mdp_" + alg)}" "{path}" {fmt} 100000 1'
                t0 = time.time()
                try:
                    r = subprocess.run(["bash", "-c", cmd], env=env, stdin=subprocess.DEVNULL,
                                       stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, timeout=300)
                    rc = r.returncode
                except subprocess.TimeoutExpired:
                    rc = "timeout"
                wall = time.time() - t0
                ts = []
                if os.path.exists(trace):
                    with open(trace) as f:
                        ts = [int(x.split()[3]) for x in f if x.startswith("A ")]
                if rc != 0 or len(ts) < 3:
                    per[alg] = {"error": f"exit {rc}, {len(ts)} ArgMax records", "wall_s": wall}
                    continue
                sec = (ts[-1] - ts[0]) / 1e9
                d = {"iters_per_s": (len(ts) - 1) / sec, "iterations": len(ts), "wall_s": wall}
                if alg == "hash" and n > 65536:
                    d["note"] = "incorrect at this n: (u<<16)|v keys alias above n = 65,536"
                ours = (configs or {}).get(name, {}).get("per_structure", {}).get(alg)
                if ours:
                    d["ours_iters_per_s"] = ours["iters_per_s"]
                    d["speedup"] = ours["iters_per_s"] / d["iters_per_s"]
                per[alg] = d
            out[name] = per
    return out


def run_e2e(T, torch, wl, kinds, args, seed, problem, m):
    """Same solves through the public C-ABI with host buffers: pinned edge
    lists uploaded and built per structure, seeded start, `steps` iterations,
    best bisection read back; wall clock."""
    n = wl["n"]
    P = m * (n - m)
    pin = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in (wl["u"], wl["v"], wl["w"])]
    u, v, w = (x.numpy() for x in pin)
    h2d = 3 * 4 * len(u)
    # one untimed pass through the same calls first: the process's first
    # graph build pays one-time costs (0.2-0.6 s seen) that no later call does
    g = T.Graph(n, u, v, w, kinds[0], drop_self_loops=problem == T.PROBLEM_MDP)
    s = T.Solver(g, problem, m=m if problem == T.PROBLEM_MDP else 0, max_iter=1, tenure_policy=T.TENURE_FIXED,
                 tenure=wl["tenure"], piter=500, gamma=150, seed=seed)
    s.init(None)
    s.step(1)
    s.result()
    s.close()
    g.close()
    t_tot = 0.0
    parts = {}
    for k in kinds:
        torch.cuda.synchronize()
        t0 = time.time()
        g = T.Graph(n, u, v, w, k, drop_self_loops=problem == T.PROBLEM_MDP)
        t1 = time.time()
        s = T.Solver(g, problem, m=m if problem == T.PROBLEM_MDP else 0, max_iter=args.steps,
                     tenure_policy=T.TENURE_FIXED, tenure=wl["tenure"], piter=500, gamma=150, seed=seed)
        s.init(None)
        t2 = time.time()
        s.step(args.steps)
        t3 = time.time()
        r = s.result()
        t4 = time.time()
        t_tot += t4 - t0
        parts[k] = {"graph_s": t1 - t0, "solver_init_s": t2 - t1, "steps_s": t3 - t2, "result_s": t4 - t3}
        assert r.iterations == args.steps and r.device_error == 0
        s.close()
        g.close()
    return {"value": P * len(kinds) * args.steps / t_tot, "unit": UNIT, "seconds": parts,
            "warmup": "one untimed graph build + init + 1 step + result before the timed structures",
            "h2d_bytes_per_step": h2d * len(kinds) / args.steps,
            "d2h_bytes_per_step": 4 * (m if problem == T.PROBLEM_MDP else n) * len(kinds) / args.steps,
            "what": "per structure: ts_graph_create from pinned host edges + ts_solver_init + "
                    "ts_solver_step(steps) + ts_solver_result, wall clock"}


def run_batched(T, torch, dev, args):
    """Batched form on a bounded prefix of the batched workload (config 4):
    `c4_instances` of its 4096 instances x 8 seeded restarts, 5000 iterations
    each, structure and cluster size per size bucket from the autotuner.
    value: solves per second of device time of one replay of the captured
    launch (inputs resident); e2e: the same through the public API from
    pinned host edge lists (graph builds, batch set-up, replay, results read
    back); plain: a stratified sample of the same solves run one at a time
    with ts_solver_* (init, step, result), wall clock; every sampled solve is
    checked equal to its batched result.  Cluster sizes are left to the
    library, which spreads the solves that would outlast the rest over more
    CTAs; the autotuner's structure choice is used as is."""
    from ts_b200 import autotune as AT
    t_tune = time.time()
    table = AT.autotune(budget_s=args.tune_budget)
    t_tune = time.time() - t_tune
    insts = T.gen.config4(instances=args.c4_instances, restarts=8, iters=5000)
    stream = torch.cuda.Stream(device=dev)
    pinned = []
    for inst in insts:
        pinned.append([torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
                       for a in (inst["u"], inst["v"], inst["w"])])
    torch.cuda.synchronize(dev)
    e2e0 = time.time()
    graphs, specs = [], []
    for inst, (u, v, w) in zip(insts, pinned):
        mdp = inst["problem"] == "mdp"
        prob = T.PROBLEM_MDP if mdp else T.PROBLEM_MAXBS
        kind, _ = table.pick(prob, inst["n"])
        sweep = table.pick_sweep(prob, inst["n"])
        g = T.Graph(inst["n"], u, v, w, kind, drop_self_loops=mdp)
        graphs.append(g)
        for sd in inst["seeds"]:
            specs.append(T.BatchJobSpec(g, prob, m=inst["m"] if mdp else 0, max_iter=inst["iters"],
                                        tenure_policy=T.TENURE_FIXED, tenure=20 if mdp else 50,
                                        piter=500, gamma=150, seed=sd, cluster=0, sweep=sweep))
    b = T.Batch(specs, stream=stream.cuda_stream)
    b.launch()
    b.sync()
    res = b.results()
    e2e = time.time() - e2e0
    info = b.info()
    # device-timed replay
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    torch.cuda.nvtx.range_push("config4 replay")  # ncu --nvtx --nvtx-include "config4 replay/"
    ev0.record(stream)
    b.launch()
    ev1.record(stream)
    torch.cuda.nvtx.range_pop()
    b.sync()
    torch.cuda.synchronize(dev)
    dev_s = ev0.elapsed_time(ev1) / 1e3
    again = b.results()
    assert all((a.best, a.best_true, a.iterations) == (c.best, c.best_true, c.iterations) for a, c in zip(res, again))
    pairs = sum(((sp.m if sp.problem == T.PROBLEM_MDP else sp.graph.n // 2)
                 * (sp.graph.n - (sp.m if sp.problem == T.PROBLEM_MDP else sp.graph.n // 2)) * r.iterations)
                for sp, r in zip(specs, res))
    # plain one-launch-per-iteration mode on a stratified sample (by work)
    order = sorted(range(len(specs)), key=lambda q: res[q].evaluations)
    stride = max(1, len(order) // args.c4_plain_sample)
    sample = order[stride // 2::stride][:args.c4_plain_sample]
    t_plain = 0.0
    identical = True
    for q in sample:
        sp = specs[q]
        t0 = time.time()
        sv = T.Solver(sp.graph, sp.problem, m=sp.m, max_iter=sp.max_iter, tenure_policy=sp.tenure_policy,
                      tenure=sp.tenure, piter=sp.piter, gamma=sp.gamma, seed=sp.seed)  # plain: its own auto sweep
        sv.init(None)
        sv.step(sp.max_iter)
        r = sv.result()
        sv.close()
        t_plain += time.time() - t0
        a = res[q]
        identical &= (r.iterations, r.evaluations, r.cur, r.best, r.best_true) == \
            (a.iterations, a.evaluations, a.cur, a.best, a.best_true) and bool(np.array_equal(r.best_sol, a.best_sol))
    # the sample is stratified over the sorted work, so its mean time per solve
    # estimates the mean over all solves
    plain_sps = len(sample) / t_plain
    b.close()
    for g in graphs:
        g.close()
    sizes = [i["n"] for i in insts]
    return {
        "workload": f"config4 prefix: {len(insts)} of 4096 instances x 8 restarts = {len(specs)} solves; "
                    "ER n log-uniform [200,20000], mean degree U[5,50], half MDP (m=U[5%,20%]n, tenure 20), "
                    "half MaxBS (tenure 50, Piter 500, gamma 150); 5000 iterations each",
        "solves": len(specs), "n_range": [min(sizes), max(sizes)],
        "solves_per_s": len(specs) / dev_s, "device_s": dev_s, "swap_gains_per_s": pairs / dev_s,
        "e2e_solves_per_s": len(specs) / e2e, "e2e_s": e2e,
        "plain_solves_per_s": plain_sps, "plain_sample": len(sample),
        "speedup_vs_plain": (len(specs) / dev_s) / plain_sps,
        "e2e_speedup_vs_plain": (len(specs) / e2e) / plain_sps,
        "identical_to_plain": bool(identical),
        "groups": info.groups, "slots": info.slots, "slot_bytes": info.slot_bytes,
        "autotune": table.as_dict(), "autotune_s": t_tune,
        "autotune_unavailable": [t for t in table.trials if "unavailable" in t],
    }


def _serve_once(T, reqs, arrivals, round_ms):
    """Submits reqs[i] at arrivals[i] (seconds from the start) to a fresh
    server and collects every completion; returns (span_s, latencies_s,
    results, stats)."""
    srv = T.Server(round_ms=round_ms)
    got, tickets = {}, []
    t0 = srv.now()
    k = 0
    while k < len(reqs) or len(got) < len(reqs):
        now = srv.now() - t0
        while k < len(reqs) and arrivals[k] <= now:
            r = reqs[k]
            mdp = r["problem"] == "mdp"
            tickets.append(srv.submit(r["n"], r["u"], r["v"], r["w"], T.PROBLEM_MDP if mdp else T.PROBLEM_MAXBS,
                                      kind="csr", m=r["m"] if mdp else 0, max_iter=r["iters"],
                                      tenure_policy=T.TENURE_FIXED, tenure=r["tenure"], seed=r["seed"]))
            k += 1
        for d in srv.poll(wait_ms=1 if k < len(reqs) else 20):
            got[d.ticket] = d
    st = srv.stats()
    srv.close()
    lat = np.array([got[tk].done_s - got[tk].submit_s for tk in tickets])
    span = max(got[tk].done_s for tk in tickets) - t0
    return span, lat, [got[tk] for tk in tickets], st


def run_served_sweep(T, torch, args):
    """Served form (config 5) at three offered loads, bounded: a pool of
    `served_requests` requests drawn as config 5 (70% MDP Chung-Lu, m = n/100,
    tenure 100; 30% Max Bisection conflict graphs, tenure 50; n log-uniform in
    [1e3, n_hi]; budgets U[1000, 10000]).  Capacity = requests / makespan when
    all arrive at once; then open-loop Poisson arrivals at 0.5x and 1x that
    capacity.  Beside each run, the plain one-at-a-time loop: the same requests
    each run alone (graph build + ts_solver_*, their measured service times)
    and queued FIFO at the same arrival times.  Every served result must equal
    its alone result."""
    t_gen = time.time()
    reqs = T.gen.config5_requests(args.served_requests, n_hi=args.served_n_hi)
    t_gen = time.time() - t_gen
    service, alone = [], []
    for r in reqs:
        mdp = r["problem"] == "mdp"
        torch.cuda.synchronize()
        a = time.time()
        g = T.Graph(r["n"], r["u"], r["v"], r["w"], "csr", drop_self_loops=mdp)
        sv = T.Solver(g, T.PROBLEM_MDP if mdp else T.PROBLEM_MAXBS, m=r["m"] if mdp else 0, max_iter=r["iters"],
                      tenure_policy=T.TENURE_FIXED, tenure=r["tenure"], seed=r["seed"])
        sv.init(None)
        sv.step(r["iters"])
        alone.append(sv.result())
        sv.close()
        g.close()
        service.append(time.time() - a)
    pct = lambda x, q: float(np.percentile(x, q))

    def summary(span, lat, res, st, arrivals):
        ok = all(d.result is not None and (d.result.best, d.result.best_true, d.result.iterations,
                                           d.result.evaluations) == (a.best, a.best_true, a.iterations, a.evaluations)
                 and bool(np.array_equal(d.result.best_sol, a.best_sol)) for d, a in zip(res, alone))
        fin, plain_lat = 0.0, []
        for arr, sv_t in zip(arrivals, service):
            fin = max(arr, fin) + sv_t
            plain_lat.append(fin - arr)
        plain_lat = np.array(plain_lat)
        return {"solves_per_s": len(reqs) / span, "span_s": span,
                "latency_s": {"p50": pct(lat, 50), "p95": pct(lat, 95), "p99": pct(lat, 99), "max": float(lat.max())},
                "plain_one_at_a_time": {"solves_per_s": len(reqs) / fin, "span_s": fin,
                                        "latency_s": {"p50": pct(plain_lat, 50), "p95": pct(plain_lat, 95),
                                                      "p99": pct(plain_lat, 99), "max": float(plain_lat.max())}},
                "identical_to_alone": bool(ok), "rounds": st.rounds,
                "executors": {e: sum(1 for d in res if d.executor == e) for e in ("packed", "plain")}}

    out = {"workload": f"config5 pool: {len(reqs)} requests, 70% MDP Chung-Lu (m=n/100, tenure 100) / 30% MaxBS "
                       f"conflict (tenure 50), n log-uniform [1000,{args.served_n_hi}], budgets U[1000,10000], "
                       "structure csr",
           "n_range": [min(r["n"] for r in reqs), max(r["n"] for r in reqs)], "generation_s": t_gen,
           "alone_service_s_total": float(sum(service))}
    zero = [0.0] * len(reqs)
    span, lat, res, st = _serve_once(T, reqs, zero, args.round_ms)
    cap = len(reqs) / span
    out["capacity_solves_per_s"] = cap
    out["saturation"] = summary(span, lat, res, st, zero)
    rng = np.random.default_rng(55)
    for f in (0.5, 1.0):
        arrivals = list(np.cumsum(rng.exponential(1.0 / (f * cap), size=len(reqs))))
        span, lat, res, st = _serve_once(T, reqs, arrivals, args.round_ms)
        d = summary(span, lat, res, st, arrivals)
        d["offered_per_s"] = f * cap
        out[f"load_{f:g}x"] = d
    out["served_vs_plain_at_saturation"] = out["saturation"]["solves_per_s"] / \
        out["saturation"]["plain_one_at_a_time"]["solves_per_s"]
    return out


def run_served(args):
    """Served workload (config 5): open-loop Poisson arrivals at `rate`/s for
    `duration` s; 70% MDP (Chung-Lu graphs) / 30% Max Bisection (conflict
    graphs), n log-uniform in [1e3, 2e5], budgets U[1000, 10000] iterations.
    The server builds each graph on the device from the request's host edge
    list, admits by HBM footprint and batches solves continuously.  Beside it,
    the plain one-at-a-time loop: the same requests each run alone (graph
    build + ts_solver_*), queued FIFO at the same arrival times."""
    import torch
    import ts_b200 as T
    torch.cuda.set_device(0)
    rng = np.random.default_rng(55)
    arrivals = []
    t = 0.0
    while True:
        t += rng.exponential(1.0 / args.rate)
        if t > args.duration:
            break
        arrivals.append(t)
    t_gen = time.time()
    reqs = T.gen.config5_requests(len(arrivals), n_hi=args.served_n_hi)
    t_gen = time.time() - t_gen
    srv = T.Server(round_ms=args.round_ms)
    got = {}
    tickets = []
    clocks = ClockSampler(0)
    clocks.start()
    t0 = srv.now()
    k = 0
    while k < len(reqs) or len(got) < len(reqs):
        now = srv.now() - t0
        while k < len(reqs) and arrivals[k] <= now:
            r = reqs[k]
            mdp = r["problem"] == "mdp"
            tk = srv.submit(r["n"], r["u"], r["v"], r["w"], T.PROBLEM_MDP if mdp else T.PROBLEM_MAXBS,
                            kind="csr", m=r["m"] if mdp else 0, max_iter=r["iters"],
                            tenure_policy=T.TENURE_FIXED, tenure=r["tenure"], seed=r["seed"])
            tickets.append(tk)
            k += 1
        wait = 1 if k < len(reqs) else 20
        for d in srv.poll(wait_ms=wait):
            got[d.ticket] = d
    clocks.stop()
    st = srv.stats()
    srv.close()
    lat = np.array([got[tk].done_s - got[tk].submit_s for tk in tickets])
    span = max(got[tk].done_s for tk in tickets) - t0
    # plain one-at-a-time loop, FIFO at the same arrivals
    service, identical = [], True
    for tk, r in zip(tickets, reqs):
        mdp = r["problem"] == "mdp"
        torch.cuda.synchronize()
        a = time.time()
        g = T.Graph(r["n"], r["u"], r["v"], r["w"], "csr", drop_self_loops=mdp)
        sv = T.Solver(g, T.PROBLEM_MDP if mdp else T.PROBLEM_MAXBS, m=r["m"] if mdp else 0, max_iter=r["iters"],
                      tenure_policy=T.TENURE_FIXED, tenure=r["tenure"], seed=r["seed"])
        sv.init(None)
        sv.step(r["iters"])
        res = sv.result()
        sv.close()
        g.close()
        service.append(time.time() - a)
        d = got[tk].result
        identical &= d is not None and (d.best, d.best_true, d.iterations, d.evaluations) == \
            (res.best, res.best_true, res.iterations, res.evaluations) and bool(np.array_equal(d.best_sol, res.best_sol))
    fin, plain_lat = 0.0, []
    for arr, sv_t in zip(arrivals, service):
        fin = max(arr, fin) + sv_t
        plain_lat.append(fin - arr)
    plain_lat = np.array(plain_lat)
    pct = lambda x, q: float(np.percentile(x, q))
    line = {
        "metric": METRIC, "value": len(tickets) / span, "unit": "solves/s", "n_gpus": 1,
        "steps": len(tickets), "warmup": 0, "ms_per_step": 1e3 * span / len(tickets), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded per request)",
        "config": {"workload": f"config5: Poisson arrivals {args.rate}/s for {args.duration} s; 70% MDP Chung-Lu "
                               f"(m=n/100, tenure 100) / 30% MaxBS conflict (tenure 50); n log-uniform "
                               f"[1000,{args.served_n_hi}]; budgets U[1000,10000]; structure csr",
                   "round_ms": args.round_ms},
        "served": {"requests": len(tickets), "latency_s": {"p50": pct(lat, 50), "p95": pct(lat, 95),
                                                           "p99": pct(lat, 99), "max": float(lat.max())},
                   "executors": {e: sum(1 for tk in tickets if got[tk].executor == e) for e in ("packed", "plain")},
                   "rounds": st.rounds, "busy_s": st.busy_s, "span_s": span},
        "plain_one_at_a_time": {"solves_per_s": len(tickets) / (fin - arrivals[0] + arrivals[0]),
                                "latency_s": {"p50": pct(plain_lat, 50), "p95": pct(plain_lat, 95),
                                              "p99": pct(plain_lat, 99), "max": float(plain_lat.max())},
                                "service_s_total": float(sum(service))},
        "identical_to_alone": bool(identical),
        "slowest": [{"n": reqs[q]["n"], "problem": reqs[q]["problem"], "iters": reqs[q]["iters"],
                     "executor": got[tickets[q]].executor, "arrival_s": round(arrivals[q], 3),
                     "latency_s": round(float(lat[q]), 3), "alone_s": round(service[q], 3)}
                    for q in np.argsort(-lat)[:6]],
        "generation_s": t_gen,
        "clocks": clocks.summary(),
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="config2",
                    help="config2 is the benchmark; the others serve profiling")
    ap.add_argument("--structures", default="", help="comma list (default: all six)")
    ap.add_argument("--n", type=int, default=0, help="config2/config3 at another size (profiling cases)")
    ap.add_argument("--no-extras", action="store_true", help="skip the e2e, CPU-baseline and batched legs")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched (config 4) leg")
    ap.add_argument("--no-served", action="store_true", help="skip the served (config 5) load sweep")
    ap.add_argument("--served-requests", type=int, default=24, help="served sweep: requests in the pool")
    ap.add_argument("--sweep", choices=["auto", "tile", "rows"], default="auto",
                    help="pair sweep of the main leg's solvers (ts_pass; auto picks by size)")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the config-1/config-3 legs and the reference CUDA build's timing")
    ap.add_argument("--c4-instances", type=int, default=40, help="batched leg: instances of config 4")
    ap.add_argument("--c4-plain-sample", type=int, default=24, help="batched leg: solves run plain")
    ap.add_argument("--tune-budget", type=float, default=30.0, help="autotuner time budget (s)")
    ap.add_argument("--rate", type=float, default=2.0, help="config5: requests per second")
    ap.add_argument("--duration", type=float, default=60.0, help="config5: arrival window (s)")
    ap.add_argument("--served-n-hi", type=int, default=200_000, help="config5: largest n")
    ap.add_argument("--round-ms", type=float, default=5.0, help="config5: server round target")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "config5":
        return run_served(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
