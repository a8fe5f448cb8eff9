"""Generates tests/golden/*.npz from the reference's OWN CUDA programs.

Runs on a GPU box, after ``oracle/build_ref.sh`` built the unmodified
reference sources (oracle/_ref/, linked with oracle/ref_shim.c).  For every
case below it writes the instance in the reference's input format, runs every
reference program of that problem with a fixed seed and an iteration cap, and
records from the shim's trace what the reference's first tabu call did: its
start solution and, per iteration, the ArgMax (flat index, float value) it
copied to the host, plus the MaxBS perturbation gains.

Instances keep every value below 2^24 so the reference's float arithmetic is
exact and comparable with the integer oracle.  The CPU test
(tests/test_golden_cpu.py) regenerates each instance with ``instance()`` and
checks the oracle against these fixtures.

    python tests/golden/make_golden.py [--only CASE] [--timing]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_BIN = os.path.join(ROOT, "oracle", "_ref")

MDP_ALGS = ["csr", "csr-bb", "csr-bitset-bb", "hash", "wswap"]  # csr-bitset does not compile
MAXBS_ALGS = ["csr", "csr-bb", "csr-bitset", "csr-bitset-bb", "hash", "wswap"]

CASES = {
    # name: (problem, generator spec, run params)
    "mdp_small": ("mdp", dict(kind="dense", n=60, p=0.3, wmax=50, seed=11), dict(m=10, iters=1500, seed=12345)),
    "mdp_er300": ("mdp", dict(kind="er", n=300, deg=8.0, seed=21), dict(m=30, iters=2000, seed=777)),
    "mdp_config1": ("mdp", dict(kind="er", n=2000, deg=20.0, seed=1), dict(m=200, iters=2000, seed=1)),
    "mdp_break": ("mdp", dict(kind="complete", n=8, w=7, seed=0), dict(m=4, iters=200, seed=3)),
    "maxbs_tiny": ("maxbs", dict(kind="dense", n=13, p=0.45, wmax=40, seed=31),
                   dict(iters=600, seed=5, maxt=16, piter=20, gamma=6)),
    "maxbs_small": ("maxbs", dict(kind="dense", n=41, p=0.25, wmax=60, seed=32),
                    dict(iters=1500, seed=6, maxt=200, piter=25, gamma=12)),
    "maxbs_er500": ("maxbs", dict(kind="er", n=500, deg=12.0, seed=33),
                    dict(iters=2000, seed=7, maxt=40, piter=40, gamma=30)),
    "maxbs_er2001": ("maxbs", dict(kind="er", n=2001, deg=8.0, seed=34),
                     dict(iters=1500, seed=8, maxt=200, piter=500, gamma=150)),
}


def instance(spec: dict):
    """Deterministic (n, u, v, w) for a case spec (0-based, u < v, no duplicates)."""
    sys.path.insert(0, os.path.join(ROOT, "graph-data-structures-local-search_b200"))
    from ts_b200 import gen

    n = spec["n"]
    if spec["kind"] == "er":
        u, v, w, _ = gen.erdos_renyi(n, spec["deg"], spec["seed"])
    elif spec["kind"] == "complete":
        a, b = np.triu_indices(n, 1)
        u, v, w = a.astype(np.int32), b.astype(np.int32), np.full(len(a), spec["w"], np.int32)
    else:
        rng = np.random.default_rng(spec["seed"])
        a, b = np.triu_indices(n, 1)
        keep = rng.random(len(a)) < spec["p"]
        u, v = a[keep].astype(np.int32), b[keep].astype(np.int32)
        w = rng.integers(1, spec["wmax"] + 1, size=len(u)).astype(np.int32)
    return n, u, v, w


def parse_trace(path: str):
    calls = []
    with open(path) as f:
        for line in f:
            t = line.split()
            if not t:
                continue
            if t[0] == "I":
                calls.append(dict(init=[int(x) for x in t[1:]], idx=[], value=[], t=[], perturb=[]))
            elif t[0] == "A" and calls:
                calls[-1]["idx"].append(int(t[1]))
                calls[-1]["value"].append(float(t[2]))
                calls[-1]["t"].append(int(t[3]))
            elif t[0] == "P" and calls:
                calls[-1]["perturb"].append((len(calls[-1]["idx"]), float(t[1])))
    return calls


def run_case(name: str, timing: bool):
    problem, spec, rp = CASES[name]
    n, u, v, w = instance(spec)
    algs = MDP_ALGS if problem == "mdp" else MAXBS_ALGS
    out = {}
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, name + ".txt")
        with open(path, "w") as f:
            if problem == "mdp":  # MDG-a branch: "n m" + 0-based lines (GPU-MDP-CSR.cu:273-280)
                f.write(f"{n} {rp['m']}\n")
                for a, b, c in zip(u, v, w):
                    f.write(f"{a} {b} {c}\n")
            else:                 # MaxBS loader: "n n E" + 1-based lines (GPU-MAXBS-CSR.cu:144-166)
                f.write(f"{n} {n} {len(u)}\n")
                for a, b, c in zip(u, v, w):
                    f.write(f"{a + 1} {b + 1} {c}\n")
        for alg in algs:
            exe = os.path.join(REF_BIN, f"{problem}_{alg}")
            if not os.path.exists(exe):
                print(f"[{name}] missing {exe}")
                continue
            trace = os.path.join(td, f"{alg}.trace")
            env = dict(os.environ, TS_REF_TRACE=trace, TS_REF_N=str(n), TS_REF_SEED=str(rp["seed"]),
                       TS_REF_LIMIT=str(rp["iters"]))
            if problem == "mdp":
                cmd = [exe, path, "MDG-a", "1000", "1"]
            else:
                cmd = [exe, path, "-seed", str(rp["seed"]), "-maxiter", str(rp["iters"]),
                       "-maxt", str(rp["maxt"]), "-piter", str(rp["piter"]),
                       "-gamma", str(rp["gamma"]), "-time", "1000", "-p", "1"]
            t0 = time.time()
            r = subprocess.run(cmd, env=env, stdin=subprocess.DEVNULL, stdout=subprocess.PIPE,
                               stderr=subprocess.STDOUT, timeout=600)
            wall = time.time() - t0
            if r.returncode != 0:
                print(f"[{name}/{alg}] exit {r.returncode}: {r.stdout[-400:]!r}")
                continue
            calls = parse_trace(trace)
            if not calls:
                print(f"[{name}/{alg}] empty trace")
                continue
            c = calls[0]
            out[alg] = c
            if timing and len(c["t"]) > 10:
                dt = (c["t"][-1] - c["t"][0]) / 1e9
                print(f"[{name}/{alg}] {len(c['t'])} iterations; "
                      f"{(len(c['t']) - 1) / dt:.0f} it/s between first and last ArgMax; wall {wall:.1f}s")
    if not out:
        return None
    ref_alg = next(iter(out))
    base = out[ref_alg]
    agree = [a for a, c in out.items()
             if c["idx"] == base["idx"] and c["value"] == base["value"] and c["init"] == base["init"]
             and c["perturb"] == base["perturb"]]
    differ = [a for a in out if a not in agree]
    fix = dict(
        init=np.array(base["init"], np.int32),
        idx=np.array(base["idx"], np.int64),
        value=np.array(base["value"], np.float64),
        perturb_at=np.array([p[0] for p in base["perturb"]], np.int64),
        perturb_value=np.array([p[1] for p in base["perturb"]], np.float64),
    )
    meta = dict(case=name, problem=problem, spec=spec, params=rp, programs_agreeing=agree,
                programs_differing=differ, records=len(base["idx"]))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **fix, meta=json.dumps(meta))
    for a in differ:
        c = out[a]
        np.savez_compressed(os.path.join(HERE, f"{name}__{a}.npz"), init=np.array(c["init"], np.int32),
                            idx=np.array(c["idx"], np.int64), value=np.array(c["value"], np.float64),
                            meta=json.dumps(dict(meta, program=a)))
    print(f"[{name}] {len(base['idx'])} records; agreeing {agree}; differing {differ}")
    return meta


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only")
    ap.add_argument("--timing", action="store_true")
    a = ap.parse_args()
    names = [a.only] if a.only else list(CASES)
    for nm in names:
        run_case(nm, a.timing)


if __name__ == "__main__":
    main()
