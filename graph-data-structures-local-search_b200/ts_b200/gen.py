"""Deterministic synthetic instances and the reference's file formats.

The MWIS-VR conflict graphs the reference runs on are not available offline;
these seeded generators stand in for them with the shapes the benchmark
configurations name:

* ``erdos_renyi``   G(n, p) by geometric skipping over the upper triangle
                    (Batagelj & Brandes 2005),
* ``conflict_graph`` unit-square points joined within a radius chosen for a
                    mean degree, plus random cliques (conflict-style graphs),
* ``chung_lu``      power-law expected degrees, edges drawn by the fast
                    Chung-Lu endpoint sampling of Pinar, Seshadhri & Kolda (2012),
                    self-loops and duplicates removed.

Node weights are int32 uniform in [1, 1000]; w(u, v) = nw_u + nw_v.  Every
generator returns 0-based (u, v, w) int32 arrays with u < v and no duplicates.

Writers/readers cover the formats the reference loaders parse:
``sparse`` / MaxBS ("n n E" + 1-based "u v w", GPU-MDP-CSR.cu:299-306,
GPU-MAXBS-CSR.cu:144-166) and ``MDG`` ("n m" + 0-based lines, GPU-MDP-CSR.cu:273-280).
"""
from __future__ import annotations

import math

import numpy as np


def node_weights(n: int, rng: np.random.Generator) -> np.ndarray:
    return rng.integers(1, 1001, size=n, dtype=np.int64).astype(np.int32)


def _finish(n: int, a: np.ndarray, b: np.ndarray, rng: np.random.Generator):
    a = np.asarray(a, np.int64)
    b = np.asarray(b, np.int64)
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    keep = lo != hi
    key = np.unique(lo[keep] * n + hi[keep])
    u = (key // n).astype(np.int32)
    v = (key % n).astype(np.int32)
    nw = node_weights(n, rng)
    w = (nw[u].astype(np.int64) + nw[v]).astype(np.int32)
    return u, v, w, nw


def _pair_from_linear(k: np.ndarray, n: int):
    # Linear index over {(i, j): i < j} in row-major order -> (i, j).
    k = k.astype(np.float64)
    i = n - 2 - np.floor(np.sqrt(-8.0 * k + 4.0 * n * (n - 1) - 7.0) / 2.0 - 0.5)
    i = i.astype(np.int64)
    kk = k.astype(np.int64)
    j = kk + i + 1 - (n * (n - 1)) // 2 + ((n - i) * ((n - i) - 1)) // 2
    return i, j


def erdos_renyi(n: int, avg_degree: float, seed: int):
    """G(n, p=avg_degree/(n-1)) with geometric skipping; returns (u, v, w, nw)."""
    rng = np.random.default_rng(seed)
    total = n * (n - 1) // 2
    p = min(1.0, avg_degree / (n - 1))
    if p >= 1.0:
        k = np.arange(total, dtype=np.int64)
    else:
        expect = int(total * p + 10 * math.sqrt(total * p + 1) + 64)
        gaps = rng.geometric(p, size=expect).astype(np.int64)
        k = np.cumsum(gaps) - 1
        while k[-1] < total:
            more = np.cumsum(rng.geometric(p, size=expect).astype(np.int64)) + k[-1]
            k = np.concatenate([k, more])
        k = k[k < total]
    i, j = _pair_from_linear(k, n)
    return _finish(n, i, j, rng)


def conflict_graph(n: int, avg_degree: float, n_cliques: int, clique_lo: int, clique_hi: int,
                   seed: int):
    """Points in the unit square joined within radius r (mean degree ~avg_degree),
    plus n_cliques cliques of size U{clique_lo..clique_hi} on random vertices."""
    rng = np.random.default_rng(seed)
    pts = rng.random((n, 2))
    r = math.sqrt(avg_degree / (math.pi * (n - 1)))
    g = max(1, int(1.0 / r))
    cell = np.minimum((pts * g).astype(np.int64), g - 1)
    cid = cell[:, 0] * g + cell[:, 1]
    order = np.argsort(cid, kind="stable")
    cid_sorted = cid[order]
    starts = np.searchsorted(cid_sorted, np.arange(g * g), side="left")
    ends = np.searchsorted(cid_sorted, np.arange(g * g), side="right")
    us, vs = [], []
    r2 = r * r
    for dx in (-1, 0, 1):
        for dy in (-1, 0, 1):
            nx = cell[:, 0] + dx
            ny = cell[:, 1] + dy
            ok = (nx >= 0) & (nx < g) & (ny >= 0) & (ny < g)
            src = np.nonzero(ok)[0]
            nc = nx[src] * g + ny[src]
            cnt = ends[nc] - starts[nc]
            rep = np.repeat(src, cnt)
            off = np.repeat(starts[nc] - np.cumsum(cnt) + cnt, cnt) + np.arange(cnt.sum())
            dst = order[off]
            keep = rep < dst
            rep, dst = rep[keep], dst[keep]
            d = pts[rep] - pts[dst]
            close = (d * d).sum(axis=1) < r2
            us.append(rep[close])
            vs.append(dst[close])
    for _ in range(n_cliques):
        sz = int(rng.integers(clique_lo, clique_hi + 1))
        mem = rng.choice(n, size=sz, replace=False)
        a, b = np.triu_indices(sz, 1)
        us.append(mem[a])
        vs.append(mem[b])
    return _finish(n, np.concatenate(us), np.concatenate(vs), rng)


def chung_lu(n: int, exponent: float, mean_degree: float, max_degree: int, seed: int):
    """Power-law expected degrees d_i ~ (i + i0)^(-1/(exponent-1)), scaled to the
    mean and capped; edges by endpoint sampling proportional to d (fast Chung-Lu)."""
    rng = np.random.default_rng(seed)
    beta = 1.0 / (exponent - 1.0)
    i0 = 1.0
    d = (np.arange(n, dtype=np.float64) + i0) ** (-beta)
    for _ in range(50):
        d = d * (mean_degree / d.mean())
        d = np.minimum(d, max_degree)
        if abs(d.mean() - mean_degree) < 1e-6 * mean_degree:
            break
    m_target = int(round(n * mean_degree / 2))
    prob = d / d.sum()
    # A few extra draws compensate for the self-loops and duplicates removed.
    draws = int(m_target * 1.03) + 1000
    a = rng.choice(n, size=draws, p=prob)
    b = rng.choice(n, size=draws, p=prob)
    perm = rng.permutation(n)  # hubs at random ids, not at the front
    return _finish(n, perm[a], perm[b], rng)


# ------------------------------------------------------------------ files
def write_sparse(path: str, n: int, u, v, w, comment: str | None = None) -> None:
    """'n n E' + 1-based 'u v w' lines (MDP 'sparse' set, MaxBS loader)."""
    with open(path, "w") as f:
        if comment:
            f.write(f"% {comment}\n")
        f.write(f"{n} {n} {len(u)}\n")
        np.savetxt(f, np.stack([np.asarray(u) + 1, np.asarray(v) + 1, np.asarray(w)], 1), fmt="%d")


def write_maxbs(path: str, n: int, u, v, w) -> None:
    """Max Bisection loader format (GPU-MAXBS-CSR.cu:144-166): no comment lines."""
    write_sparse(path, n, u, v, w, comment=None)


def write_mdg(path: str, n: int, m: int, u, v, w) -> None:
    """'n m' + 0-based 'u v w' lines (MDG-a/b/c branch, GPU-MDP-CSR.cu:273-280)."""
    with open(path, "w") as f:
        f.write(f"{n} {m}\n")
        np.savetxt(f, np.stack([np.asarray(u), np.asarray(v), np.asarray(w)], 1), fmt="%d")


def _parse_weight_column(tokens):
    """Exact fixed-point parse of decimal weights; returns (int64 array, scale)."""
    decs = 0
    for t in tokens:
        if "." in t:
            decs = max(decs, len(t.split(".", 1)[1]))
    scale = 10 ** decs
    out = np.empty(len(tokens), np.int64)
    for k, t in enumerate(tokens):
        if "." in t:
            ip, fp = t.split(".", 1)
            neg = ip.startswith("-")
            ip = ip.lstrip("+-") or "0"
            val = int(ip) * scale + int((fp + "0" * decs)[:decs] or "0")
            out[k] = -val if neg else val
        else:
            out[k] = int(t) * scale
    return out, scale


def read_graph(path: str, fmt: str = "sparse"):
    """Reads a reference-format instance. fmt: 'sparse' (also the MaxBS format),
    'MDG' (0-based, header 'n m').  Returns (n, m_or_None, u, v, w, scale) where
    decimal weights are scaled to exact integers by 10^decimals."""
    with open(path) as f:
        lines = [ln for ln in f.read().splitlines()]
    it = iter(lines)
    header = None
    for ln in it:
        if ln.strip() and not ln.startswith("%"):
            header = ln.split()
            break
    if header is None:
        raise ValueError(f"{path}: empty instance")
    rows = [ln.split() for ln in it if ln.strip() and not ln.startswith("%")]
    if fmt == "MDG":
        n, m = int(header[0]), int(header[1])
        base = 0
    else:
        n, m = int(header[0]), None
        base = 1
    if rows:
        a = np.array([int(r[0]) for r in rows], np.int64) - base
        b = np.array([int(r[1]) for r in rows], np.int64) - base
        w, scale = _parse_weight_column([r[2] for r in rows])
    else:
        a = b = w = np.zeros(0, np.int64)
        scale = 1
    if np.any(np.abs(w) > 2**31 - 1):
        raise ValueError(f"{path}: weight does not fit int32 after scaling by {scale}")
    return n, m, a.astype(np.int32), b.astype(np.int32), w.astype(np.int32), scale


# ------------------------------------------------------------------ configs
def config1():
    """MDP CSR: ER n=2000, mean degree 20, seed 1; m=200, tenure 20, 10,000 iterations."""
    u, v, w, _ = erdos_renyi(2000, 20.0, seed=1)
    return dict(n=2000, u=u, v=v, w=w, m=200, tenure=20, iters=10000)


def config2(n: int = 100_000, seed: int = 2):
    """MaxBS, conflict-style: n=100k, mean degree ~60, 2000 cliques of 8-32; tenure 50, 2000 iterations."""
    u, v, w, _ = conflict_graph(n, 60.0, 2000 if n >= 100_000 else max(1, n // 50), 8, 32, seed=seed)
    return dict(n=n, u=u, v=v, w=w, tenure=50, iters=2000)


def config3(n: int = 200_000, seed: int = 3):
    """MDP large: Chung-Lu n=200k, exponent 2.3, mean 50, max 5000; m=2000, tenure 100, 500 iterations."""
    u, v, w, _ = chung_lu(n, 2.3, 50.0, 5000, seed=seed)
    return dict(n=n, u=u, v=v, w=w, m=2000 if n >= 200_000 else max(2, n // 100), tenure=100, iters=500)


def _mix(*xs: int) -> int:
    """Deterministic 32-bit hash of a few integers (splitmix64 finaliser)."""
    h = 0x9E3779B97F4A7C15
    for x in xs:
        h = (h ^ (x + 0x9E3779B97F4A7C15 + (h << 6) + (h >> 2))) & 0xFFFFFFFFFFFFFFFF
        h ^= h >> 30
        h = (h * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        h ^= h >> 27
        h = (h * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        h ^= h >> 31
    return int(h & 0x7FFFFFFF) or 1


def config4(instances: int = 4096, restarts: int = 8, iters: int = 5000, seed: int = 4,
            n_lo: int = 200, n_hi: int = 20000, first: int = 0):
    """Batched workload: `instances` Erdos-Renyi instances with n log-uniform in
    [n_lo, n_hi], mean degree U[5, 50], node weights U[1,1000]; even instances
    MDP with m = U[5%, 20%] n, odd ones Max Bisection; `restarts` seeded solves
    each (seed = hash(instance, restart)); `iters` iterations per solve.
    Instances [first, first + instances) of the sequence, so a bounded sample
    is a prefix of the full workload."""
    rng = np.random.default_rng(seed)
    out = []
    total = first + instances
    ns = np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), size=total)).astype(np.int64)
    degs = rng.uniform(5, 50, size=total)
    fr = rng.uniform(0.05, 0.20, size=total)
    for i in range(first, total):
        n = int(ns[i])
        u, v, w, _ = erdos_renyi(n, float(min(degs[i], n - 1)), _mix(seed, i))
        mdp = i % 2 == 0
        out.append(dict(index=i, n=n, u=u, v=v, w=w, problem="mdp" if mdp else "maxbs",
                        m=max(1, int(round(fr[i] * n))) if mdp else n // 2,
                        seeds=[_mix(i, r) for r in range(restarts)], iters=iters))
    return out


def config5_requests(count: int, seed: int = 5, n_lo: int = 1000, n_hi: int = 200_000):
    """Served workload requests: 70% MDP (Chung-Lu graph as config 3, m = n/100,
    tenure 100), 30% Max Bisection (conflict graph as config 2, tenure 50);
    n log-uniform in [n_lo, n_hi]; iteration budget U[1000, 10000]; every
    graph from a per-request seed."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi))))
        mdp = rng.random() < 0.7
        iters = int(rng.integers(1000, 10001))
        s = _mix(seed, i)
        if mdp:
            u, v, w, _ = chung_lu(n, 2.3, 50.0, min(5000, n - 1), s)
            out.append(dict(n=n, u=u, v=v, w=w, problem="mdp", m=max(2, n // 100), tenure=100,
                            iters=iters, seed=s))
        else:
            u, v, w, _ = conflict_graph(n, 60.0, max(1, 2000 * n // 100_000), 8, 32, s)
            out.append(dict(n=n, u=u, v=v, w=w, problem="maxbs", m=n // 2, tenure=50, iters=iters, seed=s))
    return out
