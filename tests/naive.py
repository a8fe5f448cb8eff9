"""Independent pure-Python restatement of the reference tabu loops, for tiny
instances only.  It cross-checks the C++ oracle (a second, line-by-line
reading of src/mdp/GPU-MDP-CSR.cu:611-693 and
src/maxbisection/GPU-MAXBS-CSR.cu:401-512); it is test code.
"""
from __future__ import annotations

import math
import struct


def f32(x: float) -> float:
    return struct.unpack("f", struct.pack("f", x))[0]


def csr(n, edges, drop_self):
    rows = [[] for _ in range(n)]
    for (a, b, w) in edges:
        if drop_self and a == b:
            continue
        rows[a].append((b, w))
        rows[b].append((a, w))
    for r in rows:
        r.sort(key=lambda e: e[0])  # Python's sort is stable
    return rows


def lookup(rows, u, v):
    for (z, w) in rows[u]:
        if z == v:
            return w
    return 0


def mdp_tenure(it):
    t = it % 1500
    if 700 < t <= 800:
        return 120
    if 300 < t <= 400 or 1100 < t <= 1200:
        return 60
    if 100 < t <= 200 or 500 < t <= 600 or 900 < t <= 1000 or 1300 < t <= 1400:
        return 30
    return 15


def c2_of(c1):
    x = 0.7 * c1
    return int(math.floor(x + 0.5))  # round half away from zero (x > 0)


def maxbs_tenure(it, maxt):
    b = [1, 2, 1, 4, 1, 2, 1, 8, 1, 2, 1, 4, 1, 2, 1]
    period = 16 * maxt
    q = it - 1
    rem = int(math.fmod(q, period))  # C++ % truncates toward zero
    x = rem + 1
    pos = 1
    for bi in b:
        ten = (maxt * bi) // 8
        length = 4 * ten
        if x < pos + length:
            return ten
        pos += length
    return maxt // 8


def penalty(g):
    # float(double(-9999999999) + g)
    return int(f32(float(-9999999999 + g)))


def run_mdp(n, edges, m, init, iters, tenure_fixed=None):
    rows = csr(n, edges, True)
    inside = set(init)
    sol = sorted(inside) + sorted(set(range(n)) - inside)
    pos = {v: i for i, v in enumerate(sol)}
    vg = [0] * n
    for a in sol[:m]:
        for (z, w) in rows[a]:
            vg[z] += w
    cur = sum(w for a in sol[:m] for (z, w) in rows[a] if z in inside) // 2
    best = cur
    tab = [0] * n
    delta = n - m
    trace = []
    it = 0
    while it < iters:
        bk, bi = None, None
        for i in range(m):
            u = sol[i]
            for j in range(m, n):
                v = sol[j]
                g = vg[v] - vg[u] - lookup(rows, u, v)
                allowed = not (tab[u] > it or tab[v] > it) or cur + g > best
                key = g if allowed else -99999
                idx = i * delta + (j - m)
                if bk is None or key > bk:
                    bk, bi = key, idx
        if bk == -99999:
            trace.append((it, bi, bk, "break"))
            break
        cur += bk
        c1 = tenure_fixed if tenure_fixed is not None else mdp_tenure(it)
        c2 = c2_of(c1)
        iu, iv = bi // delta, bi % delta + m
        u, v = sol[iu], sol[iv]
        for (z, w) in rows[u]:
            vg[z] -= w
        for (z, w) in rows[v]:
            vg[z] += w
        sol[iu], sol[iv] = v, u
        tab[u] = it + c1
        tab[v] = it + c2
        pos[u], pos[v] = iv, iu
        if cur > best:
            best = cur
        trace.append((it, bi, bk, cur, best))
        it += 1
    return trace, cur, best


def run_maxbs(n, edges, part, iters, draws, piter, tenure_fixed=None, maxt=200):
    """draws: list of perturbation events (lists of flat indices)."""
    rows = csr(n, edges, False)
    m = n // 2
    delta = n - m
    sol = [v for v in range(n) if part[v] == 0] + [v for v in range(n) if part[v] == 1]
    pos = {v: i for i, v in enumerate(sol)}
    side = list(part)
    vg = [0] * n
    for a in range(n):
        same = sum(w for (z, w) in rows[a] if side[z] == side[a])
        opp = sum(w for (z, w) in rows[a] if side[z] != side[a])
        vg[a] = same - opp
    cur = sum(w for a in range(n) for (z, w) in rows[a] if z > a and side[z] != side[a])
    best = cur
    tab = [0] * n
    trace = []
    it = 0
    isi = 0
    ev = 0

    def apply(iu, iv, tt, set_tabu):
        u, v = sol[iu], sol[iv]
        for (z, w) in rows[u]:
            if pos[z] < m:
                vg[z] -= 2 * w
            else:
                vg[z] += 2 * w
        for (z, w) in rows[v]:
            if pos[z] >= m:
                vg[z] -= 2 * w
            else:
                vg[z] += 2 * w
        aux = vg[u] + vg[v] - 2 * lookup(rows, u, v)
        vg[u], vg[v] = -vg[u], -vg[v]
        sol[iu], sol[iv] = v, u
        pos[u], pos[v] = iv, iu
        if set_tabu:
            tab[u] = it + tt
            tab[v] = it + tt
        return aux

    while it < iters:
        bk, bi = None, None
        for i in range(m):
            u = sol[i]
            for j in range(m, n):
                v = sol[j]
                g = vg[u] + vg[v] + 2 * lookup(rows, u, v)
                allowed = not (tab[u] > it or tab[v] > it) or cur + g > best
                key = g if allowed else penalty(g)
                idx = i * delta + (j - m)
                if bk is None or key > bk:
                    bk, bi = key, idx
        cur += bk + 9999999999 if bk <= -2500000000 else bk
        tt = tenure_fixed if tenure_fixed is not None else maxbs_tenure(it, maxt)
        apply(bi // delta, bi % delta + m, tt, True)
        if cur > best:
            best = cur
            isi = 0
        else:
            isi += 1
        trace.append((it, bi, bk, cur, best))
        it += 1
        if isi >= piter:
            for mv in draws[ev]:
                aux = apply(mv // delta, mv % delta + m, 0, False)
                cur += aux
                trace.append((it, mv, aux, cur, best))
            ev += 1
            isi = 0
    return trace, cur, best
