// sweep.cuh -- one tabu iteration as ONE kernel launch.
//
// Replaces, per iteration, the reference's calculateSwapGain / calculateMoveGain
// (src/mdp/GPU-MDP-CSR.cu:567-584, src/maxbisection/GPU-MAXBS-CSR.cu:337-353 and
// their five structure variants), cub::DeviceReduce::ArgMax + the 8-byte D2H
// copy (:651-652 / :450-451), updateVertexEdgeGain/updateMoveGain (:523-541 /
// :355-375, WSwap :524-562 / :367-409), updateSolution/finalizeMove
// (:544-553 / :377-399), best tracking (:671-674 / :469-476) and the MaxBS
// perturbation (:480-501).
//
// Each CTA owns a tile of R inside positions (rows) x chunk_cols outside
// positions (columns) of the m x (n-m) pair space.  It evaluates every pair's
// gain in 32-bit (or 64-bit) integers, applies the tabu/aspiration filter and
// keeps a per-row maximum; no gain array exists.  The CTA then resolves the
// lowest flat index achieving its maximum (the CUB ArgMax tie rule,
// cub/thread/thread_operators.cuh:103-121) by rescanning one row, and writes one
// (key, index) record.  The last CTA to finish reduces the records, decides the
// move and applies it -- so an iteration needs no host round trip.
//
// The fast pass only tracks allowed pairs (non-tabu, or aspirated).  When no
// allowed pair exists (or, for MDP, the best allowed gain is not above the
// -99999 sentinel), the last CTA switches the state to "exact" and the next
// launch re-evaluates every pair with the reference's full key rule (MDP
// sentinel, MaxBS float-quantised penalty) in int64.
#pragma once
#include <climits>
#include <cstdint>

#include "ts_internal.cuh"

namespace tsb {

constexpr int kSweepTPB = 256;
constexpr int kColsPerLane = 4;
constexpr int kPassCols = kSweepTPB * kColsPerLane;  // 1024 columns per pass

template <int ST> struct Rows { static constexpr int R = 16; };
template <> struct Rows<S_CSR> { static constexpr int R = 32; };
template <> struct Rows<S_BITSET> { static constexpr int R = 8; };
template <> struct Rows<S_BITSET_BB> { static constexpr int R = 8; };

template <class KeyT> struct KeyLim;
template <> struct KeyLim<int32_t> {
  static constexpr int32_t none = INT32_MIN;
  __device__ static int32_t clampD(long long d) {
    return d > INT32_MAX ? INT32_MAX : (d < INT32_MIN + 1 ? INT32_MIN + 1 : (int32_t)d);
  }
};
template <> struct KeyLim<long long> {
  static constexpr long long none = LLONG_MIN;
  __device__ static long long clampD(long long d) { return d; }
};

template <int PROB, class KeyT>
__device__ __forceinline__ KeyT pair_gain(KeyT rowv, KeyT colv, int32_t w) {
  if (PROB == P_MDP) return colv - rowv - (KeyT)w;  // vg[v] - vg[u] - w(u,v)
  return rowv + colv + (KeyT)2 * (KeyT)w;           // vg[u] + vg[v] + 2 w(u,v)
}

__device__ __forceinline__ bool allowed(bool row_tabu, bool col_tabu, long long x, long long D) {
  return !(row_tabu || col_tabu) || x > D;  // GPU-MDP-CSR.cu:580, GPU-MAXBS-CSR.cu:349
}

__device__ __forceinline__ int32_t warp_max(int32_t v) { return __reduce_max_sync(0xffffffffu, v); }
__device__ __forceinline__ long long warp_max(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    long long t = __shfl_xor_sync(0xffffffffu, v, o);
    v = t > v ? t : v;
  }
  return v;
}

__device__ __forceinline__ void better_rec(long long& k, long long& i, long long k2, long long i2) {
  if (k2 > k || (k2 == k && i2 < i)) { k = k2; i = i2; }
}

// Block-wide (key desc, index asc) reduction; result valid in thread 0.
__device__ __forceinline__ void block_best(long long& k, long long& i, CtaRec* scratch) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    long long k2 = __shfl_xor_sync(0xffffffffu, k, o);
    long long i2 = __shfl_xor_sync(0xffffffffu, i, o);
    better_rec(k, i, k2, i2);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) { scratch[warp].key = k; scratch[warp].idx = i; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) better_rec(k, i, scratch[w].key, scratch[w].idx);
  }
  __syncthreads();
}

// Column loads: 4 contiguous columns per lane (16 B aligned since ldc % 4 == 0).
__device__ __forceinline__ void load4(const int32_t* p, int32_t (&o)[4]) {
  int4 t = __ldg(reinterpret_cast<const int4*>(p));
  o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w;
}
__device__ __forceinline__ void load4(const long long* p, long long (&o)[4]) {
  longlong2 a = __ldg(reinterpret_cast<const longlong2*>(p));
  longlong2 b = __ldg(reinterpret_cast<const longlong2*>(p) + 1);
  o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}

// Per-row lookup data of the staged structures: generic pointers into shared
// memory (or global memory for rows past the staging budget).
struct RowDesc {
  const void* p;   // BB: CSR row; Hash: table; Bitset: bitmap words
  const int2* q;   // Bitset: CSR row (hit path)
  int32_t len;     // BB / Bitset: CSR degree
  uint32_t mask;   // Hash: capacity - 1
};

__device__ __forceinline__ int32_t bb_lower(const int2* a, int32_t len, int32_t v) {
  // Branch-free lower_bound; the trip count depends on len only (uniform per row).
  int32_t lo = 0;
  int32_t step = len > 0 ? (1 << (31 - __clz(len))) : 0;
  for (; step > 0; step >>= 1)
    if (lo + step <= len && a[lo + step - 1].x < v) lo += step;
  return (lo < len && a[lo].x == v) ? a[lo].y : 0;
}

__device__ __forceinline__ int32_t hash_probe(const int2* t, uint32_t mask, int32_t v) {
  uint32_t slot = fmix32((uint32_t)v) & mask;
  for (uint32_t k = 0; k <= mask; k++) {
    int2 e = t[slot];
    if (e.x == v) return e.y;
    if (e.x == kHashEmpty) return 0;
    slot = (slot + 1) & mask;
  }
  return 0;
}

__device__ __forceinline__ int32_t scan_first(const int2* a, int32_t len, int32_t v) {
  for (int32_t k = 0; k < len; k++)
    if (a[k].x == v) return a[k].y;
  return 0;
}

template <int ST>
__device__ __forceinline__ int32_t staged_lookup(const RowDesc& d, int32_t v) {
  if (ST == S_BB) return bb_lower(static_cast<const int2*>(d.p), d.len, v);
  if (ST == S_HASH) return hash_probe(static_cast<const int2*>(d.p), d.mask, v);
  // Bitset guard, then the CSR row on a hit (GPU-MDP-CSR-Bitset-BuscaBinaria.cu:598-604).
  const uint64_t* words = static_cast<const uint64_t*>(d.p);
  if (!((words[v >> 6] >> (v & 63)) & 1ull)) return 0;
  return ST == S_BITSET ? scan_first(d.q, d.len, v) : bb_lower(d.q, d.len, v);
}

// Generic global-memory lookup used by the exact pass.
template <int ST, class KeyT>
__device__ __forceinline__ int32_t global_lookup(const DevGraph& g, const DevSolver<KeyT>& s,
                                                 int32_t row, int32_t col, int32_t u, int32_t v) {
  if (ST == S_WSWAP) return s.W[(long long)row * s.ldc + col];
  const long long st = g.rowptr[u];
  const int32_t deg = (int32_t)(g.rowptr[u + 1] - st);
  if (ST == S_CSR) return scan_first(g.adj + st, deg, v);
  if (ST == S_BB) return bb_lower(g.adj + st, deg, v);
  if (ST == S_HASH) {
    const long long b = g.hoff[u];
    return hash_probe(g.htab + b, (uint32_t)(g.hoff[u + 1] - b - 1), v);
  }
  if (!((g.bits[(long long)u * g.wpr + (v >> 6)] >> (v & 63)) & 1ull)) return 0;
  return ST == S_BITSET ? scan_first(g.adj + st, deg, v) : bb_lower(g.adj + st, deg, v);
}

template <class KeyT>
__device__ __forceinline__ KeyT* vg_at(const DevSolver<KeyT>& s, int32_t p) {
  return p < s.m ? s.vg_in + p : s.vg_out + (p - s.m);
}

__device__ __forceinline__ void atomic_add_key(int32_t* a, int32_t d) { atomicAdd(a, d); }
__device__ __forceinline__ void atomic_add_key(long long* a, long long d) {
  atomicAdd(reinterpret_cast<unsigned long long*>(a), (unsigned long long)d);
}

// ------------------------------------------------------------------ tail
struct TailShared {
  CtaRec red[kSweepTPB / 32];
  long long key, idx;
  int32_t action;
  int32_t wuv;
};

// Applies one swap (tabu move or perturbation move) with the whole CTA.
// Returns (in thread 0) the perturbation gain aux read after the contribution
// update, before negation (finalizeMove GPU-MAXBS-CSR.cu:381-384).
template <int PROB, int ST, class KeyT>
__device__ long long apply_swap(const DevGraph& g, const DevSolver<KeyT>& s, int32_t iu, int32_t jv,
                                long long iter, int32_t t_u, int32_t t_v, bool set_tabu,
                                TailShared& sh) {
  const int32_t m = s.m;
  const int32_t u = s.sol_in[iu], v = s.sol_out[jv];
  const long long su = g.rowptr[u], sv = g.rowptr[v];
  const int32_t nu = (int32_t)(g.rowptr[u + 1] - su), nv = (int32_t)(g.rowptr[v + 1] - sv);
  if (threadIdx.x == 0) sh.wuv = 0;
  __syncthreads();
  for (int32_t k = threadIdx.x; k < nu + nv; k += blockDim.x) {
    const bool from_u = k < nu;
    const long long at = from_u ? su + k : sv + (k - nu);
    const long long rs = from_u ? su : sv;
    const int2 e = g.adj[at];
    const int32_t z = e.x, w = e.y;
    const int32_t p = s.pos[z];
    KeyT d;
    if (PROB == P_MDP) {
      d = from_u ? -(KeyT)w : (KeyT)w;
    } else {
      const bool z_in = p < m;
      d = (from_u == z_in) ? -(KeyT)2 * (KeyT)w : (KeyT)2 * (KeyT)w;
    }
    atomic_add_key(vg_at(s, p), d);
    if (ST == S_CSR) s.cpos[g.rev[at]] = from_u ? m + jv : iu;  // new position of u / v
    const bool first = at == rs || g.adj[at - 1].x != z;
    if (PROB == P_MAXBS && from_u && z == v && first) sh.wuv = w;
    if (ST == S_WSWAP && first && z != (from_u ? u : v)) {
      // Row iu now describes v, column jv now describes u
      // (updateVertexEdgeGain, GPU-MDP-WSwap.cu:535-560).  Self-loop entries
      // (kept by the MaxBS loader) are skipped: the reference's patch would fold
      // them into W[iu][jv], and W must keep returning the CSR lookup's w(u,v).
      if (from_u && z != v) {
        if (p >= m) atomicAdd(&s.W[(long long)iu * s.ldc + (p - m)], -w);
        else atomicAdd(&s.W[(long long)p * s.ldc + jv], w);
      } else if (!from_u && z != u) {
        if (p >= m) atomicAdd(&s.W[(long long)iu * s.ldc + (p - m)], w);
        else atomicAdd(&s.W[(long long)p * s.ldc + jv], -w);
      }
    }
  }
  __syncthreads();
  long long aux = 0;
  if (threadIdx.x == 0) {
    // L2 reads: the contributions were just changed by atomics, and this CTA's
    // sweep may hold older copies of them in L1.
    KeyT a = __ldcg(s.vg_in + iu), b = __ldcg(s.vg_out + jv);
    if (PROB == P_MAXBS) {
      aux = (long long)a + (long long)b - 2LL * sh.wuv;
      a = -a;
      b = -b;
    }
    s.vg_in[iu] = b;   // v now inside at iu
    s.vg_out[jv] = a;  // u now outside at jv
    s.sol_in[iu] = v;
    s.sol_out[jv] = u;
    s.pos[u] = m + jv;
    s.pos[v] = iu;
    if (set_tabu) {
      s.tab_out[jv] = (int32_t)(iter + t_u);
      s.tab_in[iu] = (int32_t)(iter + t_v);
    } else {
      int32_t t = s.tab_in[iu];
      s.tab_in[iu] = s.tab_out[jv];
      s.tab_out[jv] = t;
    }
    long long ln = s.st->log_n;
    if (ln < s.log_cap) s.movelog[ln] = make_int2(iu, jv);
    else s.st->err |= E_LOG_FULL;
    s.st->log_n = ln + 1;
  }
  __syncthreads();
  return aux;
}

template <class KeyT>
__device__ __forceinline__ void trace_rec(const DevSolver<KeyT>& s, long long iter, long long idx,
                                          long long key, int32_t kind, int32_t t1, int32_t t2) {
  DevState* st = s.st;
  long long tn = st->trace_n;
  if (s.trace && tn < s.trace_cap) {
    TraceRec r;
    r.iter = iter; r.idx = idx; r.key = key; r.cur = st->cur; r.best = st->best;
    r.kind = kind; r.tenure = t1; r.tenure2 = t2; r.pad = 0;
    s.trace[tn] = r;
  }
  st->trace_n = tn + 1;
}

// Decision + move application by the last CTA.
template <int PROB, int ST, class KeyT>
__device__ void iteration_tail(const DevGraph& g, const DevSolver<KeyT>& s, int mode, TailShared& sh) {
  DevState* st = s.st;
  long long k = LLONG_MIN, i = LLONG_MAX;
  const int nrec = gridDim.x;
  for (int b = threadIdx.x; b < nrec; b += blockDim.x) {
    const long long rk = __ldcg(&s.recs[b].key), ri = __ldcg(&s.recs[b].idx);
    better_rec(k, i, rk, ri);
  }
  block_best(k, i, sh.red);
  if (threadIdx.x == 0) {
    int action = 0;  // 0: switch to exact, 1: move, 2: MDP break
    if (mode == 0) {
      if (k != LLONG_MIN && (PROB == P_MAXBS || k > kMdpSentinel)) action = 1;
    } else {
      action = (PROB == P_MDP && k == kMdpSentinel) ? 2 : 1;
    }
    if (action != 0 && (i < 0 || i >= s.P)) {  // cannot happen; never index with it
      st->err |= E_BAD_INDEX;
      st->done = 1;
      action = 3;
    }
    sh.action = action;
    sh.key = k;
    sh.idx = i;
    st->mode = action == 0 ? 1 : 0;
    if (action == 2) {
      st->evaluations += s.P;
      st->done = 1;
      st->stopped = 1;
      trace_rec(s, st->iter, i, k, 1, 0, 0);
    }
  }
  __syncthreads();
  if (sh.action != 1) {
    if (threadIdx.x == 0) st->counter = 0;
    return;
  }
  const long long key = sh.key, idx = sh.idx;
  const long long iter = st->iter;
  const int32_t iu = (int32_t)(idx / s.delta), jv = (int32_t)(idx % s.delta);
  int32_t t_u, t_v, t2 = 0;
  if (PROB == P_MDP) {
    const int32_t c1 = s.tenure_policy == 0 ? mdp_ref_tenure(iter) : s.tenure;
    int32_t c2 = s.c2_fixed;
    if (s.tenure_policy == 0) c2 = s.c2_tab[c1 == 15 ? 0 : c1 == 30 ? 1 : c1 == 60 ? 2 : 3];
    t_u = c1;  // tab[u] = iter + C1 (GPU-MDP-CSR.cu:549)
    t_v = c2;  // tab[v] = iter + C2 (:550)
    t2 = c2;
  } else {
    const int32_t tt = s.tenure_policy == 0 ? maxbs_ref_tenure(iter, s.maxt) : s.tenure;
    t_u = tt;
    t_v = tt;
  }
  apply_swap<PROB, ST, KeyT>(g, s, iu, jv, iter, t_u, t_v, true, sh);
  if (threadIdx.x == 0) {
    long long cur = st->cur;
    if (PROB == P_MAXBS && key < kMaxbsRecoverBelow) cur += key + kMaxbsInf;  // :456-460
    else cur += key;
    st->cur = cur;
    st->evaluations += s.P;
    if (cur > st->best) {
      st->best = cur;
      st->best_log_n = st->log_n;
      st->isi = 0;
    } else {
      st->isi += 1;
    }
    trace_rec(s, iter, idx, key, 0, t_u, t2);
    st->iter = iter + 1;
    sh.action = (PROB == P_MAXBS && st->isi >= s.piter) ? 3 : 1;
  }
  __syncthreads();
  if (PROB == P_MAXBS && sh.action == 3) {
    const long long ev = st->pert_events - st->pert_base;
    if (ev < 0 || ev >= s.draw_events) {
      if (threadIdx.x == 0) { st->err |= E_PERTURB_WINDOW; st->done = 1; }
    } else {
      for (int32_t q = 0; q < s.num_pert; q++) {
        const long long mv = s.draws[ev * s.num_pert + q];
        const int32_t pu = (int32_t)(mv / s.delta), pv = (int32_t)(mv % s.delta);
        const long long aux = apply_swap<PROB, ST, KeyT>(g, s, pu, pv, iter + 1, 0, 0, false, sh);
        if (threadIdx.x == 0) {
          st->cur += aux;
          st->pert_moves += 1;
          trace_rec(s, iter + 1, mv, aux, 2, 0, 0);
        }
        __syncthreads();
      }
      if (threadIdx.x == 0) {
        st->pert_events += 1;
        st->isi = 0;
      }
    }
  }
  if (threadIdx.x == 0) st->counter = 0;
}

// ------------------------------------------------------------------ kernel
template <int PROB, int ST, class KeyT>
__global__ void __launch_bounds__(kSweepTPB)
iter_kernel(const DevGraph g, const DevSolver<KeyT> s) {
  constexpr int R = Rows<ST>::R;
  using Lim = KeyLim<KeyT>;
  DevState* st = s.st;
  if (st->done || st->iter >= st->target) return;
  const int mode = st->mode;
  const long long iter = st->iter;
  const long long D64 = st->best - st->cur;
  const KeyT D = Lim::clampD(D64);
  const int tid = threadIdx.x, lane = tid & 31;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ KeyT s_rv[R];
  __shared__ int32_t s_ru[R];
  __shared__ int32_t s_rtab[R];
  __shared__ KeyT s_rowbest[R];
  __shared__ RowDesc s_desc[R];
  __shared__ long long s_rstart[R];
  __shared__ int32_t s_off[R + 1];
  __shared__ TailShared sh;
  __shared__ int32_t s_last;
  __shared__ long long s_mc;
  __shared__ int32_t s_rstar;
  __shared__ uint32_t s_cmin;

  const int rb = blockIdx.x / s.n_chunks, ch = blockIdx.x % s.n_chunks;
  const int32_t r0 = rb * R;
  const int32_t nr = min(R, s.m - r0);
  const int32_t c0 = ch * s.chunk_cols;
  const int32_t c_end = min(c0 + s.chunk_cols, s.delta);

  if (tid < R) {
    const bool ok = tid < nr;
    s_rv[tid] = ok ? s.vg_in[r0 + tid] : (KeyT)0;
    s_ru[tid] = ok ? s.sol_in[r0 + tid] : 0;
    s_rtab[tid] = ok ? (s.tab_in[r0 + tid] > iter) : 0;
    s_rowbest[tid] = Lim::none;
  }
  __syncthreads();

  long long my_key = LLONG_MIN, my_idx = LLONG_MAX;

  if (mode == 1) {
    // ---------------- exact pass: the reference's full key rule, int64.
    for (int32_t r = 0; r < nr; r++) {
      const int32_t u = s_ru[r];
      const long long rv = (long long)s_rv[r];
      const bool rt = s_rtab[r] != 0;
      const long long base = (long long)(r0 + r) * s.delta;
      for (int32_t c = c0 + tid; c < c_end; c += blockDim.x) {
        const int32_t v = s.sol_out[c];
        const long long cv = (long long)s.vg_out[c];
        const bool ct = s.tab_out[c] > iter;
        const int32_t w = global_lookup<ST, KeyT>(g, s, r0 + r, c, u, v);
        const long long x = pair_gain<PROB, long long>(rv, cv, w);
        long long key = x;
        if (!allowed(rt, ct, x, D64)) key = PROB == P_MDP ? kMdpSentinel : maxbs_penalty(x);
        better_rec(my_key, my_idx, key, base + c);
      }
    }
    block_best(my_key, my_idx, sh.red);
  } else {
    // ---------------- fast pass
    uint32_t* s_mask = reinterpret_cast<uint32_t*>(smem_raw);  // CSR + MDP: adjacency per column
    if (ST == S_CSR) {
      if (PROB == P_MDP)
        for (int32_t c = tid; c < s.chunk_cols; c += blockDim.x) s_mask[c] = 0u;
      if (tid < 32) {
        // row segments and their prefix (one lane per row)
        long long a0 = 0;
        int32_t d = 0;
        if (lane < nr) {
          a0 = g.rowptr[s_ru[lane]];
          d = (int32_t)(g.rowptr[s_ru[lane] + 1] - a0);
          s_rstart[lane] = a0;
        }
        int32_t incl = d;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += t;
        }
        if (lane < R) s_off[lane + 1] = incl;
        if (lane == 0) s_off[0] = 0;
      }
    } else if (ST != S_WSWAP) {
      if (tid == 0) {
        long long off = 0;  // bytes used in the staging area, 16 B aligned
        for (int r = 0; r < R; r++) {
          RowDesc d;
          d.p = nullptr; d.q = nullptr; d.len = 0; d.mask = 0;
          if (r < nr) {
            const int32_t u = s_ru[r];
            const long long rs = g.rowptr[u];
            const int32_t deg = (int32_t)(g.rowptr[u + 1] - rs);
            d.len = deg;
            if (ST == S_BB) {
              d.p = g.adj + rs;
              const long long b = 8LL * deg;
              if (off + b <= s.stage_bytes) { d.p = smem_raw + off; off += (b + 15) & ~15LL; }
            } else if (ST == S_HASH) {
              const long long hb = g.hoff[u];
              const long long cap = g.hoff[u + 1] - hb;
              d.mask = (uint32_t)(cap - 1);
              d.p = g.htab + hb;
              const long long b = 8LL * cap;
              if (off + b <= s.stage_bytes) { d.p = smem_raw + off; off += (b + 15) & ~15LL; }
            } else {
              d.p = g.bits + (long long)u * g.wpr;
              d.q = g.adj + rs;
              const long long b = 8LL * g.wpr;
              if (off + b <= s.stage_bytes) { d.p = smem_raw + off; off += b; }
            }
          }
          s_desc[r] = d;
        }
        if (ST == S_BITSET || ST == S_BITSET_BB) {  // then the CSR rows for the hit path
          for (int r = 0; r < nr; r++) {
            const long long b = 8LL * s_desc[r].len;
            if (off + b <= s.stage_bytes) {
              s_desc[r].q = reinterpret_cast<const int2*>(smem_raw + off);
              off += (b + 15) & ~15LL;
            }
          }
        }
      }
    }
    __syncthreads();
    if (ST == S_CSR) {
      // Join the rows' CSR segments with the chunk by position: cpos[k] is the
      // current position of entry k's neighbour, so adjacent pairs of the tile
      // are found with contiguous reads.  They are evaluated exactly here; for
      // MDP they are also masked out of the sweep (their w-free gain would be
      // an over-estimate; for MaxBS it is an under-estimate and harmless).
      const int32_t total = s_off[nr];
      for (int32_t f = tid; f < total; f += blockDim.x) {
        int32_t lo = 0, hi = nr - 1;  // row r with s_off[r] <= f < s_off[r+1]
        while (lo < hi) {
          const int32_t mid = (lo + hi + 1) >> 1;
          if (s_off[mid] <= f) lo = mid; else hi = mid - 1;
        }
        const int32_t r = lo;
        const long long k = s_rstart[r] + (f - s_off[r]);
        const int32_t c = s.cpos[k] - s.m;
        if (c < c0 || c >= c_end) continue;
        const int2 e = g.adj[k];
        if (k > s_rstart[r] && g.adj[k - 1].x == e.x) continue;  // duplicate pair: first entry wins
        if (PROB == P_MDP) atomicOr(&s_mask[c - c0], 1u << r);
        const KeyT x = pair_gain<PROB, KeyT>(s_rv[r], s.vg_out[c], e.y);
        if (allowed(s_rtab[r] != 0, s.tab_out[c] > iter, (long long)x, (long long)D))
          atomicMax(&s_rowbest[r], x);
      }
    } else if (ST != S_WSWAP) {
      for (int r = 0; r < nr; r++) {
        const RowDesc d = s_desc[r];
        const int32_t u = s_ru[r];
        if (__isShared(d.p)) {
          long long words;
          const long long* src;
          if (ST == S_BB) { src = reinterpret_cast<const long long*>(g.adj + g.rowptr[u]); words = d.len; }
          else if (ST == S_HASH) { src = reinterpret_cast<const long long*>(g.htab + g.hoff[u]); words = (long long)d.mask + 1; }
          else { src = reinterpret_cast<const long long*>(g.bits + (long long)u * g.wpr); words = g.wpr; }
          long long* dst = reinterpret_cast<long long*>(const_cast<void*>(d.p));
          for (long long q = tid; q < words; q += blockDim.x) dst[q] = __ldg(src + q);
        }
        if ((ST == S_BITSET || ST == S_BITSET_BB) && __isShared(d.q)) {
          const long long* src = reinterpret_cast<const long long*>(g.adj + g.rowptr[u]);
          long long* dst = reinterpret_cast<long long*>(const_cast<int2*>(d.q));
          for (long long q = tid; q < d.len; q += blockDim.x) dst[q] = __ldg(src + q);
        }
      }
    }
    __syncthreads();

    KeyT best[R];
#pragma unroll
    for (int r = 0; r < R; r++) best[r] = Lim::none;

    const int passes = s.chunk_cols / kPassCols;
    for (int pass = 0; pass < passes; pass++) {
      const int32_t cb = c0 + (pass * kSweepTPB + tid) * kColsPerLane;
      if (cb >= c_end) break;
      KeyT cv[4];
      int32_t ct4[4];
      bool valid[4], ct[4];
      if (ST == S_WSWAP) {
        // Issue every row's W load of this pass before using any: the matrix
        // streams from HBM once per iteration.
        int4 wv[R];
#pragma unroll
        for (int r = 0; r < R; r++)
          wv[r] = __ldcs(reinterpret_cast<const int4*>(s.W + (long long)(r0 + r) * s.ldc + cb));
        load4(s.vg_out + cb, cv);
        load4(s.tab_out + cb, ct4);
#pragma unroll
        for (int q = 0; q < 4; q++) {
          valid[q] = cb + q < c_end;
          ct[q] = ct4[q] > iter;
        }
#pragma unroll
        for (int r = 0; r < R; r++) {
          const KeyT t = s_rv[r];
          const int32_t w4[4] = {wv[r].x, wv[r].y, wv[r].z, wv[r].w};
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const KeyT x = pair_gain<PROB, KeyT>(t, cv[q], w4[q]);
            if (valid[q] && (!ct[q] || x > D)) best[r] = x > best[r] ? x : best[r];
          }
        }
        continue;
      }
      load4(s.vg_out + cb, cv);
      load4(s.tab_out + cb, ct4);
#pragma unroll
      for (int q = 0; q < 4; q++) {
        valid[q] = cb + q < c_end;
        ct[q] = ct4[q] > iter;
      }
      if (ST == S_CSR) {
        uint32_t mk[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
          mk[q] = valid[q] ? (PROB == P_MDP ? s_mask[cb + q - c0] : 0u) : 0xffffffffu;
          if (valid[q] && ct[q]) {
            // Tabu column: a pair is allowed only when aspirated (gain > best - cur).
#pragma unroll
            for (int r = 0; r < R; r++)
              if (!(pair_gain<PROB, KeyT>(s_rv[r], cv[q], 0) > D)) mk[q] |= 1u << r;
          }
        }
        if ((mk[0] | mk[1] | mk[2] | mk[3]) == 0u) {
#pragma unroll
          for (int r = 0; r < R; r++) {
            const KeyT t = s_rv[r];
#pragma unroll
            for (int q = 0; q < 4; q++) {
              const KeyT x = pair_gain<PROB, KeyT>(t, cv[q], 0);
              best[r] = x > best[r] ? x : best[r];
            }
          }
        } else {
#pragma unroll
          for (int r = 0; r < R; r++) {
            const KeyT t = s_rv[r];
#pragma unroll
            for (int q = 0; q < 4; q++) {
              const KeyT x = pair_gain<PROB, KeyT>(t, cv[q], 0);
              if (!((mk[q] >> r) & 1u)) best[r] = x > best[r] ? x : best[r];
            }
          }
        }
      } else {
        int32_t vx[4];
        load4(s.sol_out + cb, vx);
#pragma unroll
        for (int r = 0; r < R; r++) {
          if (r >= nr) continue;
          const KeyT t = s_rv[r];
          const RowDesc d = s_desc[r];
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const int32_t w = staged_lookup<ST>(d, vx[q]);
            const KeyT x = pair_gain<PROB, KeyT>(t, cv[q], w);
            if (valid[q] && (!ct[q] || x > D)) best[r] = x > best[r] ? x : best[r];
          }
        }
      }
    }

    // Per-row block maximum.
#pragma unroll
    for (int r = 0; r < R; r++) {
      const KeyT v = warp_max(best[r]);
      if (lane == 0 && v != Lim::none) atomicMax(&s_rowbest[r], v);
    }
    __syncthreads();
    if (tid == 0) {
      long long mc = LLONG_MIN;
      int32_t rstar = -1;
      for (int r = 0; r < nr; r++) {
        const KeyT v = s_rowbest[r];
        if (v == Lim::none) continue;
        if (s_rtab[r] && !(v > D)) continue;  // tabu row: only aspirated pairs
        if ((long long)v > mc) { mc = (long long)v; rstar = r; }
      }
      s_mc = mc;
      s_rstar = rstar;
      s_cmin = 0xffffffffu;
    }
    __syncthreads();
    if (s_rstar >= 0) {
      // Rescan the winning row: lowest column whose allowed gain equals the maximum.
      const int32_t r = s_rstar;
      const KeyT target = (KeyT)s_mc;
      const KeyT t = s_rv[r];
      const bool rt = s_rtab[r] != 0;
      uint32_t cmin = 0xffffffffu;
      for (int32_t c = c0 + tid; c < c_end; c += blockDim.x) {
        int32_t w = 0;
        if (ST == S_CSR) {
          // adjacent pairs are matched below from the row's entries; for MaxBS
          // an adjacent pair's w-free gain can never equal the row maximum.
          if (PROB == P_MDP && ((s_mask[c - c0] >> r) & 1u)) continue;
        } else if (ST == S_WSWAP) {
          w = s.W[(long long)(r0 + r) * s.ldc + c];
        } else {
          w = staged_lookup<ST>(s_desc[r], s.sol_out[c]);
        }
        const KeyT x = pair_gain<PROB, KeyT>(t, s.vg_out[c], w);
        if (x == target && allowed(rt, s.tab_out[c] > iter, (long long)x, (long long)D)) {
          cmin = (uint32_t)c;
          break;
        }
      }
      if (ST == S_CSR) {
        const long long a0 = s_rstart[r], a1 = a0 + (s_off[r + 1] - s_off[r]);
        for (long long k = a0 + tid; k < a1; k += blockDim.x) {
          const int32_t c = s.cpos[k] - s.m;
          if (c < c0 || c >= c_end) continue;
          const int2 e = g.adj[k];
          if (k > a0 && g.adj[k - 1].x == e.x) continue;
          const KeyT x = pair_gain<PROB, KeyT>(t, s.vg_out[c], e.y);
          if (x == target && allowed(rt, s.tab_out[c] > iter, (long long)x, (long long)D) &&
              (uint32_t)c < cmin)
            cmin = (uint32_t)c;
        }
      }
      cmin = __reduce_min_sync(0xffffffffu, cmin);
      if (lane == 0 && cmin != 0xffffffffu) atomicMin(&s_cmin, cmin);
      __syncthreads();
      if (tid == 0 && s_cmin != 0xffffffffu) {
        my_key = s_mc;
        my_idx = (long long)(r0 + r) * s.delta + s_cmin;
      }
    }
  }

  if (tid == 0) {
    CtaRec rec;
    rec.key = my_key;
    rec.idx = my_idx;
    s.recs[blockIdx.x] = rec;
    __threadfence();
    const unsigned prev = atomicAdd(&st->counter, 1u);
    s_last = prev == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  iteration_tail<PROB, ST, KeyT>(g, s, mode, sh);
}

}  // namespace tsb
