// packed.cuh -- one solve per CTA cluster: the start state, the iteration
// loop and the result of a solve whose state lives in a slot of HBM.  Shared
// by the batched form (batch.cu) and the server (serve.cu).
#pragma once
#include <cooperative_groups.h>

#include "sweep.cuh"

namespace tsb {

struct BatchResultDev {
  long long iterations, evaluations, cur, best, best_true, perturbations;
  int32_t stopped, err;
  int32_t complete, pad;  // complete: written when the solve has ended
};

__device__ __forceinline__ long long block_sum(long long v, long long* sc) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sc[threadIdx.x >> 5] = v;
  __syncthreads();
  long long t = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sc[w];
  __syncthreads();
  return t;
}

// Start state of a solve in its slot, by one CTA: ascending ids per side
// (initialSolution, GPU-MDP-CSR.cu:479-500), contributions and objective
// (calculateVertexGain :502-519; computeGainsFromScratch /
// computeFitnessFromScratch, GPU-MAXBS-CSR.cu:197-219), WSwap matrix
// (calculateEdgeGain, GPU-MDP-WSwap.cu:607-626) and CSR neighbour positions.
// The same values as the plain solver's init kernels.
template <int PROB, int ST, class KeyT>
__device__ void slot_init(const DevGraph& g, const DevSolver<KeyT>& s, const int32_t* init,
                          long long max_iter, long long* sc, int32_t* s_cnt) {
  const int tid = threadIdx.x, T = blockDim.x;
  const int32_t n = s.n, m = s.m;
  int32_t* flag = s.pos;  // inside flags first, positions afterwards
  for (int32_t v = tid; v < n; v += T) flag[v] = PROB == P_MDP ? 0 : (init[v] == 0);
  __syncthreads();
  if (PROB == P_MDP)
    for (int32_t i = tid; i < m; i += T) flag[init[i]] = 1;
  __syncthreads();
  const int32_t per = (n + T - 1) / T, a0 = min(n, tid * per), a1 = min(n, a0 + per);
  int32_t cnt = 0;
  for (int32_t v = a0; v < a1; v++) cnt += flag[v];
  s_cnt[tid] = cnt;
  __syncthreads();
  int32_t x = 0;
  for (int t2 = 0; t2 < tid; t2++) x += s_cnt[t2];
  int32_t y = a0 - x;
  for (int32_t v = a0; v < a1; v++) {
    if (flag[v]) { s.sol_in[x] = v; flag[v] = x; x++; }
    else { s.sol_out[y] = v; flag[v] = m + y; y++; }
  }
  for (int32_t j = s.delta + tid; j < s.ldc; j += T) s.sol_out[j] = 0;
  for (int32_t i = tid; i < m; i += T) { s.vg_in[i] = 0; s.tab_in[i] = 0; }
  for (int32_t j = tid; j < s.ldc; j += T) { s.vg_out[j] = 0; s.tab_out[j] = 0; }
  if (ST == S_WSWAP)
    for (long long q = tid; q < (long long)s.n_row_blocks * Rows<ST>::R * s.ldc; q += T) w_set(s, q, 0);
  __syncthreads();
  long long acc = 0;
  if (PROB == P_MDP) {
    for (int32_t i = 0; i < m; i++) {
      const int32_t u = s.sol_in[i];
      for (long long k = g.rowptr[u] + tid; k < g.rowptr[u + 1]; k += T) {
        const int2 e = g.adj[k];
        const int32_t p = s.pos[e.x];
        atomic_add_key(vg_at(s, p), (KeyT)e.y);
        if (p < m) acc += e.y;
      }
    }
  } else {
    for (int32_t z = tid; z < n; z += T) {
      const int32_t pz = s.pos[z];
      const bool side = pz < m;
      long long same = 0, opp = 0;
      for (long long k = g.rowptr[z]; k < g.rowptr[z + 1]; k++) {
        const int2 e = g.adj[k];
        if ((s.pos[e.x] < m) == side) {
          same += e.y;
        } else {
          opp += e.y;
          if (e.x > z) acc += e.y;
        }
      }
      *vg_at(s, pz) = (KeyT)(same - opp);
    }
  }
  if (ST == S_CSR)
    for (long long k = tid; k < g.entries; k += T) s.cpos[k] = s.pos[g.adj[k].x];
  if (ST == S_WSWAP) {
    for (int32_t i = 0; i < m; i++) {
      const int32_t u = s.sol_in[i];
      const long long k0 = g.rowptr[u];
      for (long long k = k0 + tid; k < g.rowptr[u + 1]; k += T) {
        const int2 e = g.adj[k];
        if (k > k0 && g.adj[k - 1].x == e.x) continue;  // first entry of a duplicated pair
        const int32_t p = s.pos[e.x];
        if (p >= m) w_set(s, (long long)i * s.ldc + (p - m), e.y);
      }
    }
  }
  long long obj = block_sum(acc, sc);
  if (PROB == P_MDP) obj /= 2;
  if (tid == 0) {
    DevState z;
    memset(&z, 0, sizeof(z));
    z.cur = obj;
    z.best = obj;
    z.target = max_iter;
    z.pert_limit = s.draw_events;  // every event of the solve is staged
    *s.st = z;
  }
  __syncthreads();
}

// Best solution (the current one with the moves after the last improvement
// undone; a swap is its own inverse), its objective from the graph, result.
template <int PROB, class KeyT>
__device__ void slot_finish(const DevGraph& g, const DevSolver<KeyT>& s, BatchResultDev* out,
                            int32_t* best_out, long long* sc) {
  const int tid = threadIdx.x, T = blockDim.x;
  const DevState* st = s.st;
  if (tid == 0) {
    const long long to = min(__ldcg(&st->log_n), s.log_cap);
    const long long from = __ldcg(&st->best_log_n);
    for (long long q = to - 1; q >= from; q--) {
      const int2 mv = s.movelog[q];
      const int32_t a = s.sol_in[mv.x];
      s.sol_in[mv.x] = s.sol_out[mv.y];
      s.sol_out[mv.y] = a;
    }
  }
  __syncthreads();
  for (int32_t v = tid; v < s.n; v += T) s.pos[v] = 0;
  __syncthreads();
  for (int32_t i = tid; i < s.m; i += T) s.pos[s.sol_in[i]] = 1;
  __syncthreads();
  long long acc = 0;
  for (int32_t a = tid; a < s.n; a += T) {
    const int32_t fa = s.pos[a];
    for (long long k = g.rowptr[a]; k < g.rowptr[a + 1]; k++) {
      const int2 e = g.adj[k];
      const int32_t fz = s.pos[e.x];
      if (PROB == P_MDP) {
        if (fa && fz) acc += e.y;
      } else if (e.x > a && fa != fz) {
        acc += e.y;
      }
    }
  }
  long long bt = block_sum(acc, sc);
  if (PROB == P_MDP) bt /= 2;
  if (PROB == P_MDP)
    for (int32_t i = tid; i < s.m; i += T) best_out[i] = s.sol_in[i];
  else
    for (int32_t v = tid; v < s.n; v += T) best_out[v] = s.pos[v] ? 0 : 1;
  if (tid == 0) {
    BatchResultDev r;
    r.iterations = __ldcg(&st->iter);
    r.evaluations = __ldcg(&st->evaluations);
    r.cur = __ldcg(&st->cur);
    r.best = __ldcg(&st->best);
    r.best_true = bt;
    r.perturbations = __ldcg(&st->pert_moves);
    r.stopped = __ldcg(&st->stopped);
    r.err = __ldcg(&st->err);
    r.complete = 1;
    *out = r;
  }
  __syncthreads();
}


// Runs a solve's iterations up to `stop_at` with the CTAs of the calling
// cluster: round-robin tiles, the leader merges the records over distributed
// shared memory and applies the move.  Every CTA of the cluster calls it.
template <int PROB, int ST, class KeyT>
__device__ void cluster_iterate(const DevGraph& g, const DevSolver<KeyT>& s, long long stop_at,
                                cooperative_groups::cluster_group& cl, TailShared& sh, CtaRec& s_rec) {
  const unsigned rank = cl.block_rank(), cs = cl.num_blocks();
  const int tid = threadIdx.x;
  const int ntiles = s.n_row_blocks * s.n_chunks;
  const DevState* st = s.st;
  for (;;) {
    // every CTA reads the same state: the leader wrote it before the last barrier
    const long long it = __ldcg(&st->iter);
    if (__ldcg(&st->done) || it >= stop_at) break;
    const int mode = __ldcg(&st->mode);
    const long long D64 = __ldcg(&st->best) - __ldcg(&st->cur);
    long long k = LLONG_MIN, i = LLONG_MAX;
    for (int t = (int)rank; t < ntiles; t += (int)cs) {
      long long tk, ti;
      // k (valid in thread 0, the thread that uses it): the CTA's best so far
      tile_eval<PROB, ST, KeyT, true>(g, s, mode, it, D64, t / s.n_chunks, t % s.n_chunks, tk, ti, sh,
                                      mode == 0 ? k : LLONG_MIN);
      if (tid == 0) better_rec(k, i, tk, ti);
    }
    if (tid == 0) { s_rec.key = k; s_rec.idx = i; }
    cl.sync();
    if (rank == 0) {
      if (tid == 0)
        for (unsigned r = 1; r < cs; r++) {
          const CtaRec* o = cl.map_shared_rank(&s_rec, r);
          better_rec(k, i, o->key, o->idx);
        }
      decide_apply<PROB, ST, KeyT>(g, s, mode, k, i, sh);
      __threadfence();
    }
    cl.sync();
  }
}

}  // namespace tsb
