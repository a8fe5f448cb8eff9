// solver.cu -- tabu-search state on the device and the host step loop.
//
// Replaces tabu_search (src/mdp/GPU-MDP-CSR.cu:611-693) and
// perturbationBasedTabuSearch (src/maxbisection/GPU-MAXBS-CSR.cu:401-512): their
// host-side init (initialSolution / calculateVertexGain / computeGainsFromScratch,
// GPU-MDP-CSR.cu:479-519, GPU-MAXBS-CSR.cu:197-219,307-324) runs here as device
// kernels, and the per-iteration host loop (4-5 launches + a blocking 8-byte D2H
// per iteration) becomes back-to-back launches of one iteration kernel whose
// state lives in HBM (sweep.cuh).  The host only touches the device between
// batches of iterations.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <random>
#include <string>
#include <unordered_set>
#include <vector>

#include "sweep.cuh"
#include "ts_host.h"

namespace tsb {

// glibc's rand() after srand(seed): random_r over the 128-byte TYPE_3 state,
// the generator the MDP start uses (GPU-MDP-CSR.cu:777, seeded at :1248),
// kept private so the library never touches the process-wide rand() state.
struct GlibcRand {
  struct random_data rd;
  char state[128];
  explicit GlibcRand(unsigned seed) {
    std::memset(&rd, 0, sizeof(rd));
    std::memset(state, 0, sizeof(state));
    initstate_r(seed, state, sizeof(state), &rd);
  }
  int next() {
    int32_t r = 0;
    random_r(&rd, &r);
    return r;
  }
};

// One perturbation event: k distinct flat move indices (GPU-MAXBS-CSR.cu:481-492).
void draw_event(std::mt19937& rng, int64_t P, int k, std::vector<long long>& out) {
  std::unordered_set<long long> used;
  for (int q = 0; q < k; q++) {
    long long mv;
    do {
      if (P - 1 <= INT32_MAX) {
        std::uniform_int_distribution<int> d(0, (int)(P - 1));
        mv = d(rng);
      } else {  // past the reference's int range (it overflows there)
        std::uniform_int_distribution<long long> d(0, P - 1);
        mv = d(rng);
      }
    } while (used.count(mv));
    used.insert(mv);
    out.push_back(mv);
  }
}

void mdp_random_set(int32_t n, int32_t m, uint32_t seed, std::vector<int32_t>& ids) {
  GlibcRand r(seed);
  std::vector<uint8_t> used(n, 0);
  ids.clear();
  while ((int32_t)ids.size() < m) {
    int32_t idx = r.next() % n;
    if (!used[idx]) { used[idx] = 1; ids.push_back(idx); }
  }
}

void maxbs_random_part(std::mt19937& rng, int32_t n, std::vector<uint8_t>& side0) {
  std::vector<int> vertices(n);
  for (int32_t i = 0; i < n; i++) vertices[i] = i;
  std::shuffle(vertices.begin(), vertices.end(), rng);  // randomPartition :187-195
  side0.assign(n, 0);
  for (int32_t i = 0; i < n / 2; i++) side0[vertices[i]] = 1;
}

int32_t staging_bytes(const ts_graph* g, int R) {
  // Sized for rows up to the 90th-percentile degree (larger rows are read
  // from global memory), so small rows do not cost occupancy.
  if (g->deg90 < 0) {
    const int32_t n = g->n;
    std::vector<int64_t> deg(n);
    for (int32_t r = 0; r < n; r++) deg[r] = g->h_rowptr[r + 1] - g->h_rowptr[r];
    std::nth_element(deg.begin(), deg.begin() + (int64_t)n * 9 / 10, deg.end());
    g->deg90 = std::max<int64_t>(1, deg[(int64_t)n * 9 / 10]);
  }
  const int64_t d90 = g->deg90;
  auto r16 = [](int64_t b) { return (b + 15) & ~15LL; };
  int64_t slots = d90;  // keys + weights of one row
  if (g->kind == S_HASH) slots = hash_capacity(d90);
  int64_t row_bytes = 2 * r16(4 * slots);
  if (g->kind == S_BB || g->kind == S_BITSET_BB) {  // + bucket directory
    int64_t nb = 16;
    while (nb < 2 * d90 && nb < 4096) nb <<= 1;
    row_bytes += r16(4 * (nb + 1));
  }
  if (g->kind == S_BITSET || g->kind == S_BITSET_BB) row_bytes += 8 * g->wpr;  // bitmap row
  const int64_t cap = (g->kind == S_BITSET || g->kind == S_BITSET_BB) ? 216 * 1024 : 96 * 1024;
  const int64_t head = g->kind == S_BB ? 16LL * R : 0;  // CSR+BB: compact row descriptors
  return (int32_t)std::min<int64_t>(cap, std::max<int64_t>(8 * 1024, head + R * row_bytes));
}

bool wswap_w16(const ts_graph* g) { return g->max_abs_w <= 32767; }

// CTAs per tile of the plain kernel's fast pass.  A tile's work units are its
// index groups (rows whose entries fit one index) and its heavy rows (more
// entries than an index holds); at most the graph's 32 largest degrees share
// a tile.  When those would make several units, each tile gets up to half
// that many CTAs, so a tile that collects hub rows (MDP moves hubs into the
// solution early) runs its units side by side; slices of a tile without that
// many units only read their rows' degrees and return.  The cap per
// structure is the measured best on the Chung-Lu graph (n = 200,000, degrees
// to 4,800; caps 2, 3, 4, 6 and 8 timed): Hash and CSR+Bitset 4, CSR+BB 3,
// CSR+Bitset+BB 2 -- the structures with the cheaper sweeps lose more to the
// slices without work.
int32_t tile_slices(const ts_graph* g, const TileGeom& t) {
  if (!t.fast || g->kind == S_CSR || t.fast_ecap <= 0 || g->h_rowptr.size() < 2) return 1;
  const size_t n = g->h_rowptr.size() - 1;
  std::vector<int64_t> deg(n);
  for (size_t i = 0; i < n; i++) deg[i] = g->h_rowptr[i + 1] - g->h_rowptr[i];
  const size_t k = std::min<size_t>(kFastRows, n);
  std::partial_sort(deg.begin(), deg.begin() + k, deg.end(), std::greater<int64_t>());
  int64_t heavy = 0, light = 0;
  for (size_t i = 0; i < k; i++) {
    if (deg[i] > t.fast_ecap) heavy++;
    else light += deg[i];
  }
  const int64_t units = heavy + (light + t.fast_ecap - 1) / t.fast_ecap;
  const int64_t cap = g->kind == S_BB ? 3 : (g->kind == S_BITSET_BB ? 2 : 4);
  return (int32_t)std::max<int64_t>(1, std::min<int64_t>(cap, (units + 1) / 2));
}

TileGeom tile_geometry(const ts_graph* g, int32_t problem, int32_t m, bool wide, int64_t min_tiles,
                       int32_t pass, bool persist) {
  TileGeom t;
  const int kind = g->kind;
  const int64_t delta = (int64_t)g->n - m;
  int32_t ecap = 0;
  if (!wide && kind != S_WSWAP && kind != S_CSR) {
    // two 512-thread CTAs per SM: ~104 KB of index each
    ecap = fast_ecap_for(kind, g->wpr, 104 * 1024);
  }
  // Below ~4 million pairs an iteration is a chain of latencies, and the
  // per-row pass's smaller tiles spread it over more SMs.  CSR with the
  // adjacency mask (MDP, or a negative weight) stays on the per-row pass: its
  // join already marks the adjacent pairs, and on the Chung-Lu graph (n =
  // 200,000, m = 2,000) it is ~30% faster than the tile pass once hubs are
  // inside.
  const bool masked_csr = kind == S_CSR && (problem == P_MDP || g->neg_w);
  const bool want_tile = pass == TS_PASS_TILE ||
                         (pass == TS_PASS_AUTO && !masked_csr && (int64_t)m * delta >= (1LL << 22));
  t.fast = (want_tile && !wide && kind != S_WSWAP && (kind == S_CSR || ecap > 0)) ? 1 : 0;
  t.fast_ecap = t.fast ? ecap : 0;
  t.rows = t.fast ? kFastRows : rows_of(kind);
  t.n_row_blocks = (int32_t)((m + t.rows - 1) / t.rows);
  const bool mdp_csr = masked_csr;
  t.adj_mask = mdp_csr ? 1 : 0;
  const int64_t pc = pass_cols_of(kind, persist);
  const int64_t full = ((delta + pc - 1) / pc) * pc;
  int64_t max_cols = full;
  if (kind == S_WSWAP) max_cols = 8 * pc;
  if (mdp_csr) max_cols = 16 * pc;  // the per-column mask stays within 64 KB
  if (t.fast && kind != S_CSR) {
    // a heavy row's column bitmap reuses the index memory: 8 columns per byte
    const int64_t fit = (int64_t)fast_layout(kind, ecap, g->wpr).total * 8;
    max_cols = std::max<int64_t>(pc, std::min<int64_t>(max_cols, (fit / pc) * pc));
  }
  const int64_t want_chunks = std::max<int64_t>(1, (min_tiles + t.n_row_blocks - 1) / t.n_row_blocks);
  int64_t cols = (delta + want_chunks - 1) / want_chunks;
  cols = ((cols + pc - 1) / pc) * pc;
  cols = std::max<int64_t>(pc, std::min<int64_t>(cols, max_cols));
  t.chunk_cols = (int32_t)cols;
  t.n_chunks = (int32_t)((delta + cols - 1) / cols);
  t.stage_bytes = 0;
  if (kind == S_CSR) {
    t.smem = mdp_csr ? sizeof(uint32_t) * (size_t)cols : 16;
  } else if (kind == S_WSWAP) {
    t.smem = 16;
  } else if (t.fast) {
    t.smem = fast_layout(kind, ecap, g->wpr).total;
  } else {
    t.stage_bytes = staging_bytes(g, t.rows);
    t.smem = (size_t)t.stage_bytes;
  }
  return t;
}

namespace {

constexpr int kInitTPB = 256;

inline int grid_for(int64_t n, int tpb = kInitTPB) {
  int64_t b = (n + tpb - 1) / tpb;
  if (b < 1) b = 1;
  if (b > 148 * 32) b = 148 * 32;
  return (int)b;
}

template <class KeyT>
__global__ void k_init_mdp(const DevGraph g, const DevSolver<KeyT> s, unsigned long long* obj2) {
  // calculateVertexGain (GPU-MDP-CSR.cu:502-519): vg[z] += w for z in N(S).
  for (int32_t i = blockIdx.x; i < s.m; i += gridDim.x) {
    const int32_t u = s.sol_in[i];
    unsigned long long acc = 0;
    for (long long k = g.rowptr[u] + threadIdx.x; k < g.rowptr[u + 1]; k += blockDim.x) {
      const int2 e = g.adj[k];
      const int32_t p = s.pos[e.x];
      atomic_add_key(vg_at(s, p), (KeyT)e.y);
      if (p < s.m) acc += (unsigned long long)(long long)e.y;
    }
    if (acc) atomicAdd(obj2, acc);
  }
}

template <class KeyT>
__global__ void k_init_maxbs(const DevGraph g, const DevSolver<KeyT> s, unsigned long long* cut) {
  // computeGainsFromScratch / computeFitnessFromScratch (GPU-MAXBS-CSR.cu:197-219).
  for (int32_t z = blockIdx.x * blockDim.x + threadIdx.x; z < s.n; z += gridDim.x * blockDim.x) {
    const int32_t pz = s.pos[z];
    const bool side = pz < s.m;
    long long same = 0, opp = 0;
    unsigned long long c = 0;
    for (long long k = g.rowptr[z]; k < g.rowptr[z + 1]; k++) {
      const int2 e = g.adj[k];
      const bool sy = s.pos[e.x] < s.m;
      if (sy == side) same += e.y;
      else {
        opp += e.y;
        if (e.x > z) c += (unsigned long long)(long long)e.y;
      }
    }
    *vg_at(s, pz) = (KeyT)(same - opp);
    if (c) atomicAdd(cut, c);
  }
}

// W[i][j] = w(sol_in[i], sol_out[j]) (calculateEdgeGain, GPU-MDP-WSwap.cu:607-626),
// first entry of a duplicated pair.
template <class KeyT>
__global__ void k_init_wswap(const DevGraph g, const DevSolver<KeyT> s) {
  for (int32_t i = blockIdx.x; i < s.m; i += gridDim.x) {
    const int32_t u = s.sol_in[i];
    const long long a0 = g.rowptr[u];
    for (long long k = a0 + threadIdx.x; k < g.rowptr[u + 1]; k += blockDim.x) {
      const int2 e = g.adj[k];
      if (k > a0 && g.adj[k - 1].x == e.x) continue;
      const int32_t p = s.pos[e.x];
      if (p >= s.m) w_set(s, (long long)i * s.ldc + (p - s.m), e.y);
    }
  }
}

// cpos[k] = current position of entry k's neighbour (CSR structure).
template <class KeyT>
__global__ void k_init_cpos(const DevGraph g, const DevSolver<KeyT> s) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < g.entries;
       k += (long long)gridDim.x * blockDim.x)
    s.cpos[k] = s.pos[g.adj[k].x];
}

// Objective of a set / bisection given per-vertex flags (1 = inside / side 0).
__global__ void k_objective(const DevGraph g, int32_t problem, const uint8_t* in,
                            unsigned long long* out) {
  for (int32_t a = blockIdx.x * blockDim.x + threadIdx.x; a < g.n; a += gridDim.x * blockDim.x) {
    unsigned long long acc = 0;
    for (long long k = g.rowptr[a]; k < g.rowptr[a + 1]; k++) {
      const int2 e = g.adj[k];
      if (problem == P_MDP) {
        if (in[a] && in[e.x]) acc += (unsigned long long)(long long)e.y;
      } else if (e.x > a && in[a] != in[e.x]) {
        acc += (unsigned long long)(long long)e.y;
      }
    }
    if (acc) atomicAdd(out, acc);
  }
}

// Largest iteration grid launched with programmatic dependent launch (one
// CTA per SM or fewer).
constexpr int kPdlMaxGrid = 148;

template <int PROB, int ST, class KeyT>
cudaError_t launch_iter(const DevGraph& g, const DevSolver<KeyT>& s, int grid, size_t smem,
                        cudaStream_t st, int count) {
  auto fn = iter_kernel<PROB, ST, KeyT>;
  if constexpr (ST == S_WSWAP) {
    if (s.w16) fn = iter_kernel<PROB, ST, KeyT, true>;  // compiled for the 16-bit matrix
  }
  cudaError_t e = allow_dyn_smem(reinterpret_cast<const void*>(fn), smem);
  if (e != cudaSuccess) return e;
  if (grid > kPdlMaxGrid) {
    for (int i = 0; i < count; i++) fn<<<grid, Tpb<ST>::v, smem, st>>>(g, s);
    return cudaGetLastError();
  }
  // One wave or less: an iteration is a chain of latencies, so each grid is
  // launched while the previous one finishes (programmatic stream
  // serialization; its CTAs wait in griddepcontrol.wait), hiding the launch
  // of the dependent chain.  Measured on the 2,000-vertex MDP case: 5-15%
  // more iterations/s.  Larger grids gain nothing and Hash on the bisection
  // graph (1,563 CTAs) lost 9%, so they launch plainly.
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)Tpb<ST>::v);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  for (int i = 0; i < count; i++) {
    e = cudaLaunchKernelEx(&cfg, fn, g, s);
    if (e != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

template <int PROB, class KeyT>
cudaError_t launch_iter_st(int kind, const DevGraph& g, const DevSolver<KeyT>& s, int grid,
                           size_t smem, cudaStream_t st, int count) {
  switch (kind) {
    case S_CSR: return launch_iter<PROB, S_CSR, KeyT>(g, s, grid, smem, st, count);
    case S_HASH: return launch_iter<PROB, S_HASH, KeyT>(g, s, grid, smem, st, count);
    case S_WSWAP: return launch_iter<PROB, S_WSWAP, KeyT>(g, s, grid, smem, st, count);
    case S_BITSET: return launch_iter<PROB, S_BITSET, KeyT>(g, s, grid, smem, st, count);
    case S_BB: return launch_iter<PROB, S_BB, KeyT>(g, s, grid, smem, st, count);
    default: return launch_iter<PROB, S_BITSET_BB, KeyT>(g, s, grid, smem, st, count);
  }
}

// Resident CTAs per SM of the WSwap iteration kernel (the one for the
// matrix's element width).
template <int PROB, class KeyT>
int wswap_blocks_for(bool w16) {
  int nb = 0;
  const cudaError_t e =
      w16 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, iter_kernel<PROB, S_WSWAP, KeyT, true>,
                                                          Tpb<S_WSWAP>::v, 16)
          : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, iter_kernel<PROB, S_WSWAP, KeyT, false>,
                                                          Tpb<S_WSWAP>::v, 16);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return nb;
}
int wswap_blocks_per_sm(int problem, bool wide, bool w16) {
  if (problem == P_MDP) return wide ? wswap_blocks_for<P_MDP, long long>(w16) : wswap_blocks_for<P_MDP, int32_t>(w16);
  return wide ? wswap_blocks_for<P_MAXBS, long long>(w16) : wswap_blocks_for<P_MAXBS, int32_t>(w16);
}

// Column split of a streamed sweep into whole waves: the matrix streams at full
// bandwidth only while every resident CTA slot is busy, so among the splits
// with at least one full wave of tiles (columns a multiple of pc, between lo
// and cap) take the one whose last wave is fullest; near-ties go to more
// tiles.  Returns `fallback` when no split fills a wave.
int64_t wave_cols(int64_t delta, int64_t rows, int64_t pc, int64_t lo, int64_t cap, int64_t slots,
                  int64_t fallback) {
  if (slots <= 0 || rows <= 0) return fallback;
  double best = -1.0;
  int64_t pick = fallback, pick_tiles = 0;
  const int64_t max_nc = (delta + pc - 1) / pc;
  for (int64_t nc = 1; nc <= max_nc; nc++) {
    const int64_t c = (((delta + nc - 1) / nc + pc - 1) / pc) * pc;
    if (c > cap || c < lo) continue;
    const int64_t tiles = rows * ((delta + c - 1) / c);
    if (tiles < slots) continue;
    const int64_t waves = (tiles + slots - 1) / slots;
    const double eff = (double)rows * (double)delta / (double)c / ((double)waves * (double)slots);
    if (eff > best + 0.005) {
      best = eff;
      pick = c;
      pick_tiles = tiles;
    } else if (eff >= best - 0.005 && tiles > pick_tiles) {
      best = std::max(best, eff);
      pick = c;
      pick_tiles = tiles;
    }
  }
  return pick;
}

}  // namespace
}  // namespace tsb

using namespace tsb;

struct ts_solver {
  ts_graph* g = nullptr;
  ts_params p{};
  bool wide = false;
  int32_t n = 0, m = 0, delta = 0, ldc = 0;
  int64_t P = 0;
  int R = 0;
  int32_t n_row_blocks = 0, n_chunks = 0, chunk_cols = 0, stage_bytes = 0;
  int32_t adj_mask = 0, fast = 0, fast_ecap = 0, w16 = 0, n_slices = 1;
  size_t dyn_smem = 0;
  int grid = 0;
  int32_t num_pert = 1;
  int64_t log_cap = 0, trace_cap = 0;
  int64_t window_events = 0;
  DevBuf sol_in, sol_out, vg_in, vg_out, tab_in, tab_out, pos, W, cpos, st, recs, movelog, trace, draws;
  std::mt19937 rng;
  std::vector<long long> host_draws;  // every perturbation event drawn so far, k draws each
  int64_t events_drawn = 0;
  bool external_draws = false;  // perturbation events given by the caller (no more are drawn)
  bool initialized = false;
  int64_t admitted_target = 0;
  DevState* h_st = nullptr;  // pinned mirror

  template <class KeyT>
  DevSolver<KeyT> dev() const {
    DevSolver<KeyT> s;
    std::memset(&s, 0, sizeof(s));
    s.n = n; s.m = m; s.delta = delta; s.ldc = ldc;
    s.problem = p.problem;
    s.tenure_policy = p.tenure_policy;
    s.tenure = p.tenure;
    s.maxt = p.maxt;
    s.piter = p.piter;
    s.num_pert = num_pert;
    const int c1s[4] = {15, 30, 60, 120};
    for (int i = 0; i < 4; i++) s.c2_tab[i] = (int32_t)round(0.7 * c1s[i]);  // :664
    s.c2_fixed = (int32_t)round(0.7 * p.tenure);
    s.n_row_blocks = n_row_blocks; s.n_chunks = n_chunks; s.chunk_cols = chunk_cols;
    s.stage_bytes = stage_bytes;
    s.adj_mask = adj_mask;
    s.tile_rows = R;
    s.fast = fast;
    s.fast_ecap = fast_ecap;
    s.n_slices = n_slices;
    s.w16 = w16;
    s.P = P;
    s.sol_in = sol_in.as<int32_t>(); s.sol_out = sol_out.as<int32_t>();
    s.vg_in = vg_in.as<KeyT>(); s.vg_out = vg_out.as<KeyT>();
    s.tab_in = tab_in.as<int32_t>(); s.tab_out = tab_out.as<int32_t>();
    s.pos = pos.as<int32_t>();
    s.W = W.as<int32_t>();
    s.cpos = cpos.as<int32_t>();
    s.st = st.as<DevState>();
    s.recs = recs.as<CtaRec>();
    s.movelog = movelog.as<int2>();
    s.log_cap = log_cap;
    s.trace = p.trace ? trace.as<TraceRec>() : nullptr;
    s.trace_cap = trace_cap;
    s.draws = draws.as<long long>();
    s.draw_events = window_events;
    return s;
  }
};

namespace {

ts_status read_state(ts_solver* s) {
  TS_CUDA(cudaMemcpyAsync(s->h_st, s->st.p, sizeof(DevState), cudaMemcpyDeviceToHost, s->g->stream));
  TS_CUDA(cudaStreamSynchronize(s->g->stream));
  return TS_OK;
}

ts_status write_state(ts_solver* s) {
  TS_CUDA(cudaMemcpyAsync(s->st.p, s->h_st, sizeof(DevState), cudaMemcpyHostToDevice, s->g->stream));
  TS_CUDA(cudaStreamSynchronize(s->g->stream));
  return TS_OK;
}

template <class KeyT>
ts_status launch_batch(ts_solver* s, int count) {
  DevSolver<KeyT> d = s->dev<KeyT>();
  DevGraph g = s->g->dev();
  cudaError_t e = s->p.problem == P_MDP
                      ? launch_iter_st<P_MDP, KeyT>(s->g->kind, g, d, s->grid, s->dyn_smem, s->g->stream, count)
                      : launch_iter_st<P_MAXBS, KeyT>(s->g->kind, g, d, s->grid, s->dyn_smem, s->g->stream, count);
  if (e != cudaSuccess) return cuda_fail(e, "iteration kernel launch");
  return TS_OK;
}

// MaxBS: make sure the device window holds the draws of every perturbation
// event that can happen before `target` (events are at least piter apart).
ts_status prepare_draws(ts_solver* s, int64_t iters_ahead) {
  if (s->p.problem != P_MAXBS) return TS_OK;
  const int64_t consumed = s->h_st->pert_events;
  int64_t need = iters_ahead / std::max(1, s->p.piter) + 2;
  if (need > s->window_events) need = s->window_events;
  const int k = s->num_pert;
  if (s->external_draws) {
    // caller's stream: a perturbation past its end sets the device error word
    need = std::max<int64_t>(0, std::min<int64_t>(need, s->events_drawn - consumed));
  }
  while (s->events_drawn < consumed + need) {
    draw_event(s->rng, s->P, k, s->host_draws);
    s->events_drawn++;
  }
  TS_CUDA(cudaMemcpyAsync(s->draws.p, s->host_draws.data() + consumed * k,
                          sizeof(long long) * need * k, cudaMemcpyHostToDevice, s->g->stream));
  s->h_st->pert_base = consumed;
  s->h_st->pert_limit = need;
  return TS_OK;
}

template <class KeyT>
ts_status init_device(ts_solver* s, const std::vector<uint8_t>& inside) {
  const int32_t n = s->n, m = s->m;
  cudaStream_t st = s->g->stream;
  std::vector<int32_t> sin(m), sout(s->ldc, 0), pos(n);
  int32_t x = 0, y = 0;
  for (int32_t v = 0; v < n; v++) {  // initialSolution: ascending ids per side
    if (inside[v]) { sin[x] = v; pos[v] = x; x++; }
    else { sout[y] = v; pos[v] = m + y; y++; }
  }
  TS_CUDA(cudaMemcpyAsync(s->sol_in.p, sin.data(), sizeof(int32_t) * m, cudaMemcpyHostToDevice, st));
  TS_CUDA(cudaMemcpyAsync(s->sol_out.p, sout.data(), sizeof(int32_t) * s->ldc, cudaMemcpyHostToDevice, st));
  TS_CUDA(cudaMemcpyAsync(s->pos.p, pos.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
  TS_CUDA(cudaMemsetAsync(s->vg_in.p, 0, s->vg_in.bytes, st));
  TS_CUDA(cudaMemsetAsync(s->vg_out.p, 0, s->vg_out.bytes, st));
  TS_CUDA(cudaMemsetAsync(s->tab_in.p, 0, s->tab_in.bytes, st));
  TS_CUDA(cudaMemsetAsync(s->tab_out.p, 0, s->tab_out.bytes, st));
  DevBuf acc;
  ts_status rc;
  if ((rc = acc.alloc(sizeof(unsigned long long), "alloc")) != TS_OK) return rc;
  TS_CUDA(cudaMemsetAsync(acc.p, 0, sizeof(unsigned long long), st));
  DevSolver<KeyT> d = s->dev<KeyT>();
  DevGraph g = s->g->dev();
  if (s->p.problem == P_MDP) k_init_mdp<KeyT><<<grid_for((int64_t)m * 32), kInitTPB, 0, st>>>(g, d, acc.as<unsigned long long>());
  else k_init_maxbs<KeyT><<<grid_for(n), kInitTPB, 0, st>>>(g, d, acc.as<unsigned long long>());
  TS_CUDA(cudaGetLastError());
  if (s->g->kind == S_WSWAP) {
    TS_CUDA(cudaMemsetAsync(s->W.p, 0, s->W.bytes, st));
    k_init_wswap<KeyT><<<grid_for((int64_t)m * 32), kInitTPB, 0, st>>>(g, d);
    TS_CUDA(cudaGetLastError());
  }
  if (s->g->kind == S_CSR && s->g->entries > 0) {
    k_init_cpos<KeyT><<<grid_for(s->g->entries), kInitTPB, 0, st>>>(g, d);
    TS_CUDA(cudaGetLastError());
  }
  unsigned long long obj = 0;
  TS_CUDA(cudaMemcpyAsync(&obj, acc.p, sizeof(obj), cudaMemcpyDeviceToHost, st));
  TS_CUDA(cudaStreamSynchronize(st));
  long long objective = (long long)obj;
  if (s->p.problem == P_MDP) objective /= 2;
  std::memset(s->h_st, 0, sizeof(DevState));
  s->h_st->cur = objective;
  s->h_st->best = objective;
  return write_state(s);
}

ts_status objective_of(ts_solver* s, const std::vector<uint8_t>& inside, long long* out) {
  cudaStream_t st = s->g->stream;
  DevBuf flags, acc;
  ts_status rc;
  if ((rc = flags.alloc(s->n, "alloc")) != TS_OK) return rc;
  if ((rc = acc.alloc(sizeof(unsigned long long), "alloc")) != TS_OK) return rc;
  TS_CUDA(cudaMemcpyAsync(flags.p, inside.data(), s->n, cudaMemcpyHostToDevice, st));
  TS_CUDA(cudaMemsetAsync(acc.p, 0, sizeof(unsigned long long), st));
  k_objective<<<grid_for(s->n), kInitTPB, 0, st>>>(s->g->dev(), s->p.problem, flags.as<uint8_t>(),
                                                   acc.as<unsigned long long>());
  TS_CUDA(cudaGetLastError());
  unsigned long long v = 0;
  TS_CUDA(cudaMemcpyAsync(&v, acc.p, sizeof(v), cudaMemcpyDeviceToHost, st));
  TS_CUDA(cudaStreamSynchronize(st));
  long long r = (long long)v;
  if (s->p.problem == P_MDP) r /= 2;
  *out = r;
  return TS_OK;
}

// Current inside set and the best one (by undoing the moves logged after the
// last improvement; a swap is its own inverse).
ts_status fetch_sets(ts_solver* s, std::vector<int32_t>& sin, std::vector<int32_t>& sout,
                     bool best) {
  cudaStream_t st = s->g->stream;
  sin.assign(s->m, 0);
  sout.assign(s->ldc, 0);
  TS_CUDA(cudaMemcpyAsync(sin.data(), s->sol_in.p, sizeof(int32_t) * s->m, cudaMemcpyDeviceToHost, st));
  TS_CUDA(cudaMemcpyAsync(sout.data(), s->sol_out.p, sizeof(int32_t) * s->ldc, cudaMemcpyDeviceToHost, st));
  TS_CUDA(cudaStreamSynchronize(st));
  if (best) {
    const int64_t from = s->h_st->best_log_n, to = std::min<int64_t>(s->h_st->log_n, s->log_cap);
    if (to > from) {
      std::vector<int2> tail(to - from);
      TS_CUDA(cudaMemcpyAsync(tail.data(), s->movelog.as<int2>() + from, sizeof(int2) * (to - from),
                              cudaMemcpyDeviceToHost, st));
      TS_CUDA(cudaStreamSynchronize(st));
      for (int64_t k = (int64_t)tail.size() - 1; k >= 0; k--) std::swap(sin[tail[k].x], sout[tail[k].y]);
    }
  }
  return TS_OK;
}

}  // namespace

extern "C" {

ts_status ts_params_default(int32_t problem, ts_params* out) {
  if (!out || (problem != TS_PROBLEM_MDP && problem != TS_PROBLEM_MAXBS)) {
    set_error("ts_params_default: bad argument");
    return TS_ERR_INVALID_ARG;
  }
  std::memset(out, 0, sizeof(*out));
  out->problem = problem;
  if (problem == TS_PROBLEM_MDP) {
    out->m = 100;                 // 'sparse' data set, GPU-MDP-CSR.cu:306
    out->max_iter = 50000;        // :55
    out->tenure_policy = TS_TENURE_REF;
    out->tenure = 15;
  } else {
    out->max_iter = 1000000;      // MacutParams, GPU-MAXBS-CSR.cu:71
    out->tenure_policy = TS_TENURE_REF;
    out->tenure = 25;
  }
  out->maxt = 200;
  out->piter = 500;
  out->gamma = 150;
  out->seed = 1;
  return TS_OK;
}

ts_status ts_solver_create(ts_graph* g, const ts_params* p, ts_solver** out) {
  tsb::TraceRange tr_("ts_solver_create");
  if (!out) { set_error("ts_solver_create: out is NULL"); return TS_ERR_INVALID_ARG; }
  *out = nullptr;
  if (!g || !p) { set_error("ts_solver_create: NULL argument"); return TS_ERR_INVALID_ARG; }
  if (p->problem != TS_PROBLEM_MDP && p->problem != TS_PROBLEM_MAXBS) {
    set_error("ts_solver_create: unknown problem");
    return TS_ERR_INVALID_ARG;
  }
  const int32_t n = g->n;
  const int32_t m = p->problem == TS_PROBLEM_MDP ? p->m : n / 2;
  if (m < 1 || m >= n) { set_error("ts_solver_create: need 1 <= m < n"); return TS_ERR_INVALID_ARG; }
  if (p->max_iter < 0 || p->piter < 1 || p->gamma < 0 || p->maxt < 1 || p->pass < 0 || p->pass > 2 ||
      (p->tenure_policy != TS_TENURE_REF && p->tenure_policy != TS_TENURE_FIXED) || p->tenure < 0) {
    set_error("ts_solver_create: bad parameters");
    return TS_ERR_INVALID_ARG;
  }
  TS_CUDA(cudaSetDevice(g->device));
  auto* s = new ts_solver;
  s->g = g;
  s->p = *p;
  s->n = n;
  s->m = m;
  s->delta = n - m;
  s->ldc = (s->delta + 3) & ~3;
  s->P = (int64_t)m * s->delta;
  // 32-bit pair keys while every gain stays within +-2^30.
  s->wide = 4 * g->max_wdeg >= (1LL << 30);
  // Tiles per iteration: the index structures balance their uneven rows
  // over many tiles; CSR and WSwap prefer few wide ones.  One CTA per tile;
  // the hardware schedules them.
  const bool staged = g->kind != S_CSR && g->kind != S_WSWAP;
  const int64_t min_grid = staged ? 4 * 148 : (g->kind == S_WSWAP ? 4 * 148 : 2 * 148);
  const TileGeom tg = tile_geometry(g, p->problem, m, s->wide, min_grid, p->pass, false);
  s->R = tg.rows;
  s->w16 = g->kind == S_WSWAP && wswap_w16(g) ? 1 : 0;
  s->fast = tg.fast;
  s->fast_ecap = tg.fast_ecap;
  s->n_row_blocks = tg.n_row_blocks;
  s->adj_mask = tg.adj_mask;
  int64_t cols = tg.chunk_cols;
  if (g->kind == S_WSWAP) {
    const int64_t pc = pass_cols_of(g->kind);
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device) != cudaSuccess) {
      cudaGetLastError();
      sms = 0;  // no wave split: the default chunking stands
    }
    const int64_t slots = (int64_t)wswap_blocks_per_sm(p->problem, s->wide, s->w16 != 0) * sms;
    cols = wave_cols(s->delta, s->n_row_blocks, pc, 8 * pc, 64 * pc, slots, cols);
  }
  s->chunk_cols = (int32_t)cols;
  s->n_chunks = (int32_t)((s->delta + cols - 1) / cols);
  s->n_slices = tile_slices(g, tg);
  s->grid = s->n_row_blocks * s->n_chunks * s->n_slices;
  s->stage_bytes = tg.stage_bytes;
  s->dyn_smem = tg.smem;
  const int32_t g_eff = std::min(p->gamma, n);
  s->num_pert = std::max(1, g_eff / 2);  // GPU-MAXBS-CSR.cu:433-434
  int64_t pert_moves = p->problem == TS_PROBLEM_MAXBS ? (p->max_iter / p->piter + 1) * s->num_pert : 0;
  s->log_cap = p->max_iter + pert_moves + 1;
  s->trace_cap = p->trace ? p->max_iter + pert_moves + 2 : 0;
  s->window_events = p->problem == TS_PROBLEM_MAXBS ? 64 : 1;
  const size_t kb = s->wide ? sizeof(long long) : sizeof(int32_t);
  ts_status rc = TS_OK;
  auto A = [&](DevBuf& b, size_t bytes, const char* what) {
    if (rc == TS_OK) rc = b.alloc(bytes, what);
  };
  A(s->sol_in, sizeof(int32_t) * (size_t)m, "alloc sol_in");
  A(s->sol_out, sizeof(int32_t) * (size_t)s->ldc, "alloc sol_out");
  A(s->vg_in, kb * (size_t)m, "alloc vg_in");
  A(s->vg_out, kb * (size_t)s->ldc, "alloc vg_out");
  A(s->tab_in, sizeof(int32_t) * (size_t)m, "alloc tab_in");
  A(s->tab_out, sizeof(int32_t) * (size_t)s->ldc, "alloc tab_out");
  A(s->pos, sizeof(int32_t) * (size_t)n, "alloc pos");
  A(s->st, sizeof(DevState), "alloc state");
  A(s->recs, sizeof(CtaRec) * (size_t)s->grid, "alloc records");
  A(s->movelog, sizeof(int2) * (size_t)s->log_cap, "alloc move log");
  if (p->trace) A(s->trace, sizeof(TraceRec) * (size_t)s->trace_cap, "alloc trace");
  A(s->draws, sizeof(long long) * (size_t)(s->window_events * s->num_pert), "alloc draws");
  if (g->kind == S_WSWAP) {
    // Padded to whole row blocks so a tile never reads past the matrix.
    size_t rows = (size_t)s->n_row_blocks * s->R;
    A(s->W, (s->w16 ? sizeof(int16_t) : sizeof(int32_t)) * rows * (size_t)s->ldc, "alloc WSwap matrix");
  }
  if (g->kind == S_CSR) A(s->cpos, sizeof(int32_t) * (size_t)std::max<int64_t>(1, g->entries), "alloc cpos");
  if (rc == TS_OK) {
    cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&s->h_st), sizeof(DevState));
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaMallocHost state");
  }
  if (rc != TS_OK) { delete s; return rc; }
  std::memset(s->h_st, 0, sizeof(DevState));
  *out = s;
  return TS_OK;
}

ts_status ts_solver_init(ts_solver* s, const int32_t* initial) {
  tsb::TraceRange tr_("ts_solver_init");
  if (!s) { set_error("ts_solver_init: NULL solver"); return TS_ERR_INVALID_ARG; }
  TS_CUDA(cudaSetDevice(s->g->device));
  const int32_t n = s->n, m = s->m;
  std::vector<uint8_t> inside(n, 0);
  s->rng.seed(s->p.seed);
  s->host_draws.clear();
  s->events_drawn = 0;
  s->external_draws = false;
  if (s->p.problem == P_MDP) {
    if (!initial) {
      std::vector<int32_t> ids;
      mdp_random_set(n, m, s->p.seed, ids);
      for (int32_t v : ids) inside[v] = 1;
    } else {
      for (int32_t i = 0; i < m; i++) {
        int32_t v = initial[i];
        if (v < 0 || v >= n || inside[v]) {
          set_error("ts_solver_init: MDP initial set must hold m distinct ids in [0, n)");
          return TS_ERR_INVALID_ARG;
        }
        inside[v] = 1;
      }
    }
  } else {
    if (!initial) {
      maxbs_random_part(s->rng, n, inside);
    } else {
      int32_t zeros = 0;
      for (int32_t v = 0; v < n; v++) {
        if (initial[v] != 0 && initial[v] != 1) {
          set_error("ts_solver_init: MaxBS partition entries must be 0 or 1");
          return TS_ERR_INVALID_ARG;
        }
        inside[v] = initial[v] == 0;
        zeros += inside[v];
      }
      if (zeros != m) {
        set_error("ts_solver_init: MaxBS partition must put floor(n/2) vertices in part 0");
        return TS_ERR_INVALID_ARG;
      }
    }
  }
  ts_status rc = s->wide ? init_device<long long>(s, inside) : init_device<int32_t>(s, inside);
  if (rc != TS_OK) return rc;
  s->initialized = true;
  return TS_OK;
}

}  // extern "C"

namespace {

// Admits up to k iterations: target = iter + k (bounded by max_iter and, for
// MaxBS, by the perturbation-draw window), draws staged, state written.
// Requires a synchronised state mirror (read_state).
ts_status prepare_batch(ts_solver* s, int64_t k, int64_t* admitted) {
  *admitted = 0;
  if (s->h_st->done) return TS_OK;
  int64_t sub = std::min<int64_t>(k, s->p.max_iter - s->h_st->iter);
  if (sub < 0) sub = 0;
  if (s->p.problem == P_MAXBS) {
    // A batch may meet at most window_events - 2 perturbation events.
    sub = std::min<int64_t>(sub, (s->window_events - 2) * (int64_t)s->p.piter);
  }
  s->h_st->target = s->h_st->iter + sub;
  ts_status rc;
  if ((rc = prepare_draws(s, sub)) != TS_OK) return rc;
  if ((rc = write_state(s)) != TS_OK) return rc;
  s->admitted_target = s->h_st->target;
  *admitted = sub;
  return TS_OK;
}

ts_status enqueue_launches(ts_solver* s, int64_t launches) {
  while (launches > 0) {
    int c = (int)std::min<int64_t>(launches, 1 << 20);
    ts_status rc = s->wide ? launch_batch<long long>(s, c) : launch_batch<int32_t>(s, c);
    if (rc != TS_OK) return rc;
    launches -= c;
  }
  return TS_OK;
}

// Waits for the admitted batch; tops it up when exact passes consumed launches.
ts_status finish_batch(ts_solver* s) {
  ts_status rc;
  for (int guard = 0; guard < 1 << 20; guard++) {
    if ((rc = read_state(s)) != TS_OK) return rc;
    if (s->h_st->err) {
      set_error("device error word set (" + std::to_string(s->h_st->err) + ")");
      return TS_ERR_DEVICE;
    }
    if (s->h_st->done || s->h_st->iter >= s->admitted_target) return TS_OK;
    if ((rc = enqueue_launches(s, s->admitted_target - s->h_st->iter + 1)) != TS_OK) return rc;
  }
  set_error("no progress");
  return TS_ERR_DEVICE;
}

}  // namespace

extern "C" {

ts_status ts_solver_set_perturbations(ts_solver* s, const int64_t* draws, int64_t n_events) {
  if (!s || n_events < 0 || (n_events > 0 && !draws)) {
    set_error("ts_solver_set_perturbations: bad argument");
    return TS_ERR_INVALID_ARG;
  }
  if (!s->initialized) {
    set_error("ts_solver_set_perturbations: call ts_solver_init first");
    return TS_ERR_STATE;
  }
  if (s->p.problem != P_MAXBS) {
    set_error("ts_solver_set_perturbations: only Max Bisection perturbs");
    return TS_ERR_INVALID_ARG;
  }
  TS_CUDA(cudaSetDevice(s->g->device));
  ts_status rc = read_state(s);
  if (rc != TS_OK) return rc;
  if (s->h_st->iter != 0 || s->h_st->pert_events != 0) {
    set_error("ts_solver_set_perturbations: the search has already started");
    return TS_ERR_STATE;
  }
  const int64_t words = n_events * s->num_pert;
  for (int64_t q = 0; q < words; q++)
    if (draws[q] < 0 || draws[q] >= s->P) {
      set_error("ts_solver_set_perturbations: move index out of range");
      return TS_ERR_INVALID_ARG;
    }
  s->host_draws.assign(draws, draws + words);
  s->events_drawn = n_events;
  s->external_draws = true;
  return TS_OK;
}

ts_status ts_solver_step(ts_solver* s, int64_t k, int64_t* done_iters) {
  tsb::TraceRange tr_("ts_solver_step");
  if (done_iters) *done_iters = 0;
  if (!s) { set_error("ts_solver_step: NULL solver"); return TS_ERR_INVALID_ARG; }
  if (!s->initialized) { set_error("ts_solver_step: call ts_solver_init first"); return TS_ERR_STATE; }
  if (k < 0) { set_error("ts_solver_step: negative k"); return TS_ERR_INVALID_ARG; }
  TS_CUDA(cudaSetDevice(s->g->device));
  ts_status rc = read_state(s);
  if (rc != TS_OK) return rc;
  const int64_t start = s->h_st->iter;
  int64_t remaining = k;
  while (remaining > 0 && !s->h_st->done && s->h_st->iter < s->p.max_iter) {
    int64_t sub = 0;
    if ((rc = prepare_batch(s, remaining, &sub)) != TS_OK) return rc;
    if (sub <= 0) break;
    const int64_t iter0 = s->h_st->iter;
    if ((rc = enqueue_launches(s, sub)) != TS_OK) return rc;
    if ((rc = finish_batch(s)) != TS_OK) return rc;
    remaining -= s->h_st->iter - iter0;
  }
  if (done_iters) *done_iters = s->h_st->iter - start;
  return TS_OK;
}

ts_status ts_solver_prepare(ts_solver* s, int64_t k, int64_t* prepared) {
  if (prepared) *prepared = 0;
  if (!s) { set_error("ts_solver_prepare: NULL solver"); return TS_ERR_INVALID_ARG; }
  if (!s->initialized) { set_error("ts_solver_prepare: call ts_solver_init first"); return TS_ERR_STATE; }
  if (k < 0) { set_error("ts_solver_prepare: negative k"); return TS_ERR_INVALID_ARG; }
  TS_CUDA(cudaSetDevice(s->g->device));
  ts_status rc = read_state(s);
  if (rc != TS_OK) return rc;
  int64_t sub = 0;
  if ((rc = prepare_batch(s, k, &sub)) != TS_OK) return rc;
  if (prepared) *prepared = sub;
  return TS_OK;
}

ts_status ts_solver_enqueue(ts_solver* s, int64_t k) {
  tsb::TraceRange tr_("ts_solver_enqueue");
  if (!s || k < 0) { set_error("ts_solver_enqueue: bad argument"); return TS_ERR_INVALID_ARG; }
  if (!s->initialized) { set_error("ts_solver_enqueue: call ts_solver_init first"); return TS_ERR_STATE; }
  TS_CUDA(cudaSetDevice(s->g->device));
  return enqueue_launches(s, k);
}

ts_status ts_solver_sync(ts_solver* s, int64_t* iter) {
  tsb::TraceRange tr_("ts_solver_sync");
  if (iter) *iter = 0;
  if (!s) { set_error("ts_solver_sync: NULL solver"); return TS_ERR_INVALID_ARG; }
  if (!s->initialized) { set_error("ts_solver_sync: call ts_solver_init first"); return TS_ERR_STATE; }
  TS_CUDA(cudaSetDevice(s->g->device));
  ts_status rc = finish_batch(s);
  if (rc != TS_OK) return rc;
  if (iter) *iter = s->h_st->iter;
  return TS_OK;
}

ts_status ts_solver_result(ts_solver* s, ts_result* out, int32_t* best_sol) {
  tsb::TraceRange tr_("ts_solver_result");
  if (!s || !out) { set_error("ts_solver_result: NULL argument"); return TS_ERR_INVALID_ARG; }
  if (!s->initialized) { set_error("ts_solver_result: call ts_solver_init first"); return TS_ERR_STATE; }
  TS_CUDA(cudaSetDevice(s->g->device));
  ts_status rc = read_state(s);
  if (rc != TS_OK) return rc;
  std::vector<int32_t> sin, sout;
  if ((rc = fetch_sets(s, sin, sout, true)) != TS_OK) return rc;
  std::vector<uint8_t> inside(s->n, 0);
  for (int32_t v : sin) inside[v] = 1;
  long long bt = 0;
  if ((rc = objective_of(s, inside, &bt)) != TS_OK) return rc;
  std::memset(out, 0, sizeof(*out));
  out->iterations = s->h_st->iter;
  out->evaluations = s->h_st->evaluations;
  out->cur = s->h_st->cur;
  out->best = s->h_st->best;
  out->best_true = bt;
  out->perturbations = s->h_st->pert_moves;
  out->stopped = s->h_st->stopped;
  out->m = s->m;
  out->n = s->n;
  out->device_error = s->h_st->err;
  if (best_sol) {
    if (s->p.problem == P_MDP) {
      std::memcpy(best_sol, sin.data(), sizeof(int32_t) * s->m);
    } else {
      for (int32_t v = 0; v < s->n; v++) best_sol[v] = inside[v] ? 0 : 1;
    }
  }
  return TS_OK;
}

ts_status ts_solver_state(ts_solver* s, int32_t* sol, int32_t* pos, int32_t* tab, int64_t* vg) {
  if (!s) { set_error("ts_solver_state: NULL solver"); return TS_ERR_INVALID_ARG; }
  if (!s->initialized) { set_error("ts_solver_state: call ts_solver_init first"); return TS_ERR_STATE; }
  TS_CUDA(cudaSetDevice(s->g->device));
  cudaStream_t st = s->g->stream;
  const int32_t n = s->n, m = s->m, d = s->delta;
  std::vector<int32_t> sin(m), sout(s->ldc), tin(m), tout(s->ldc), p(n);
  std::vector<long long> vin(m), vout(s->ldc);
  TS_CUDA(cudaMemcpyAsync(sin.data(), s->sol_in.p, 4 * (size_t)m, cudaMemcpyDeviceToHost, st));
  TS_CUDA(cudaMemcpyAsync(sout.data(), s->sol_out.p, 4 * (size_t)s->ldc, cudaMemcpyDeviceToHost, st));
  TS_CUDA(cudaMemcpyAsync(tin.data(), s->tab_in.p, 4 * (size_t)m, cudaMemcpyDeviceToHost, st));
  TS_CUDA(cudaMemcpyAsync(tout.data(), s->tab_out.p, 4 * (size_t)s->ldc, cudaMemcpyDeviceToHost, st));
  TS_CUDA(cudaMemcpyAsync(p.data(), s->pos.p, 4 * (size_t)n, cudaMemcpyDeviceToHost, st));
  if (s->wide) {
    TS_CUDA(cudaMemcpyAsync(vin.data(), s->vg_in.p, 8 * (size_t)m, cudaMemcpyDeviceToHost, st));
    TS_CUDA(cudaMemcpyAsync(vout.data(), s->vg_out.p, 8 * (size_t)s->ldc, cudaMemcpyDeviceToHost, st));
    TS_CUDA(cudaStreamSynchronize(st));
  } else {
    std::vector<int32_t> a(m), b(s->ldc);
    TS_CUDA(cudaMemcpyAsync(a.data(), s->vg_in.p, 4 * (size_t)m, cudaMemcpyDeviceToHost, st));
    TS_CUDA(cudaMemcpyAsync(b.data(), s->vg_out.p, 4 * (size_t)s->ldc, cudaMemcpyDeviceToHost, st));
    TS_CUDA(cudaStreamSynchronize(st));
    for (int32_t i = 0; i < m; i++) vin[i] = a[i];
    for (int32_t j = 0; j < s->ldc; j++) vout[j] = b[j];
  }
  for (int32_t i = 0; i < m; i++) {
    if (sol) sol[i] = sin[i];
    if (tab) tab[sin[i]] = tin[i];
    if (vg) vg[sin[i]] = vin[i];
  }
  for (int32_t j = 0; j < d; j++) {
    if (sol) sol[m + j] = sout[j];
    if (tab) tab[sout[j]] = tout[j];
    if (vg) vg[sout[j]] = vout[j];
  }
  if (pos) std::memcpy(pos, p.data(), 4 * (size_t)n);
  return TS_OK;
}

ts_status ts_solver_trace(ts_solver* s, ts_trace_rec* out, int64_t cap, int64_t* n_out) {
  if (!s || (cap > 0 && !out)) { set_error("ts_solver_trace: bad argument"); return TS_ERR_INVALID_ARG; }
  if (n_out) *n_out = 0;
  if (!s->p.trace) { set_error("ts_solver_trace: solver created without trace"); return TS_ERR_STATE; }
  TS_CUDA(cudaSetDevice(s->g->device));
  ts_status rc = read_state(s);
  if (rc != TS_OK) return rc;
  int64_t have = std::min<int64_t>(s->h_st->trace_n, s->trace_cap);
  int64_t cnt = std::min<int64_t>(have, cap);
  static_assert(sizeof(ts_trace_rec) == sizeof(TraceRec), "trace record layout");
  if (cnt > 0) {
    TS_CUDA(cudaMemcpyAsync(out, s->trace.p, sizeof(TraceRec) * cnt, cudaMemcpyDeviceToHost, s->g->stream));
    TS_CUDA(cudaStreamSynchronize(s->g->stream));
  }
  if (n_out) *n_out = have;
  return TS_OK;
}

ts_status ts_random_start(int32_t problem, int32_t n, int32_t m, uint32_t seed, int32_t* out) {
  if (!out || n < 2 || (problem == TS_PROBLEM_MDP && (m < 1 || m >= n)) ||
      (problem != TS_PROBLEM_MDP && problem != TS_PROBLEM_MAXBS)) {
    set_error("ts_random_start: bad argument");
    return TS_ERR_INVALID_ARG;
  }
  if (problem == TS_PROBLEM_MDP) {
    std::vector<int32_t> ids;
    mdp_random_set(n, m, seed, ids);
    std::memcpy(out, ids.data(), sizeof(int32_t) * m);
  } else {
    std::mt19937 rng;
    rng.seed(seed);
    std::vector<uint8_t> side0;
    maxbs_random_part(rng, n, side0);
    for (int32_t v = 0; v < n; v++) out[v] = side0[v] ? 0 : 1;
  }
  return TS_OK;
}

ts_status ts_perturb_draws(int32_t n, uint32_t seed, int32_t gamma, int32_t init_random,
                           int32_t n_events, int64_t* out) {
  if (!out || n < 2 || n_events < 0 || gamma < 0) {
    set_error("ts_perturb_draws: bad argument");
    return TS_ERR_INVALID_ARG;
  }
  std::mt19937 rng;
  rng.seed(seed);
  if (init_random) {
    std::vector<uint8_t> side0;
    maxbs_random_part(rng, n, side0);
  }
  const int k = std::max(1, std::min(gamma, n) / 2);
  const int64_t m = n / 2, P = m * (int64_t)(n - m);
  std::vector<long long> d;
  for (int32_t e = 0; e < n_events; e++) draw_event(rng, P, k, d);
  for (size_t i = 0; i < d.size(); i++) out[i] = d[i];
  return TS_OK;
}

ts_status ts_solver_info_get(const ts_solver* s, ts_solver_info* out) {
  if (!s || !out) { set_error("ts_solver_info_get: NULL argument"); return TS_ERR_INVALID_ARG; }
  std::memset(out, 0, sizeof(*out));
  out->grid = s->grid;
  out->tile_rows = s->R;
  out->chunk_cols = s->chunk_cols;
  out->n_chunks = s->n_chunks;
  out->threads = tpb_of(s->g->kind);
  out->dyn_smem_bytes = (int32_t)s->dyn_smem;
  out->key_bytes = s->wide ? 8 : 4;
  out->w_bytes = s->g->kind == S_WSWAP ? (s->w16 ? 2 : 4) : 0;
  out->slices = s->n_slices;
  return TS_OK;
}

ts_status ts_solver_destroy(ts_solver* s) {
  if (!s) return TS_OK;
  cudaSetDevice(s->g->device);
  cudaStreamSynchronize(s->g->stream);
  if (s->h_st) cudaFreeHost(s->h_st);
  delete s;
  return TS_OK;
}

}  // extern "C"
