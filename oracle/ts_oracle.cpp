// ts_oracle.cpp -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// CPU restatement (exact int64) of the reference tabu-search iteration for the
// Maximum Diversity Problem and Max Bisection.  Used only as the checker in
// tests/, by __graft_entry__.smoke() and as the timed CPU baseline in bench.py.
// Every function cites the reference lines it follows; see ts_oracle.h.
#include "ts_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <random>
#include <unordered_set>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

struct or_graph {
  int32_t n = 0;
  std::vector<int64_t> rowptr;  // n+1
  std::vector<int32_t> col;     // sorted by neighbour, stable in input order
  std::vector<int32_t> w;
};

extern "C" or_graph* or_graph_create(int32_t n, int64_t num_edges, const int32_t* u,
                                     const int32_t* v, const int32_t* w,
                                     int drop_self_loops) {
  // Loader semantics: GPU-MDP-CSR.cu:324-358 (self-loops dropped :340) and
  // GPU-MAXBS-CSR.cu:156-170 (kept: both push_backs land in row u).
  // Row sort by neighbour id: createCSR GPU-MDP-CSR.cu:211-227.
  if (n < 0) return nullptr;
  auto* g = new or_graph;
  g->n = n;
  std::vector<int64_t> deg(n, 0);
  for (int64_t e = 0; e < num_edges; e++) {
    if (u[e] < 0 || u[e] >= n || v[e] < 0 || v[e] >= n) { delete g; return nullptr; }
    if (drop_self_loops && u[e] == v[e]) continue;
    deg[u[e]]++;
    deg[v[e]]++;
  }
  g->rowptr.assign(n + 1, 0);
  for (int32_t i = 0; i < n; i++) g->rowptr[i + 1] = g->rowptr[i] + deg[i];
  std::vector<int64_t> fill(g->rowptr.begin(), g->rowptr.end() - 1);
  g->col.resize(g->rowptr[n]);
  g->w.resize(g->rowptr[n]);
  for (int64_t e = 0; e < num_edges; e++) {
    if (drop_self_loops && u[e] == v[e]) continue;
    int64_t a = fill[u[e]]++;
    g->col[a] = v[e]; g->w[a] = w[e];
    int64_t b = fill[v[e]]++;
    g->col[b] = u[e]; g->w[b] = w[e];
  }
  std::vector<std::pair<int32_t, int32_t>> tmp;
  for (int32_t r = 0; r < n; r++) {
    int64_t s = g->rowptr[r], t = g->rowptr[r + 1];
    tmp.clear();
    for (int64_t k = s; k < t; k++) tmp.push_back({g->col[k], g->w[k]});
    std::stable_sort(tmp.begin(), tmp.end(),
                     [](const std::pair<int32_t, int32_t>& a,
                        const std::pair<int32_t, int32_t>& b) { return a.first < b.first; });
    for (int64_t k = s; k < t; k++) { g->col[k] = tmp[k - s].first; g->w[k] = tmp[k - s].second; }
  }
  return g;
}

extern "C" void or_graph_destroy(or_graph* g) { delete g; }
extern "C" int64_t or_graph_num_entries(const or_graph* g) { return g->rowptr[g->n]; }

// gpu_edge, GPU-MDP-CSR.cu:555-564: first matching entry of u's row, else 0.
extern "C" int32_t or_lookup(const or_graph* g, int32_t u, int32_t v) {
  for (int64_t k = g->rowptr[u]; k < g->rowptr[u + 1]; k++)
    if (g->col[k] == v) return g->w[k];
  return 0;
}

extern "C" void or_mdp_random_initial(int32_t n, int32_t m, uint32_t seed, int32_t* sol) {
  // GPU-MDP-CSR.cu:1248 srand, :773-784 rejection sampling with rand()%n.
  srand(seed);
  std::vector<char> used(n, 0);
  int32_t k = 0;
  while (k < m) {
    int32_t idx = rand() % n;
    if (!used[idx]) { sol[k++] = idx; used[idx] = 1; }
  }
}

static void maxbs_shuffle_partition(std::mt19937& rng, int32_t n, int32_t* part) {
  // randomPartition GPU-MAXBS-CSR.cu:187-195.
  std::vector<int> vertices(n);
  std::iota(vertices.begin(), vertices.end(), 0);
  std::shuffle(vertices.begin(), vertices.end(), rng);
  for (int32_t i = 0; i < n; i++) part[i] = 1;
  for (int32_t i = 0; i < n / 2; i++) part[vertices[i]] = 0;
}

extern "C" void or_maxbs_random_partition(int32_t n, uint32_t seed, int32_t* part) {
  std::mt19937 rng;
  rng.seed(seed);  // macut GPU-MAXBS-CSR.cu:682
  maxbs_shuffle_partition(rng, n, part);
}

// Draws of one perturbation event: GPU-MAXBS-CSR.cu:481-492.
static void perturb_event(std::mt19937& rng, int64_t P, int32_t k, int64_t* out) {
  std::unordered_set<int64_t> used;
  for (int32_t p = 0; p < k; p++) {
    int64_t mv;
    do {
      if (P - 1 <= INT32_MAX) {
        std::uniform_int_distribution<int> d(0, (int)(P - 1));
        mv = d(rng);
      } else {  // beyond the reference's int range (it overflows there)
        std::uniform_int_distribution<long long> d(0, P - 1);
        mv = d(rng);
      }
    } while (used.count(mv));
    used.insert(mv);
    out[p] = mv;
  }
}

extern "C" void or_maxbs_perturb_draws(int32_t n, uint32_t seed, int32_t init_random,
                                       int32_t n_events, int32_t k, int64_t* out) {
  std::mt19937 rng;
  rng.seed(seed);
  if (init_random) {
    std::vector<int32_t> part(n);
    maxbs_shuffle_partition(rng, n, part.data());
  }
  int64_t m = n / 2, P = m * (int64_t)(n - m);
  for (int32_t e = 0; e < n_events; e++) perturb_event(rng, P, k, out + (int64_t)e * k);
}

extern "C" int32_t or_mdp_tenure(int64_t iter) {
  // determine_tabu_tenure GPU-MDP-CSR.cu:461-476 (alpha 15, T 1500 :53-54).
  const int alpha = 15, T = 1500;
  int temp = (int)(iter % T);
  if (temp > 700 && temp <= 800) return 8 * alpha;
  if ((temp > 300 && temp <= 400) || (temp > 1100 && temp <= 1200)) return 4 * alpha;
  if ((temp > 100 && temp <= 200) || (temp > 500 && temp <= 600) ||
      (temp > 900 && temp <= 1000) || (temp > 1300 && temp <= 1400))
    return 2 * alpha;
  return alpha;
}

extern "C" int32_t or_mdp_c2(int32_t c1) { return (int32_t)round(0.7 * c1); }  // :664

extern "C" int32_t or_maxbs_tenure(int64_t iter, int32_t maxt) {
  // tabuTenure GPU-MAXBS-CSR.cu:248-263.
  static const int b[15] = {1, 2, 1, 4, 1, 2, 1, 8, 1, 2, 1, 4, 1, 2, 1};
  long long period = 16LL * maxt;
  long long it = ((iter - 1) % period) + 1;
  long long pos = 1;
  for (int i = 0; i < 15; i++) {
    long long tenure = (1LL * maxt * b[i]) / 8;
    long long length = 4LL * tenure;
    if (it < pos + length) return (int32_t)tenure;
    pos += length;
  }
  return maxt / 8;
}

extern "C" int64_t or_round_f32(int64_t x) {
  // IEEE binary32 round-to-nearest-even of an integer (24 significant bits).
  if (x == 0) return 0;
  int neg = x < 0;
  uint64_t a = neg ? (uint64_t)0 - (uint64_t)x : (uint64_t)x;
  int msb = 63 - __builtin_clzll(a);
  if (msb <= 23) return x;
  int shift = msb - 23;
  uint64_t q = a >> shift, rem = a & ((1ULL << shift) - 1), half = 1ULL << (shift - 1);
  if (rem > half || (rem == half && (q & 1))) q++;
  uint64_t r = q << shift;
  return neg ? -(int64_t)r : (int64_t)r;
}

// d_gain = INF + d_gain with INF = -9999999999.0 (double), stored as float:
// GPU-MAXBS-CSR.cu:7,:350.
extern "C" int64_t or_maxbs_penalty(int64_t g) { return or_round_f32(g - 9999999999LL); }

namespace {

struct Best { int64_t key; int64_t idx; };

inline void better(Best& a, const Best& b) {  // (key desc, idx asc)
  if (b.key > a.key || (b.key == a.key && b.idx < a.idx)) a = b;
}

struct State {
  const or_graph* g;
  int32_t n, m, delta;
  int64_t P;
  std::vector<int32_t> sol, pos, tab;
  std::vector<int64_t> vg;
  int64_t cur = 0, best = 0;
};

// All-pairs evaluation + ArgMax of one iteration (calculateSwapGain :567-584 /
// calculateMoveGain :337-353 followed by cub::DeviceReduce::ArgMax).
Best sweep(const State& s, int problem, int64_t iter, int threads, int32_t row_limit = -1) {
  const int32_t n = s.n, delta = s.delta;
  const int32_t m = s.m, rows = row_limit < 0 ? s.m : row_limit;
  std::vector<int64_t> pvg(n);
  std::vector<char> ptab(n);
  for (int32_t p = 0; p < n; p++) {
    pvg[p] = s.vg[s.sol[p]];
    ptab[p] = s.tab[s.sol[p]] > iter;
  }
  const int64_t cur = s.cur, bestw = s.best;
  int nt = threads > 0 ? threads : 1;
#ifdef _OPENMP
  if (threads <= 0) nt = omp_get_max_threads();
#else
  nt = 1;
#endif
  std::vector<Best> part(nt, Best{INT64_MIN, INT64_MAX});
#pragma omp parallel num_threads(nt)
  {
    int t = 0;
#ifdef _OPENMP
    t = omp_get_thread_num();
#endif
    int32_t r0 = (int32_t)((int64_t)rows * t / nt), r1 = (int32_t)((int64_t)rows * (t + 1) / nt);
    std::vector<int32_t> stamp(n, -1), wmark(n, 0);
    Best b{INT64_MIN, INT64_MAX};
    for (int32_t i = r0; i < r1; i++) {
      int32_t u = s.sol[i];
      // w(u, .) for this row: first entry of a duplicated pair wins (gpu_edge).
      for (int64_t k = s.g->rowptr[u]; k < s.g->rowptr[u + 1]; k++) {
        int32_t z = s.g->col[k];
        if (stamp[z] != i) { stamp[z] = i; wmark[z] = s.g->w[k]; }
      }
      const int64_t vu = pvg[i];
      const bool tu = ptab[i];
      const int64_t base = (int64_t)i * delta - m;
      for (int32_t j = m; j < n; j++) {
        int32_t v = s.sol[j];
        int64_t w = stamp[v] == i ? wmark[v] : 0;
        int64_t gain, key;
        if (problem == OR_MDP) gain = pvg[j] - vu - w;
        else gain = vu + pvg[j] + 2 * w;
        bool allowed = !(tu || ptab[j]) || (cur + gain > bestw);
        if (allowed) key = gain;
        else key = problem == OR_MDP ? -99999 : or_maxbs_penalty(gain);
        if (key > b.key) { b.key = key; b.idx = base + j; }
      }
    }
    part[t] = b;
  }
  Best r{INT64_MIN, INT64_MAX};
  for (int t = 0; t < nt; t++) better(r, part[t]);
  return r;
}

void mdp_apply(State& s, int32_t iu, int32_t iv, int64_t iter, int32_t c1, int32_t c2) {
  // updateVertexEdgeGain :523-541 then updateSolution :544-553.
  const or_graph* g = s.g;
  int32_t u = s.sol[iu], v = s.sol[iv];
  for (int64_t k = g->rowptr[u]; k < g->rowptr[u + 1]; k++) s.vg[g->col[k]] -= g->w[k];
  for (int64_t k = g->rowptr[v]; k < g->rowptr[v + 1]; k++) s.vg[g->col[k]] += g->w[k];
  s.sol[iu] = v; s.sol[iv] = u;
  s.tab[u] = (int32_t)(iter + c1);
  s.tab[v] = (int32_t)(iter + c2);
  s.pos[u] = iv; s.pos[v] = iu;
}

// updateMoveGain :355-375 then finalizeMove :377-399.  Returns aux (the
// perturbation gain read after the update, before negation).
int64_t maxbs_apply(State& s, int32_t iu, int32_t iv, int64_t iter, int32_t tt, int update_tabu) {
  const or_graph* g = s.g;
  const int32_t m = s.m;
  int32_t u = s.sol[iu], v = s.sol[iv];
  for (int64_t k = g->rowptr[u]; k < g->rowptr[u + 1]; k++) {
    int32_t z = g->col[k];
    int64_t w2 = 2 * (int64_t)g->w[k];
    if (s.pos[z] < m) s.vg[z] -= w2; else s.vg[z] += w2;
  }
  for (int64_t k = g->rowptr[v]; k < g->rowptr[v + 1]; k++) {
    int32_t z = g->col[k];
    int64_t w2 = 2 * (int64_t)g->w[k];
    if (s.pos[z] >= m) s.vg[z] -= w2; else s.vg[z] += w2;
  }
  int64_t aux = 0;
  if (!update_tabu) aux = s.vg[u] + s.vg[v] - 2 * (int64_t)or_lookup(g, u, v);
  s.vg[u] = -s.vg[u];
  s.vg[v] = -s.vg[v];
  s.sol[iu] = v; s.sol[iv] = u;
  s.pos[u] = iv; s.pos[v] = iu;
  if (update_tabu) { s.tab[u] = (int32_t)(iter + tt); s.tab[v] = (int32_t)(iter + tt); }
  return aux;
}

int64_t mdp_objective(const or_graph* g, const std::vector<char>& in) {
  int64_t twice = 0;
  for (int32_t a = 0; a < g->n; a++) {
    if (!in[a]) continue;
    for (int64_t k = g->rowptr[a]; k < g->rowptr[a + 1]; k++)
      if (in[g->col[k]]) twice += g->w[k];
  }
  return twice / 2;
}

int64_t maxbs_cut(const or_graph* g, const std::vector<int32_t>& part) {
  // computeFitnessFromScratch GPU-MAXBS-CSR.cu:197-206.
  int64_t f = 0;
  for (int32_t a = 0; a < g->n; a++)
    for (int64_t k = g->rowptr[a]; k < g->rowptr[a + 1]; k++) {
      int32_t b = g->col[k];
      if (b > a && part[b] != part[a]) f += g->w[k];
    }
  return f;
}

}  // namespace

static int build_state(const or_graph* g, const or_params* p, const int32_t* initial, State& s,
                       std::mt19937& rng, std::vector<int32_t>* part_out);

static int build_state(const or_graph* g, const or_params* p, const int32_t* initial, State& s,
                       std::mt19937& rng, std::vector<int32_t>* part_out) {
  s.g = g;
  s.n = g->n;
  const int problem = p->problem;
  s.m = problem == OR_MDP ? p->m : g->n / 2;
  if (s.m < 1 || s.m >= s.n) return 1;
  s.delta = s.n - s.m;
  s.P = (int64_t)s.m * s.delta;
  const int32_t n = s.n, m = s.m;
  s.sol.assign(n, 0); s.pos.assign(n, 0); s.tab.assign(n, 0); s.vg.assign(n, 0);
  std::vector<char> inside(n, 0);
  rng.seed(p->seed);
  std::vector<int32_t> part(n, 1);
  if (problem == OR_MDP) {
    std::vector<int32_t> init(m);
    if (p->init_mode == OR_INIT_RANDOM) or_mdp_random_initial(n, m, p->seed, init.data());
    else std::copy(initial, initial + m, init.begin());
    for (int32_t i = 0; i < m; i++) {
      if (init[i] < 0 || init[i] >= n || inside[init[i]]) return 2;
      inside[init[i]] = 1;
    }
  } else {
    if (p->init_mode == OR_INIT_RANDOM) maxbs_shuffle_partition(rng, n, part.data());
    else std::copy(initial, initial + n, part.begin());
    int32_t c0 = 0;
    for (int32_t i = 0; i < n; i++) c0 += part[i] == 0;
    if (c0 != m) return 2;
    for (int32_t i = 0; i < n; i++) inside[i] = part[i] == 0;
  }
  // initialSolution: inside first, each side in ascending vertex id
  // (GPU-MDP-CSR.cu:479-499, GPU-MAXBS-CSR.cu:307-324).
  {
    int32_t x = 0, y = m;
    for (int32_t i = 0; i < n; i++) {
      if (inside[i]) { s.sol[x] = i; s.pos[i] = x; x++; }
      else { s.sol[y] = i; s.pos[i] = y; y++; }
    }
  }
  if (problem == OR_MDP) {
    // calculateVertexGain GPU-MDP-CSR.cu:502-519.
    for (int32_t i = 0; i < m; i++) {
      int32_t a = s.sol[i];
      for (int64_t k = g->rowptr[a]; k < g->rowptr[a + 1]; k++) s.vg[g->col[k]] += g->w[k];
    }
    s.cur = mdp_objective(g, inside);
  } else {
    // computeGainsFromScratch :208-219 and computeFitnessFromScratch :197-206.
    for (int32_t a = 0; a < n; a++) {
      int64_t same = 0, opp = 0;
      for (int64_t k = g->rowptr[a]; k < g->rowptr[a + 1]; k++) {
        if (part[g->col[k]] == part[a]) same += g->w[k]; else opp += g->w[k];
      }
      s.vg[a] = same - opp;
    }
    s.cur = maxbs_cut(g, part);
  }
  s.best = s.cur;
  if (part_out) *part_out = part;
  return 0;
}

extern "C" double or_sweep_sample(const or_graph* g, const or_params* p, const int32_t* initial,
                                  int32_t rows, int32_t sweeps, int64_t* pairs, int64_t* last_key,
                                  int64_t* last_idx) {
  State s;
  std::mt19937 rng;
  if (build_state(g, p, initial, s, rng, nullptr) != 0) return -1.0;
  if (rows < 1 || rows > s.m) rows = s.m;
  Best b{0, 0};
  double t0 = 0.0;
#ifdef _OPENMP
  t0 = omp_get_wtime();
#endif
  for (int32_t k = 0; k < sweeps; k++) b = sweep(s, p->problem, 0, p->threads, rows);
  double t1 = t0;
#ifdef _OPENMP
  t1 = omp_get_wtime();
#endif
  if (pairs) *pairs = (int64_t)rows * s.delta * sweeps;
  if (last_key) *last_key = b.key;
  if (last_idx) *last_idx = b.idx;
  return t1 - t0;
}

extern "C" int or_run(const or_graph* g, const or_params* p, const int32_t* initial,
                      or_result* res, or_trace_rec* trace, int64_t trace_cap,
                      int32_t* out_sol, int32_t* out_pos, int32_t* out_tab, int64_t* out_vg,
                      int32_t* out_best_sol) {
  State s;
  std::mt19937 rng;
  std::vector<int32_t> part;
  int rc0 = build_state(g, p, initial, s, rng, &part);
  if (rc0 != 0) return rc0;
  const int problem = p->problem;
  const int32_t n = s.n, m = s.m;
  s.best = s.cur;
  std::vector<int32_t> best_sol(s.sol.begin(), s.sol.end());

  // Perturbation draws continue the generator after the optional shuffle.
  const int32_t g_eff = std::min(p->gamma, n);
  const int32_t num_pert = std::max(1, g_eff / 2);  // :433-434
  std::vector<int64_t> draws(num_pert);

  int64_t ntr = 0;
  auto rec = [&](int64_t it, int64_t idx, int64_t key, int kind, int t1, int t2) {
    if (trace && ntr < trace_cap) {
      or_trace_rec& r = trace[ntr];
      r.iter = it; r.idx = idx; r.key = key; r.cur = s.cur; r.best = s.best;
      r.kind = kind; r.tenure = t1; r.tenure2 = t2; r.pad = 0;
    }
    ntr++;
  };

  int64_t iter = 0, evals = 0, isi = 0;
  int stopped = 0;
  while (iter < p->max_iter) {
    evals += s.P;
    Best b = sweep(s, problem, iter, p->threads);
    int32_t iu = (int32_t)(b.idx / s.delta);
    int32_t iv = (int32_t)(b.idx % s.delta) + m;
    if (problem == OR_MDP) {
      if (b.key == -99999) {  // :657-658
        rec(iter, b.idx, b.key, OR_REC_BREAK, 0, 0);
        stopped = 1;
        break;
      }
      s.cur += b.key;
      int32_t c1 = p->tenure_policy == OR_TENURE_REF ? or_mdp_tenure(iter) : p->tenure_fixed;
      int32_t c2 = or_mdp_c2(c1);
      mdp_apply(s, iu, iv, iter, c1, c2);
      if (s.cur > s.best) {  // :671-674
        s.best = s.cur;
        std::copy(s.sol.begin(), s.sol.begin() + m, best_sol.begin());
      }
      rec(iter, b.idx, b.key, OR_REC_MOVE, c1, c2);
      iter++;
    } else {
      // :456-460: penalised keys are recognised by magnitude, not by origin.
      if (b.key <= -2500000000LL) s.cur += b.key + 9999999999LL;
      else s.cur += b.key;
      int32_t tt = p->tenure_policy == OR_TENURE_REF ? or_maxbs_tenure(iter, p->maxt)
                                                     : p->tenure_fixed;
      maxbs_apply(s, iu, iv, iter, tt, 1);
      if (s.cur > s.best) {  // :469-476
        s.best = s.cur;
        best_sol = s.sol;
        isi = 0;
      } else {
        isi++;
      }
      rec(iter, b.idx, b.key, OR_REC_MOVE, tt, 0);
      iter++;
      if (isi >= p->piter) {  // :480-501
        perturb_event(rng, s.P, num_pert, draws.data());
        for (int32_t k = 0; k < num_pert; k++) {
          int32_t pu = (int32_t)(draws[k] / s.delta);
          int32_t pv = (int32_t)(draws[k] % s.delta) + m;
          int64_t aux = maxbs_apply(s, pu, pv, iter, 0, 0);
          s.cur += aux;
          rec(iter, draws[k], aux, OR_REC_PERTURB, 0, 0);
        }
        isi = 0;
      }
    }
  }

  if (res) {
    res->iterations = iter;
    res->evaluations = evals;
    res->cur = s.cur;
    res->best = s.best;
    res->n_trace = ntr;
    res->stopped = stopped;
    res->pad = 0;
    if (problem == OR_MDP) {
      std::vector<char> in(n, 0);
      for (int32_t i = 0; i < m; i++) in[best_sol[i]] = 1;
      res->best_true = mdp_objective(g, in);
    } else {
      std::vector<int32_t> bp(n, 1);
      for (int32_t i = 0; i < m; i++) bp[best_sol[i]] = 0;
      res->best_true = maxbs_cut(g, bp);
    }
  }
  if (out_sol) std::copy(s.sol.begin(), s.sol.end(), out_sol);
  if (out_pos) std::copy(s.pos.begin(), s.pos.end(), out_pos);
  if (out_tab) std::copy(s.tab.begin(), s.tab.end(), out_tab);
  if (out_vg) std::copy(s.vg.begin(), s.vg.end(), out_vg);
  if (out_best_sol) {
    int32_t cnt = problem == OR_MDP ? m : n;
    std::copy(best_sol.begin(), best_sol.begin() + cnt, out_best_sol);
  }
  return 0;
}
