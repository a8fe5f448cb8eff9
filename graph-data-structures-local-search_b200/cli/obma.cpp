// obma.cpp -- OBMA host driver (see obma.h).  Each function names the
// reference function it restates; the random calls come in the same order.
#include "obma.h"

#include <algorithm>

namespace tscli {

namespace {

int64_t absdiff(int64_t a, int64_t b) { return a > b ? a - b : b - a; }

// calculate_rank(0, ...) (GPU-MDP-CSR.cu:153-207): rank = 1 + place in the
// ascending order; equal values take consecutive ranks in index order.
template <class T>
void calculate_rank(const std::vector<T>& a, std::vector<int>& b) {
  const int nbr = (int)a.size();
  std::vector<T> c = a;
  for (int i = 1; i < nbr; i++)
    for (int j = nbr - 1; j >= i; j--)
      if (c[j - 1] > c[j]) std::swap(c[j - 1], c[j]);
  std::vector<int> flag(nbr, 0);
  b.assign(nbr, 0);
  for (int i = 0; i < nbr; i++)
    for (int j = 0; j < nbr; j++)
      if (flag[j] == 0 && a[i] == c[j]) {
        b[i] = j + 1;
        flag[j] = 1;
        break;
      }
}

}  // namespace

Obma::Obma(const ObmaConfig& cfg, const HostCSR& csr, ts_graph* g) : c_(cfg), csr_(csr) {
  if (2LL * c_.m > c_.n)
    throw std::runtime_error("OBMA needs m <= n/2 (its opposite solutions take m of the n-m others)");
  ts_params p;
  check(ts_params_default(TS_PROBLEM_MDP, &p), "ts_params_default");
  p.m = c_.m;
  p.max_iter = c_.ts_iters;
  p.tenure_policy = c_.tenure_policy;
  p.tenure = c_.tenure;
  check(ts_solver_create(g, &p, &solver_), "ts_solver_create");
  eps_ = 99999LL * c_.scale;
  vertex_.assign(c_.n, 0);
  pop_.assign(PS + 1, std::vector<int32_t>(c_.m));
  pop_cost_.assign(PS + 1, 0);
  dist_.assign(PS + 1, std::vector<float>(PS + 1, 0.0f));
  pop_distance_.assign(PS + 1, 0.0f);
  pop_score_.assign(PS + 1, 0.0f);
}

Obma::~Obma() {
  if (solver_) ts_solver_destroy(solver_);
}

bool Obma::time_up() const {
  if (c_.max_generations > 0) return false;
  return clock_.seconds() >= c_.time_limit;
}

// tabu_search (:611-693) on the device; improved_* = the best of the search.
void Obma::tabu_search(const std::vector<int32_t>& sol) {
  Stopwatch tw;
  check(ts_solver_init(solver_, sol.data()), "ts_solver_init");
  int64_t done = 0;
  if (c_.max_generations > 0) {
    check(ts_solver_step(solver_, c_.ts_iters, &done), "ts_solver_step");
  } else {
    // the reference stops a search once the trial's time is over (:679-680)
    while (done < c_.ts_iters) {
      const int64_t k = std::min<int64_t>(1000, c_.ts_iters - done);
      int64_t d = 0;
      check(ts_solver_step(solver_, k, &d), "ts_solver_step");
      done += d;
      if (d < k || clock_.seconds() > c_.time_limit) break;
    }
  }
  ts_result r;
  improved_sol_.assign(c_.m, 0);
  check(ts_solver_result(solver_, &r, improved_sol_.data()), "ts_solver_result");
  improved_cost_ = r.best;
  improved_time_ = clock_.seconds();
  total_iterations += r.iterations;
  total_evaluations += r.evaluations;
  if (c_.verbose && r.iterations > 1)
    std::printf("Iteracoes: %lld\tTime Tabu: %.10lf\tSol: %.10lf\n", (long long)r.iterations, tw.seconds(),
                (double)improved_cost_ / (double)c_.scale);
}

// ascend_sort (:741-752); leaves vertex_ marking the set.
void Obma::ascend_sort(std::vector<int32_t>& sol) {
  std::fill(vertex_.begin(), vertex_.end(), 0);
  for (int32_t v : sol) vertex_[v] = 1;
  int32_t cnt = 0;
  for (int32_t i = 0; i < c_.n; i++)
    if (vertex_[i] == 1) sol[cnt++] = i;
}

// is_duplicate_sol (:696-713)
bool Obma::is_duplicate(int index) const {
  for (int i = 0; i < index; i++)
    if (pop_[i] == improved_sol_) return true;
  return false;
}

// calculate_sol_distance (:716-738)
float Obma::distance(int x1, int x2) const {
  int u = 0, v = 0, sharing = 0;
  const std::vector<int32_t>& a = pop_[x1];
  const std::vector<int32_t>& b = pop_[x2];
  while (u < c_.m && v < c_.m) {
    if (a[u] == b[v]) { sharing++; u++; v++; }
    else if (a[u] < b[v]) u++;
    else v++;
  }
  return 1 - (float)sharing / (float)c_.m;
}

void Obma::update_best() {  // update_best_sol (:446-452)
  best_time_ = improved_time_;
  best_cost_ = improved_cost_;
  best_sol_ = improved_sol_;
}

// build_pool_with_OBL (:755-896)
void Obma::build_pool() {
  const int32_t n = c_.n, m = c_.m, delta = n - m;
  std::vector<int32_t> sol, opp, elite;
  best_cost_ = -1;
  int nbr_sol = 0;
  while (nbr_sol < PS) {
    std::fill(vertex_.begin(), vertex_.end(), 0);
    sol.clear();
    while ((int32_t)sol.size() < m) {
      const int32_t idx = rnd_.next() % n;
      if (vertex_[idx] == 0) {
        sol.push_back(idx);
        vertex_[idx] = 1;
      }
    }
    tabu_search(sol);
    ascend_sort(improved_sol_);
    const int64_t elite_cost = improved_cost_;
    elite = improved_sol_;
    opp.clear();
    if (delta != m) {
      std::vector<int32_t> avail;
      for (int32_t i = 0; i < n; i++)
        if (vertex_[i] == 0) avail.push_back(i);
      int32_t nav = (int32_t)avail.size();
      while ((int32_t)opp.size() < m) {
        const int32_t idx = rnd_.next() % nav;
        opp.push_back(avail[idx]);
        nav--;
        avail[idx] = avail[nav];
      }
    } else {
      for (int32_t i = 0; i < n; i++)
        if (vertex_[i] == 0) opp.push_back(i);
    }
    tabu_search(opp);
    ascend_sort(improved_sol_);
    if (improved_cost_ < elite_cost || (absdiff(improved_cost_, elite_cost) < eps_ && rnd_.next() % 2 == 0)) {
      improved_cost_ = elite_cost;
      improved_sol_ = elite;
    }
    std::fill(vertex_.begin(), vertex_.end(), 0);
    for (int32_t v : improved_sol_) vertex_[v] = 1;
    while (is_duplicate(nbr_sol)) {  // move one element until the solution is new
      const int32_t index = rnd_.next() % m;
      const int32_t out = improved_sol_[index];
      int64_t out_gain = 0;
      for (int32_t x : improved_sol_)
        if (x != out) out_gain += csr_.edge(x, out);
      int32_t in;
      do {
        in = rnd_.next() % n;
      } while (vertex_[in] != 0);
      int64_t in_gain = 0;
      for (int32_t x : improved_sol_)
        if (x != out) in_gain += csr_.edge(x, in);
      vertex_[in] = 1;
      vertex_[out] = 0;
      improved_sol_[index] = in;
      improved_cost_ += in_gain - out_gain;
      ascend_sort(improved_sol_);
    }
    pop_cost_[nbr_sol] = improved_cost_;
    pop_[nbr_sol] = improved_sol_;
    nbr_sol++;
    if (improved_cost_ > best_cost_) update_best();
  }
  for (int i = 0; i < PS; i++) {
    for (int j = i + 1; j < PS; j++) {
      dist_[i][j] = distance(i, j);
      dist_[j][i] = dist_[i][j];
    }
    dist_[i][i] = 0.0f;
  }
}

// crossover_with_greedy (:899-1060)
void Obma::crossover() {
  const int32_t n = c_.n, m = c_.m, delta = n - m;
  int p[NP];
  int is_choose[PS] = {0};
  int nbr_p = 0;
  while (nbr_p < NP) {
    const int cp = rnd_.next() % PS;
    if (is_choose[cp] == 0) {
      p[nbr_p++] = cp;
      is_choose[cp] = 1;
    }
  }
  std::fill(vertex_.begin(), vertex_.end(), 0);
  for (int i = 0; i < NP; i++)
    for (int32_t v : pop_[p[i]]) vertex_[v]++;
  std::vector<int32_t> remaining[NP];
  for (int i = 0; i < NP; i++)
    for (int32_t v : pop_[p[i]])
      if (vertex_[v] == 1) {
        remaining[i].push_back(v);
        vertex_[v] = 0;
      }
  offspring_.clear();
  for (int32_t i = 0; i < n; i++)
    if (vertex_[i] == NP) {
      offspring_.push_back(i);
      vertex_[i] = 1;
    }
  std::vector<int32_t> best_idx;
  while ((int32_t)offspring_.size() < m) {
    const int ip = (int)(offspring_.size() % NP);
    int64_t max_profit = INT32_MIN;
    best_idx.clear();
    for (int32_t i = 0; i < (int32_t)remaining[ip].size(); i++) {
      int64_t profit = 0;
      for (int32_t x : offspring_) profit += csr_.edge(remaining[ip][i], x);
      if (profit > max_profit) {
        max_profit = profit;
        best_idx.assign(1, i);
      } else if (absdiff(profit, max_profit) < eps_) {
        best_idx.push_back(i);
      }
    }
    const int32_t irv = best_idx[rnd_.next() % (int)best_idx.size()];
    const int32_t cv = remaining[ip][irv];
    offspring_.push_back(cv);
    vertex_[cv] = 1;
    remaining[ip][irv] = remaining[ip].back();
    remaining[ip].pop_back();
  }
  opposite_.clear();
  if (delta > m) {
    std::vector<int32_t> avail;
    for (int32_t i = 0; i < n; i++)
      if (vertex_[i] == 0) avail.push_back(i);
    int32_t nav = (int32_t)avail.size();
    while ((int32_t)opposite_.size() < m) {
      const int32_t idx = rnd_.next() % nav;
      opposite_.push_back(avail[idx]);
      nav--;
      avail[idx] = avail[nav];
    }
  } else {
    for (int32_t i = 0; i < n; i++)
      if (vertex_[i] == 0) opposite_.push_back(i);
  }
}

// rank_based_pool_updating (:1062-1140)
void Obma::pool_update() {
  pop_cost_[PS] = improved_cost_;
  pop_[PS] = improved_sol_;
  for (int i = 0; i < PS; i++) {
    dist_[i][PS] = distance(i, PS);
    dist_[PS][i] = dist_[i][PS];
  }
  dist_[PS][PS] = 0.0f;
  for (int i = 0; i < PS + 1; i++) {
    float avg = 0.0f;
    for (int j = 0; j < PS + 1; j++)
      if (j != i) avg += dist_[i][j];
    pop_distance_[i] = avg / PS;
  }
  std::vector<int> cost_rank, distance_rank;
  calculate_rank(pop_cost_, cost_rank);
  calculate_rank(pop_distance_, distance_rank);
  for (int i = 0; i < PS + 1; i++)
    pop_score_[i] = (float)(ALPHA * cost_rank[i] + (1.0 - ALPHA) * distance_rank[i]);
  float min_score = (float)INT32_MAX;
  int worst = 0;
  for (int i = 0; i < PS + 1; i++)
    if (pop_score_[i] < min_score) {
      min_score = pop_score_[i];
      worst = i;
    }
  if (worst != PS && !is_duplicate(PS)) {
    pop_cost_[worst] = improved_cost_;
    pop_[worst] = improved_sol_;
    for (int i = 0; i < PS; i++) {
      dist_[i][worst] = dist_[PS][i];
      dist_[worst][i] = dist_[i][worst];
    }
    dist_[worst][worst] = 0.0f;
  }
}

// OBMA (:1143-1208)
ObmaStats Obma::run(unsigned seed) {
  rnd_.reseed(seed);
  clock_.reset();
  int64_t nbr_gen = 0;
  best_cost_ = -1;
  best_time_ = 0;
  std::printf("using OBL!!!\n");
  build_pool();
  for (;;) {
    crossover();
    tabu_search(offspring_);
    ascend_sort(improved_sol_);
    if (improved_cost_ > best_cost_) update_best();
    pool_update();
    tabu_search(opposite_);
    ascend_sort(improved_sol_);
    if (improved_cost_ > best_cost_) update_best();
    pool_update();
    if (c_.max_generations > 0) {
      if (nbr_gen + 1 >= c_.max_generations) break;
    } else if (time_up()) {
      break;
    }
    nbr_gen++;
  }
  ObmaStats s;
  s.best_cost = best_cost_;
  s.best_time = best_time_;
  s.nbr_gen = nbr_gen;
  s.best_sol = best_sol_;
  return s;
}

}  // namespace tscli
