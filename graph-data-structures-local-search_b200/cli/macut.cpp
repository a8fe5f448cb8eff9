// macut.cpp -- MACUT host driver (see macut.h).  Each function names the
// reference function it restates; the generator calls come in the same order.
#include "macut.h"

#include <algorithm>
#include <iomanip>
#include <iostream>
#include <numeric>
#include <unordered_set>

namespace tscli {

void perturbation_event(std::mt19937& rng, int64_t P, int k, std::vector<int64_t>& out) {
  std::unordered_set<int64_t> used;
  for (int q = 0; q < k; q++) {
    int64_t mv;
    do {
      if (P - 1 <= INT32_MAX) {
        std::uniform_int_distribution<int> d(0, (int)(P - 1));
        mv = d(rng);
      } else {
        std::uniform_int_distribution<int64_t> d(0, P - 1);
        mv = d(rng);
      }
    } while (used.count(mv));
    used.insert(mv);
    out.push_back(mv);
  }
}

Macut::Macut(const MacutConfig& cfg, const HostCSR& csr, ts_graph* g) : c_(cfg), csr_(csr) {
  m_ = c_.n / 2;
  P_ = (int64_t)m_ * (c_.n - m_);
  k_ = std::max(1, std::min(c_.gamma, c_.n) / 2);
  const int64_t events = c_.max_iter / std::max(1, c_.piter) + 1;
  if (events * k_ > (1LL << 26))
    throw std::runtime_error("-maxiter / -piter asks for more than 2^26 perturbation moves per search");
  ts_params p;
  check(ts_params_default(TS_PROBLEM_MAXBS, &p), "ts_params_default");
  p.max_iter = c_.max_iter;
  p.piter = c_.piter;
  p.gamma = c_.gamma;
  p.maxt = c_.maxt;
  p.tenure_policy = c_.tenure_policy;
  p.tenure = c_.tenure;
  p.seed = c_.seed;
  check(ts_solver_create(g, &p, &solver_), "ts_solver_create");
}

Macut::~Macut() {
  if (solver_) ts_solver_destroy(solver_);
}

bool Macut::time_up() const {
  if (c_.max_generations > 0) return false;
  return clock_.seconds() >= c_.time_limit;
}

int Macut::rand_int(int lo, int hi) {  // randInt (:48-51)
  std::uniform_int_distribution<int> d(lo, hi);
  return d(rng_);
}

void Macut::random_partition(MaxbsSolution& s) {  // randomPartition (:187-195)
  std::vector<int> vertices(c_.n);
  std::iota(vertices.begin(), vertices.end(), 0);
  std::shuffle(vertices.begin(), vertices.end(), rng_);
  s.part.assign(c_.n, 1);
  for (int i = 0; i < m_; i++) s.part[vertices[i]] = 0;
}

int64_t Macut::fitness_of(const std::vector<int32_t>& part) const {  // :196-205
  int64_t f = 0;
  for (int32_t v = 0; v < c_.n; v++)
    for (int64_t k = csr_.rowptr[v]; k < csr_.rowptr[v + 1]; k++) {
      const int32_t u = csr_.col[k];
      if (u > v && part[u] != part[v]) f += csr_.w[k];
    }
  return f;
}

// perturbationBasedTabuSearch (:401-512) on the device.  Its perturbation
// moves are drawn here from a copy of the generator; afterwards the generator
// advances by exactly the events the search used.
MaxbsSolution Macut::pbts(const MaxbsSolution& start) {
  check(ts_solver_init(solver_, start.part.data()), "ts_solver_init");
  const int64_t events = c_.max_iter / std::max(1, c_.piter) + 1;
  std::vector<int64_t> draws;
  draws.reserve((size_t)(events * k_));
  std::mt19937 probe = rng_;
  for (int64_t e = 0; e < events; e++) perturbation_event(probe, P_, k_, draws);
  check(ts_solver_set_perturbations(solver_, draws.data(), events), "ts_solver_set_perturbations");
  if (c_.max_generations > 0) {
    check(ts_solver_step(solver_, c_.max_iter, nullptr), "ts_solver_step");
  } else {
    int64_t done = 0;
    while (done < c_.max_iter && !time_up()) {  // the reference checks timeUp every iteration
      const int64_t k = std::min<int64_t>(1000, c_.max_iter - done);
      int64_t d = 0;
      check(ts_solver_step(solver_, k, &d), "ts_solver_step");
      done += d;
      if (d < k) break;
    }
  }
  ts_result r;
  MaxbsSolution best;
  best.part.assign(c_.n, 0);
  check(ts_solver_result(solver_, &r, best.part.data()), "ts_solver_result");
  best.fitness = r.best;
  iterations_count += r.iterations;
  evaluations_count += r.evaluations;
  std::vector<int64_t> scratch;
  for (int64_t e = 0; e < r.perturbations / k_; e++) perturbation_event(rng_, P_, k_, scratch);
  return best;
}

static bool same_partition(const MaxbsSolution& a, const MaxbsSolution& b) {  // samePartition (:514-521)
  bool eq = true, comp = true;
  for (size_t i = 0; i < a.part.size(); i++) {
    if (a.part[i] != b.part[i]) eq = false;
    if (a.part[i] == b.part[i]) comp = false;
  }
  return eq || comp;
}

void Macut::apply_random_swap(MaxbsSolution& s) {  // applyRandomSwap (:283-291)
  const int n = (int)s.part.size();
  const int u = rand_int(0, n - 1);
  int v = rand_int(0, n - 1);
  while (s.part[v] == s.part[u]) v = rand_int(0, n - 1);
  std::swap(s.part[u], s.part[v]);
  s.fitness = fitness_of(s.part);
}

// generatePopulation (:523-575)
std::vector<MaxbsSolution> Macut::generate_population() {
  std::vector<MaxbsSolution> candidates;
  const int p = c_.p;
  int attempts = 0;
  const int max_attempts = 20 * p + 100;
  while ((int)candidates.size() < 2 * p && attempts < max_attempts && !time_up()) {
    attempts++;
    MaxbsSolution start;
    random_partition(start);
    MaxbsSolution local = pbts(start);
    bool dup = false;
    for (auto& c : candidates)
      if (same_partition(c, local)) {
        dup = true;
        break;
      }
    if (!dup) candidates.push_back(local);
  }
  std::sort(candidates.begin(), candidates.end(),
            [](const MaxbsSolution& a, const MaxbsSolution& b) { return a.fitness > b.fitness; });
  const int keep = std::min((int)candidates.size(), p);
  std::vector<MaxbsSolution> pop(candidates.begin(), candidates.begin() + keep);
  while ((int)pop.size() < 2 && !pop.empty()) {
    MaxbsSolution clone = pop[0];
    if (c_.n > 1) apply_random_swap(clone);
    pop.push_back(clone);
  }
  if (pop.empty()) {
    MaxbsSolution s;
    random_partition(s);
    s.fitness = fitness_of(s.part);
    pop.push_back(s);
    MaxbsSolution s2 = s;
    if (c_.n > 1) apply_random_swap(s2);
    pop.push_back(s2);
  }
  return pop;
}

void Macut::repair(MaxbsSolution& s) {  // repairBisection (:577-602)
  const int n = (int)s.part.size(), k = n / 2;
  std::vector<int> S1, S2;
  for (int v = 0; v < n; v++) (s.part[v] == 0 ? S1 : S2).push_back(v);
  std::shuffle(S1.begin(), S1.end(), rng_);
  std::shuffle(S2.begin(), S2.end(), rng_);
  while ((int)S1.size() > k) {
    const int v = S1.back();
    S1.pop_back();
    s.part[v] = 1;
    S2.push_back(v);
  }
  while ((int)S1.size() < k) {
    const int v = S2.back();
    S2.pop_back();
    s.part[v] = 0;
    S1.push_back(v);
  }
}

// recombination (:604-657)
MaxbsSolution Macut::recombination(const std::vector<const MaxbsSolution*>& parents) {
  const int n = c_.n, m = (int)parents.size();
  std::vector<char> assigned(n, 0);
  MaxbsSolution off;
  off.part.assign(n, 0);
  auto build_side = [&](int side) {
    int best_count = -1, best_combo = 0;
    for (int combo = 0; combo < (1 << m); combo++) {
      int cnt = 0;
      for (int v = 0; v < n; v++) {
        if (assigned[v]) continue;
        bool all = true;
        for (int i = 0; i < m; i++)
          if (parents[i]->part[v] != ((combo >> i) & 1)) {
            all = false;
            break;
          }
        if (all) cnt++;
      }
      if (cnt > best_count) {
        best_count = cnt;
        best_combo = combo;
      }
    }
    for (int v = 0; v < n; v++) {
      if (assigned[v]) continue;
      bool all = true;
      for (int i = 0; i < m; i++)
        if (parents[i]->part[v] != ((best_combo >> i) & 1)) {
          all = false;
          break;
        }
      if (all) {
        off.part[v] = side;
        assigned[v] = 1;
      }
    }
  };
  build_side(0);
  build_side(1);
  for (int v = 0; v < n; v++)
    if (!assigned[v]) off.part[v] = rand_int(0, 1);
  repair(off);
  off.fitness = fitness_of(off.part);
  return off;
}

void Macut::pool_update(const MaxbsSolution& off, std::vector<MaxbsSolution>& pop) {  // poolUpdating (:659-670)
  for (auto& s : pop)
    if (same_partition(s, off)) return;
  int worst = 0;
  for (size_t i = 1; i < pop.size(); i++)
    if (pop[i].fitness < pop[worst].fitness) worst = (int)i;
  if (off.fitness > pop[worst].fitness) pop[worst] = off;
}

// macut (:672-732)
MaxbsSolution Macut::run(int64_t* generations) {
  clock_.reset();
  rng_.seed(c_.seed);
  std::cerr << "[MACUT] Gerando populacao inicial (p=" << c_.p << ")...\n";
  std::vector<MaxbsSolution> pop = generate_population();
  MaxbsSolution best = *std::max_element(pop.begin(), pop.end(), [](const MaxbsSolution& a, const MaxbsSolution& b) {
    return a.fitness < b.fitness;
  });
  std::cerr << "[MACUT] Melhor da populacao inicial: f = " << std::fixed << std::setprecision(3)
            << (double)best.fitness / (double)c_.scale << "\n";
  int64_t gen = 0;
  for (;;) {
    if (c_.max_generations > 0 ? gen >= c_.max_generations : time_up()) break;
    gen++;
    const int max_m = std::min(4, (int)pop.size());
    const int m = max_m >= 2 ? rand_int(2, max_m) : max_m;
    std::vector<int> idx(pop.size());
    std::iota(idx.begin(), idx.end(), 0);
    std::shuffle(idx.begin(), idx.end(), rng_);
    std::vector<const MaxbsSolution*> parents;
    for (int i = 0; i < m; i++) parents.push_back(&pop[idx[i]]);
    MaxbsSolution off = recombination(parents);
    MaxbsSolution improved = pbts(off);
    if (improved.fitness > best.fitness) {
      best = improved;
      std::cerr << "[MACUT] Geracao " << gen << " | nova melhor solucao: f = "
                << (double)best.fitness / (double)c_.scale << " | t = " << std::fixed << std::setprecision(1)
                << elapsed() << "s\n";
    }
    pool_update(improved, pop);
  }
  *generations = gen;
  return best;
}

}  // namespace tscli
