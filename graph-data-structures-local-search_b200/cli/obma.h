// obma.h -- opposition-based memetic algorithm (OBMA) for the Maximum
// Diversity Problem, the host driver of the reference's mdp_<alg> programs
// (src/mdp/GPU-MDP-CSR.cu:696-1208), calling the B200 tabu search through the
// C-ABI.  Integer objectives; the reference's tie tolerance `epsilon` (99999,
// :50) is kept, in weight units times the instance scale.
#pragma once
#include <cstdint>
#include <vector>

#include "common.h"

namespace tscli {

struct ObmaConfig {
  int32_t n = 0, m = 0;
  int64_t scale = 1;
  int64_t ts_iters = 50000;          // max_iter of tabu_search (:55)
  int32_t tenure_policy = TS_TENURE_REF;
  int32_t tenure = 15;
  double time_limit = 60.0;          // seconds for one trial
  int64_t max_generations = 0;       // > 0: stop after that many generations, ignore time
  bool verbose = true;               // per-search "Iteracoes" lines
};

struct ObmaStats {
  int64_t best_cost = -1;
  double best_time = 0;
  int64_t nbr_gen = 0;
  std::vector<int32_t> best_sol;     // ascending ids
};

class Obma {
 public:
  Obma(const ObmaConfig& cfg, const HostCSR& csr, ts_graph* g);
  ~Obma();
  // One trial from srand(seed); the iteration/evaluation counters accumulate
  // over trials like the reference's globals.
  ObmaStats run(unsigned seed);
  int64_t total_iterations = 0;
  int64_t total_evaluations = 0;

 private:
  static constexpr int PS = 10;   // population size (:52)
  static constexpr int NP = 2;    // parents (:51)
  static constexpr int ALPHA = 15;  // score weight (:53)
  ObmaConfig c_;
  const HostCSR& csr_;
  ts_solver* solver_ = nullptr;
  GlibcRand rnd_{1};
  Stopwatch clock_;
  int64_t eps_;
  std::vector<int32_t> vertex_, improved_sol_, best_sol_, offspring_, opposite_;
  int64_t improved_cost_ = 0, best_cost_ = -1;
  double improved_time_ = 0, best_time_ = 0;
  std::vector<std::vector<int32_t>> pop_;
  std::vector<int64_t> pop_cost_;
  std::vector<std::vector<float>> dist_;
  std::vector<float> pop_distance_, pop_score_;

  bool time_up() const;
  void tabu_search(const std::vector<int32_t>& sol);
  void ascend_sort(std::vector<int32_t>& sol);
  bool is_duplicate(int index) const;
  float distance(int x1, int x2) const;
  void update_best();
  void build_pool();
  void crossover();
  void pool_update();
};

}  // namespace tscli
