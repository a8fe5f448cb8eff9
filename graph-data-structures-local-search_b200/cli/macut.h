// macut.h -- memetic algorithm for Max Bisection (MACUT), the host driver of
// the reference's maxbs_<alg> programs (src/maxbisection/GPU-MAXBS-CSR.cu:514-732),
// calling the B200 perturbation-based tabu search through the C-ABI.  One
// mt19937 drives everything, as in the reference: starts, recombination,
// repairs and every search's perturbation moves (handed to the device search
// with ts_solver_set_perturbations).
#pragma once
#include <cstdint>
#include <random>
#include <vector>

#include "common.h"

namespace tscli {

struct MacutConfig {
  int32_t n = 0;
  int64_t scale = 1;
  int32_t p = 10;
  int32_t piter = 500;
  int32_t gamma = 150;
  int64_t max_iter = 1000000;
  int32_t maxt = 200;
  double time_limit = 60.0;
  unsigned seed = 0;
  int32_t tenure_policy = TS_TENURE_REF;
  int32_t tenure = 25;
  int64_t max_generations = 0;  // > 0: that many generations, time ignored
};

struct MaxbsSolution {
  std::vector<int32_t> part;  // 0: first subset (floor(n/2) vertices), 1: second
  int64_t fitness = 0;
};

class Macut {
 public:
  Macut(const MacutConfig& cfg, const HostCSR& csr, ts_graph* g);
  ~Macut();
  MaxbsSolution run(int64_t* generations);
  int64_t fitness_of(const std::vector<int32_t>& part) const;  // computeFitnessFromScratch
  double elapsed() const { return clock_.seconds(); }
  int64_t iterations_count = 0;
  int64_t evaluations_count = 0;

 private:
  MacutConfig c_;
  const HostCSR& csr_;
  ts_solver* solver_ = nullptr;
  std::mt19937 rng_;
  Stopwatch clock_;
  int32_t m_ = 0, k_ = 1;
  int64_t P_ = 0;

  bool time_up() const;
  int rand_int(int lo, int hi);
  void random_partition(MaxbsSolution& s);
  MaxbsSolution pbts(const MaxbsSolution& start);
  void apply_random_swap(MaxbsSolution& s);
  std::vector<MaxbsSolution> generate_population();
  void repair(MaxbsSolution& s);
  MaxbsSolution recombination(const std::vector<const MaxbsSolution*>& parents);
  void pool_update(const MaxbsSolution& off, std::vector<MaxbsSolution>& pop);
};

// One perturbation event of k distinct flat move indices from `rng`
// (GPU-MAXBS-CSR.cu:481-492); past the int range the draw is 64-bit.
void perturbation_event(std::mt19937& rng, int64_t P, int k, std::vector<int64_t>& out);

}  // namespace tscli
