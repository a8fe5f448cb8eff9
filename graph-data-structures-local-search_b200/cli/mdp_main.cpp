// mdp_main.cpp -- drop-in for the reference's mdp_<alg> programs
// (main, src/mdp/GPU-MDP-CSR.cu:1210-1300): same arguments, same stdout lines.
//
//   mdp_<alg> <instance> <dataset> <time_s> <repeats> [options]
//     dataset: MDG-a MDG-b MDG-c b2500 p30005000 nenad sparse
//   options this build adds (after the four positional arguments):
//     --seed S        trial r uses srand(S + r - 1) (default: time(NULL) per trial)
//     --gens G        G generations per trial, no time limit (deterministic runs)
//     --iters I       tabu iterations per search (default 50000)
//     --m M           selected-set size (default: the data set's)
//     --tenure ref|fixed:T
//     --alg NAME      lookup structure (default: from the program name)
//     --quiet         no per-search lines
//     --check-instance  print the parsed instance (n m edges scale weight-sum) and exit
#include <cmath>
#include <ctime>
#include <iomanip>
#include <iostream>

#include "common.h"
#include "instance.h"
#include "obma.h"

using namespace tscli;

int main(int argc, char** argv) {
  if (argc < 5) {
    std::cout << std::endl << "### Input the following parameters ###" << std::endl;
    std::cout << "Instance,data set,limit time,number of repeats" << std::endl;
    return 0;
  }
  const std::string instance_name = argv[1];
  const std::string dataset = argv[2];
  const double limit_time = std::atof(argv[3]);
  const int nbr_repeat = std::atoi(argv[4]);
  bool have_seed = false;
  unsigned seed = 0;
  ObmaConfig cfg;
  int32_t kind = struct_from_program(argv[0], "mdp");
  int32_t m_override = 0;
  bool check_only = false;
  try {
    for (int a = 5; a < argc; a++) {
      const std::string o = argv[a];
      auto next = [&]() -> std::string {
        if (a + 1 >= argc) throw std::runtime_error("missing value after " + o);
        return argv[++a];
      };
      if (o == "--seed") { seed = (unsigned)std::stoul(next()); have_seed = true; }
      else if (o == "--gens") cfg.max_generations = std::stoll(next());
      else if (o == "--iters") cfg.ts_iters = std::stoll(next());
      else if (o == "--m") m_override = std::stoi(next());
      else if (o == "--tenure") parse_tenure(next(), &cfg.tenure_policy, &cfg.tenure);
      else if (o == "--alg") kind = ts_struct_from_name(next().c_str());
      else if (o == "--quiet") cfg.verbose = false;
      else if (o == "--check-instance") check_only = true;
      else throw std::runtime_error("unknown option " + o);
    }
    if (kind < 0) kind = TS_STRUCT_CSR;
    if (nbr_repeat < 1) throw std::runtime_error("number of repeats must be >= 1");

    Instance I = read_mdp(instance_name, dataset);
    if (m_override > 0) I.m = m_override;
    if (check_only) {
      long long sum = 0;
      for (int32_t x : I.w) sum += x;
      std::printf("%d %d %zu %lld %lld %d\n", I.n, I.m, I.w.size(), (long long)I.scale, sum, I.rounded ? 1 : 0);
      return 0;
    }
    std::cout << "Dataset: " << dataset << std::endl;
    if (dataset.rfind("MDG", 0) == 0) std::cout << I.n << "-" << I.m << std::endl;
    const double density = (double)I.declared_edges / ((double)I.n * (I.n - 1) / 2.0);
    std::cout << "The statistics of the instance " << instance_name << std::endl;
    std::cout << "n = " << I.n << ", m = " << I.m << ", m/n = " << (float)I.m / (float)I.n
              << ", e = " << I.declared_edges << ", and density = " << density << std::endl;
    std::cout << "Finish loading data!" << std::endl;
    if (I.rounded) std::cerr << "warning: weights with more than 3 decimals were rounded" << std::endl;

    ts_graph* g = nullptr;
    check(ts_graph_create(I.n, (int64_t)I.u.size(), I.u.data(), I.v.data(), I.w.data(), kind, 1, nullptr, &g),
          "ts_graph_create");
    HostCSR csr(I.n, I.u, I.v, I.w, true);
    cfg.n = I.n;
    cfg.m = I.m;
    cfg.scale = I.scale;
    cfg.time_limit = limit_time;
    const double S = (double)I.scale;
    {
      Obma obma(cfg, csr, g);
      std::vector<double> costs;
      double avg_best_cost = 0, avg_best_time = 0, max_best_cost = -1, avg_min_best_time = 0;
      int nbr_success = 0;
      for (int r = 1; r <= nbr_repeat; r++) {
        const unsigned s = have_seed ? seed + (unsigned)(r - 1) : (unsigned)time(nullptr);
        ObmaStats st = obma.run(s);
        const double bc = (double)st.best_cost / S;
        std::printf("finish %d-th trial,nbr_gen = %lld,best_cost = %f,best_time = %f\n", r, (long long)st.nbr_gen,
                    bc, st.best_time);
        // check_and_store_result (:412-435): the set and its objective from the graph
        int64_t true_cost = 0;
        for (size_t i = 0; i < st.best_sol.size(); i++) {
          if (st.best_sol[i] < 0 || st.best_sol[i] >= I.n) {
            std::printf("### element:%d is out of range: %d-%d", st.best_sol[i], 0, I.n - 1);
            return 1;
          }
          for (size_t j = i + 1; j < st.best_sol.size(); j++) true_cost += csr.edge(st.best_sol[i], st.best_sol[j]);
        }
        if (true_cost != st.best_cost) {
          std::printf("Find a error solution: its sol_cost = %f, while its true_sol_ost =%f\n", bc,
                      (double)true_cost / S);
          return 1;
        }
        costs.push_back(bc);
        avg_best_cost += bc;
        avg_best_time += st.best_time;
        if (bc > max_best_cost) {
          max_best_cost = bc;
          avg_min_best_time = st.best_time;
          nbr_success = 1;
        } else if (std::fabs(bc - max_best_cost) < 0.1) {
          nbr_success++;
          avg_min_best_time += st.best_time;
        }
      }
      const double avg_iterations = (double)obma.total_iterations / nbr_repeat;
      const double avg_evaluations = (double)obma.total_evaluations / nbr_repeat;
      avg_best_cost /= nbr_repeat;
      avg_best_time /= nbr_repeat;
      avg_min_best_time /= nbr_success;
      double sd = 0;
      for (double c : costs) sd += (c - avg_best_cost) * (c - avg_best_cost);
      sd = std::sqrt(sd / nbr_repeat);
      const double gap = max_best_cost - avg_best_cost;
      std::printf("---------------------------------------------------------\n");
      std::printf("%.3lf, %.3lf\n", avg_best_cost, avg_best_time);
      std::printf("---------------------------------------------------------\n");
      std::printf("%.3lf, %.3lf, %.3lf, %.3lf, %d, %.3lf, %3lf\n", max_best_cost, avg_min_best_time, gap, sd,
                  nbr_success, avg_evaluations, avg_evaluations);
      std::fflush(stdout);
      std::cout << "finishing...!" << std::endl;
      std::cout << "found best objective = " << std::setprecision(10) << max_best_cost << std::endl;
      std::cout << "number of times to find the best solution = " << nbr_success << std::endl;
      std::cout << "average value of the best objective value = " << std::setprecision(10) << avg_best_cost << std::endl;
      std::cout << "average value of the best time (second) = " << std::setprecision(10) << avg_best_time << std::endl;
      std::cout << "average number of iterations per run = " << std::setprecision(10) << avg_iterations << std::endl;
      std::cout << "average number of evaluations per run = " << std::setprecision(10) << avg_evaluations
                << std::endl;
    }
    ts_graph_destroy(g);
  } catch (const std::exception& e) {
    std::fflush(stdout);
    std::cerr << e.what() << std::endl;
    return 1;
  }
  return 0;
}
