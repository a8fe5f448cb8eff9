// maxbs_main.cpp -- drop-in for the reference's maxbs_<alg> programs
// (main, src/maxbisection/GPU-MAXBS-CSR.cu:734-808): same options, same output.
//
//   maxbs_<alg> <graph> [-p P] [-piter I] [-gamma G] [-maxiter N] [-maxt T]
//               [-time S] [-seed X] [-out FILE]
//   options this build adds:
//     -gens G          G generations, no time limit (deterministic runs)
//     -tenure ref|fixed:T
//     -alg NAME        lookup structure (default: from the program name)
//     -check-instance  print the parsed instance (n m edges scale weight-sum) and exit
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>

#include "common.h"
#include "instance.h"
#include "macut.h"

using namespace tscli;

static void usage(const char* prog) {
  std::cerr << "Uso: " << prog << " <arquivo_grafo> [opcoes]\n"
            << "  -p <int>        tamanho da populacao          (default 10)\n"
            << "  -piter <int>    Piter                          (default 500)\n"
            << "  -gamma <int>    forca da perturbacao           (default 150)\n"
            << "  -maxiter <long> MaxIter da busca tabu           (default 1000000)\n"
            << "  -maxt <int>     maxt                             (default time(200))\n"
            << "  -time <double>  tempo limite total em segundos (default 60)\n"
            << "  -seed <int>     semente aleatoria               (default time(0))\n"
            << "  -out <file>     grava a melhor particao encontrada\n"
            << "  -gens <int>     numero de geracoes, sem limite de tempo\n"
            << "  -tenure ref|fixed:T\n"
            << "  -alg <nome>     csr hash wswap csr-bitset csr-bb csr-bitset-bb\n";
}

int main(int argc, char** argv) {
  std::ios::sync_with_stdio(false);
  if (argc < 2) {
    usage(argv[0]);
    return 1;
  }
  MacutConfig cfg;
  cfg.seed = (unsigned)time(nullptr);
  std::string out_file;
  int32_t kind = struct_from_program(argv[0], "maxbs");
  bool check_only = false;
  try {
    Instance I = read_maxbs(argv[1]);
    for (int a = 2; a < argc; a++) {
      const std::string o = argv[a];
      auto next = [&]() -> std::string {
        if (a + 1 >= argc) throw std::runtime_error("missing value after " + o);
        return argv[++a];
      };
      if (o == "-p") cfg.p = std::stoi(next());
      else if (o == "-piter") cfg.piter = std::stoi(next());
      else if (o == "-gamma") cfg.gamma = std::stoi(next());
      else if (o == "-maxiter") cfg.max_iter = std::stoll(next());
      else if (o == "-maxt") cfg.maxt = std::stoi(next());
      else if (o == "-time") cfg.time_limit = std::stod(next());
      else if (o == "-seed") cfg.seed = (unsigned)std::stoul(next());
      else if (o == "-out") out_file = next();
      else if (o == "-gens") cfg.max_generations = std::stoll(next());
      else if (o == "-tenure") parse_tenure(next(), &cfg.tenure_policy, &cfg.tenure);
      else if (o == "-alg") kind = ts_struct_from_name(next().c_str());
      else if (o == "-check-instance") check_only = true;
      else {
        std::cerr << "Opcao desconhecida: " << o << "\n";
        usage(argv[0]);
        return 1;
      }
    }
    if (check_only) {
      long long sum = 0;
      for (int32_t x : I.w) sum += x;
      std::printf("%d %d %zu %lld %lld %d\n", I.n, I.m, I.w.size(), (long long)I.scale, sum, I.rounded ? 1 : 0);
      return 0;
    }
    if (kind < 0) kind = TS_STRUCT_CSR;
    if (cfg.p < 1 || cfg.piter < 1 || cfg.maxt < 1 || cfg.max_iter < 0 || cfg.gamma < 0)
      throw std::runtime_error("parameters must be positive");
    if (I.rounded) std::cerr << "warning: weights with more than 3 decimals were rounded\n";
    std::cerr << "[MACUT] Grafo: n=" << I.n << ", m=" << I.declared_edges << "\n";
    std::cerr << "[MACUT] Parametros: p=" << cfg.p << " Piter=" << cfg.piter << " gamma=" << cfg.gamma
              << " MaxIter=" << cfg.max_iter << " maxt=" << cfg.maxt << " time=" << cfg.time_limit
              << "s seed=" << cfg.seed << "\n";
    ts_graph* g = nullptr;
    check(ts_graph_create(I.n, (int64_t)I.u.size(), I.u.data(), I.v.data(), I.w.data(), kind, 0, nullptr, &g),
          "ts_graph_create");
    HostCSR csr(I.n, I.u, I.v, I.w, false);
    cfg.n = I.n;
    cfg.scale = I.scale;
    const double S = (double)I.scale;
    {
      Macut macut(cfg, csr, g);
      int64_t generations = 0;
      MaxbsSolution best = macut.run(&generations);
      // The search's bookkeeping follows the reference's, whose recovery of a
      // penalised move's gain (GPU-MAXBS-CSR.cu:456-460) is quantised by float
      // rounding; the independent check recomputes the cut from the graph.
      const int64_t verify = macut.fitness_of(best.part);
      std::cout << "==================================================\n";
      std::cout << std::fixed << std::setprecision(3);
      std::cout << "Melhor valor de corte encontrado (f_best):  " << (double)best.fitness / S << "\n";
      std::cout << "Verificacao independente do fitness:        " << (double)verify / S << "\n";
      std::cout << "Numero de geracoes (ciclos evolutivos):     " << generations << "\n";
      std::cout << "Tempo total:                                " << std::fixed << std::setprecision(2)
                << macut.elapsed() << " s\n";
      std::cout << "Iteracoes total:                            " << macut.iterations_count << "\n";
      std::cout << "Avaliacoes total:                           " << macut.evaluations_count << "\n";
      std::cout << "==================================================\n";
      std::cout.flush();
      if (!out_file.empty()) {
        std::ofstream fout(out_file);
        fout << "# Particao encontrada por MACUT. f = " << (double)best.fitness / S << "\n";
        fout << "# vertice(1-indexado) subconjunto(1 ou 2)\n";
        for (int32_t v = 0; v < I.n; v++) fout << (v + 1) << " " << (best.part[v] + 1) << "\n";
        std::cerr << "[MACUT] Particao salva em " << out_file << "\n";
      }
    }
    ts_graph_destroy(g);
  } catch (const std::exception& e) {
    std::cout.flush();
    std::cerr << e.what() << "\n";
    return 1;
  }
  return 0;
}
