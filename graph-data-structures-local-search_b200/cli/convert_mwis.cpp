// convert_mwis.cpp -- MWIS-VR instance converter (src/convert_mwis.cpp of the
// reference): <dir>/<name>/conflict_graph.txt ("n m" + m lines "u v", 1-based)
// and node_weights.txt (n lines "vertex weight", integer weights) become
// <out>/<name>.txt in the Max Bisection format: "n n E" then E lines
// "u v w" with u < v, duplicates removed, sorted by (u, v), and
// w = (weight_u + weight_v) / 1000 written exactly with three decimals.
//
// Same output byte for byte; the edges are deduplicated in memory (a sort of
// packed 64-bit keys) instead of through an external `sort` process.
//
//   convert_mwis <instances_dir> <output_dir> [NAME]
#include <algorithm>
#include <cstdint>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

namespace fs = std::filesystem;

// (a + b) / 1000 with exactly three decimals; 128-bit sum, sign first.
static void write_weight(std::ostream& out, int64_t a, int64_t b) {
  __int128 s = (__int128)a + b;
  if (s < 0) {
    out << '-';
    s = -s;
  }
  const unsigned rest = (unsigned)(s % 1000);
  out << (unsigned long long)(s / 1000) << '.' << (char)('0' + rest / 100) << (char)('0' + (rest / 10) % 10)
      << (char)('0' + rest % 10);
}

static void convert(const fs::path& in, const fs::path& out_dir, const std::string& name) {
  const fs::path dir = in / name;
  std::ifstream gf(dir / "conflict_graph.txt");
  std::ifstream wf(dir / "node_weights.txt");
  if (!gf || !wf) throw std::runtime_error("Arquivos ausentes na instancia " + name);
  uint64_t n = 0, m = 0;
  if (!(gf >> n >> m) || n == 0 || n > 0xFFFFFFFFull) throw std::runtime_error("Cabecalho invalido: " + name);
  std::vector<int64_t> weight(n + 1, 0);
  std::vector<char> seen(n + 1, 0);
  for (uint64_t i = 0; i < n; i++) {
    uint64_t v = 0;
    int64_t wt = 0;
    if (!(wf >> v >> wt) || v == 0 || v > n || seen[v])
      throw std::runtime_error("Pesos incompletos, repetidos ou invalidos em " + name);
    weight[v] = wt;
    seen[v] = 1;
  }
  std::string extra;
  if (wf >> extra) throw std::runtime_error("Dados extras em node_weights.txt: " + name);
  std::vector<uint64_t> keys;
  keys.reserve(m);
  for (uint64_t i = 0; i < m; i++) {
    uint64_t u = 0, v = 0;
    if (!(gf >> u >> v) || u == 0 || v == 0 || u > n || v > n)
      throw std::runtime_error("Aresta ausente ou invalida em " + name);
    if (u > v) std::swap(u, v);
    keys.push_back(u << 32 | v);
  }
  if (gf >> extra) throw std::runtime_error("Ha mais arestas do que indica o cabecalho: " + name);
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  fs::create_directories(out_dir);
  const fs::path part = out_dir / (name + ".txt.part");
  const fs::path fin = out_dir / (name + ".txt");
  {
    std::ofstream o(part, std::ios::trunc);
    if (!o) throw std::runtime_error("Falha ao criar saida: " + name);
    o << n << ' ' << n << ' ' << keys.size() << '\n';
    for (uint64_t k : keys) {
      const uint64_t u = k >> 32, v = k & 0xFFFFFFFFull;
      o << u << ' ' << v << ' ';
      write_weight(o, weight[u], weight[v]);
      o << '\n';
    }
    if (!o) throw std::runtime_error("Falha ao gravar a saida: " + name);
  }
  fs::rename(part, fin);
  std::cout << name << ": " << n << " vertices, " << keys.size() << " arestas (" << (m - keys.size())
            << " duplicatas removidas) -> " << fin.string() << '\n';
}

int main(int argc, char** argv) {
  if (argc != 3 && argc != 4) {
    std::cerr << "Uso: " << argv[0] << " <instancias_mwis> <graph_instances> [NOME_DA_INSTANCIA]\n";
    return 1;
  }
  try {
    const fs::path in = argv[1], out = argv[2];
    if (!fs::is_directory(in)) throw std::runtime_error("Pasta de instancias nao encontrada: " + in.string());
    fs::create_directories(out);
    if (argc == 4) {
      convert(in, out, argv[3]);
    } else {
      std::vector<std::string> names;
      for (const auto& e : fs::directory_iterator(in))
        if (e.is_directory() && fs::exists(e.path() / "conflict_graph.txt")) names.push_back(e.path().filename().string());
      std::sort(names.begin(), names.end());
      if (names.empty()) throw std::runtime_error("Nenhuma instancia encontrada em " + in.string());
      for (const auto& nm : names) convert(in, out, nm);
    }
  } catch (const std::exception& e) {
    std::cerr << "Erro: " << e.what() << '\n';
    return 1;
  }
  return 0;
}
