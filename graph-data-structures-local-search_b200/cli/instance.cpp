// instance.cpp -- readers of the reference's instance files (see instance.h).
#include "instance.h"

#include <cstdio>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace tscli {

int32_t decimals_of(const std::string& tok) {
  const size_t dot = tok.find('.');
  if (dot == std::string::npos) return 0;
  size_t end = tok.size();
  const size_t e = tok.find_first_of("eE", dot);
  if (e != std::string::npos) end = e;
  int32_t d = (int32_t)(end - dot - 1);
  // trailing zeros add no precision
  while (d > 0 && tok[dot + d] == '0') d--;
  return d;
}

int64_t parse_fixed(const std::string& tok, int32_t decimals, bool* rounded) {
  size_t i = 0;
  bool neg = false;
  if (i < tok.size() && (tok[i] == '-' || tok[i] == '+')) neg = tok[i++] == '-';
  if (tok.find_first_of("eE") != std::string::npos) {
    // exponent notation: go through a double, exact for the values files hold
    double x = std::stod(tok);
    double s = 1;
    for (int k = 0; k < decimals; k++) s *= 10;
    const double y = x * s;
    const int64_t r = (int64_t)(y < 0 ? y - 0.5 : y + 0.5);
    if (rounded && (double)r != y) *rounded = true;
    return r;
  }
  int64_t ip = 0;
  bool any = false;
  for (; i < tok.size() && tok[i] >= '0' && tok[i] <= '9'; i++) {
    ip = ip * 10 + (tok[i] - '0');
    any = true;
  }
  int64_t frac = 0;
  int32_t got = 0;
  bool round_up = false, extra = false;
  if (i < tok.size() && tok[i] == '.') {
    i++;
    for (; i < tok.size() && tok[i] >= '0' && tok[i] <= '9'; i++) {
      any = true;
      if (got < decimals) {
        frac = frac * 10 + (tok[i] - '0');
        got++;
      } else {
        if (!extra) round_up = tok[i] >= '5';
        if (tok[i] != '0') extra = true;
      }
    }
  }
  if (!any || i != tok.size()) throw std::runtime_error("bad number '" + tok + "'");
  for (; got < decimals; got++) frac *= 10;
  int64_t s = 1;
  for (int k = 0; k < decimals; k++) s *= 10;
  int64_t r = ip * s + frac + (round_up ? 1 : 0);
  if (extra && rounded) *rounded = true;
  return neg ? -r : r;
}

std::string format_scaled(int64_t value, int64_t scale, int digits) {
  char buf[64];
  std::snprintf(buf, sizeof(buf), "%.*f", digits, (double)value / (double)scale);
  return buf;
}

namespace {

struct RawEdge {
  int64_t a, b;
  std::string w;
};

void finish(Instance& I, const std::vector<RawEdge>& raw, bool drop_self, int64_t weight_mult) {
  int32_t d = 0;
  for (const RawEdge& e : raw) d = std::max(d, decimals_of(e.w));
  I.max_decimals = d;
  if (d > 3) d = 3;
  I.scale = 1;
  for (int k = 0; k < d; k++) I.scale *= 10;
  I.u.reserve(raw.size());
  I.v.reserve(raw.size());
  I.w.reserve(raw.size());
  for (const RawEdge& e : raw) {
    if (drop_self && e.a == e.b) continue;
    const int64_t w = parse_fixed(e.w, d, &I.rounded) * weight_mult;
    if (w > INT32_MAX || w < INT32_MIN)
      throw std::runtime_error("weight " + e.w + " does not fit int32 at scale " + std::to_string(I.scale));
    I.u.push_back((int32_t)e.a);
    I.v.push_back((int32_t)e.b);
    I.w.push_back((int32_t)w);
  }
}

}  // namespace

Instance read_mdp(const std::string& path, const std::string& dataset) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("### Fail to open file: " + path);
  Instance I;
  std::string line;
  int64_t n = 0, m = 0, pairs = 0;
  bool one_based = false;
  int64_t mult = 1;
  if (dataset == "MDG-a" || dataset == "MDG-b" || dataset == "MDG-c") {
    std::getline(f, line);
    std::istringstream(line) >> n >> m;
    pairs = n * (n - 1) / 2;
  } else if (dataset == "b2500") {
    std::getline(f, line);
    std::istringstream(line) >> n >> pairs;
    m = 1000;
    one_based = true;
    mult = 2;
  } else if (dataset == "p30005000") {
    std::getline(f, line);
    std::istringstream(line) >> n >> pairs;
    m = n / 2;
    one_based = true;
  } else if (dataset == "nenad") {
    std::getline(f, line);
    std::istringstream(line) >> n >> pairs;
    m = 100;
  } else if (dataset == "sparse") {
    do {
      if (!std::getline(f, line)) throw std::runtime_error("no header in " + path);
    } while (line.empty() || line[0] == '%');
    std::istringstream(line) >> n >> n >> pairs;
    m = 100;
    one_based = true;
  } else {
    throw std::runtime_error("data set is wrong!");
  }
  if (n < 2 || n > INT32_MAX) throw std::runtime_error("bad vertex count in " + path);
  I.n = (int32_t)n;
  I.m = (int32_t)m;
  I.declared_edges = pairs;
  std::vector<RawEdge> raw;
  while (std::getline(f, line)) {
    std::istringstream iss(line);
    RawEdge e;
    if (!(iss >> e.a >> e.b >> e.w)) continue;  // blank or short line
    if (one_based) {
      e.a--;
      e.b--;
    }
    if (e.a < 0 || e.b < 0 || e.a >= n || e.b >= n)
      throw std::runtime_error("### Read Date Error : line = " + std::to_string(e.a) +
                               ", column = " + std::to_string(e.b));
    raw.push_back(std::move(e));
  }
  finish(I, raw, true, mult);
  return I;
}

Instance read_maxbs(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("Erro: nao foi possivel abrir o arquivo do grafo: " + path);
  Instance I;
  int64_t n = 0, n2 = 0, E = 0;
  if (!(f >> n >> n2 >> E) || n < 2 || n > INT32_MAX || E < 0)
    throw std::runtime_error("bad header in " + path);
  I.n = (int32_t)n;
  I.m = (int32_t)(n / 2);
  I.declared_edges = E;
  std::vector<RawEdge> raw;
  raw.reserve((size_t)E);
  for (int64_t k = 0; k < E; k++) {
    RawEdge e;
    if (!(f >> e.a >> e.b >> e.w)) throw std::runtime_error("file ends after " + std::to_string(k) + " edges");
    e.a--;
    e.b--;
    if (e.a < 0 || e.b < 0 || e.a >= n || e.b >= n)
      throw std::runtime_error("edge " + std::to_string(k + 1) + " out of range");
    raw.push_back(std::move(e));
  }
  finish(I, raw, false, 1);
  return I;
}

}  // namespace tscli
