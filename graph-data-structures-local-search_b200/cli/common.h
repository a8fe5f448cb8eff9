// common.h -- shared pieces of the drop-in programs: C-ABI error handling,
// host CSR lookups for the drivers' own arithmetic, clocks and generators.
#pragma once
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "ts_b200.h"

namespace tscli {

inline void check(ts_status st, const char* what) {
  if (st != TS_OK)
    throw std::runtime_error(std::string(what) + ": " + ts_status_string(st) + ": " + ts_last_error());
}

// Rows sorted by neighbour id; w(u,v) is the first entry of a duplicated pair,
// as in the device structures (diversity_edge, src/mdp/GPU-MDP-CSR.cu:238-252).
struct HostCSR {
  int32_t n = 0;
  std::vector<int64_t> rowptr;
  std::vector<int32_t> col, w;
  HostCSR() = default;
  HostCSR(int32_t n_, const std::vector<int32_t>& u, const std::vector<int32_t>& v,
          const std::vector<int32_t>& wt, bool drop_self) {
    n = n_;
    rowptr.assign((size_t)n + 1, 0);
    for (size_t k = 0; k < u.size(); k++) {
      if (drop_self && u[k] == v[k]) continue;
      rowptr[u[k] + 1]++;
      rowptr[v[k] + 1]++;
    }
    for (int32_t x = 0; x < n; x++) rowptr[x + 1] += rowptr[x];
    std::vector<int64_t> fill(rowptr.begin(), rowptr.end() - 1);
    std::vector<std::pair<int32_t, int32_t>> e((size_t)rowptr[n]);
    for (size_t k = 0; k < u.size(); k++) {
      if (drop_self && u[k] == v[k]) continue;
      e[(size_t)fill[u[k]]++] = {v[k], wt[k]};
      e[(size_t)fill[v[k]]++] = {u[k], wt[k]};
    }
    col.resize(e.size());
    w.resize(e.size());
    for (int32_t x = 0; x < n; x++) {
      std::stable_sort(e.begin() + rowptr[x], e.begin() + rowptr[x + 1],
                       [](const std::pair<int32_t, int32_t>& a, const std::pair<int32_t, int32_t>& b) {
                         return a.first < b.first;
                       });
    }
    for (size_t k = 0; k < e.size(); k++) {
      col[k] = e[k].first;
      w[k] = e[k].second;
    }
  }
  int64_t edge(int32_t a, int32_t b) const {
    int64_t lo = rowptr[a], hi = rowptr[a + 1];
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (col[mid] < b) lo = mid + 1;
      else hi = mid;
    }
    return (lo < rowptr[a + 1] && col[lo] == b) ? w[lo] : 0;
  }
};

// glibc's rand() stream after srand(seed), kept private to the program.
struct GlibcRand {
  struct random_data rd;
  char state[128];
  explicit GlibcRand(unsigned seed) { reseed(seed); }
  void reseed(unsigned seed) {
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

struct Stopwatch {
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  void reset() { t0 = std::chrono::steady_clock::now(); }
  double seconds() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

// Tenure option "ref" or "fixed:T".
inline void parse_tenure(const std::string& s, int32_t* policy, int32_t* tenure) {
  if (s == "ref") {
    *policy = TS_TENURE_REF;
  } else if (s.rfind("fixed:", 0) == 0) {
    *policy = TS_TENURE_FIXED;
    *tenure = std::atoi(s.c_str() + 6);
  } else {
    throw std::runtime_error("tenure must be 'ref' or 'fixed:T'");
  }
}

// Structure name from the program name "<problem>_<alg>".
inline int32_t struct_from_program(const char* argv0, const char* prefix) {
  std::string b = argv0;
  const size_t sl = b.find_last_of('/');
  if (sl != std::string::npos) b = b.substr(sl + 1);
  const std::string p = std::string(prefix) + "_";
  if (b.rfind(p, 0) != 0) return -1;
  return ts_struct_from_name(b.substr(p.size()).c_str());
}

}  // namespace tscli
