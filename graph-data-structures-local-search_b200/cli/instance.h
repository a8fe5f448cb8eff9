// instance.h -- instance files of the reference's two programs, read into an
// integer edge list for the C-ABI.
//
// Weights in the files are decimal numbers (the converter writes thousandths,
// src/convert_mwis.cpp:19-31).  They are read as exact fixed-point integers:
// the scale is 10^d for the largest number d <= 3 of decimals in the file, so
// integer files keep scale 1 and converted files get 1000.  Objectives are
// printed divided by the scale.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace tscli {

struct Instance {
  int32_t n = 0;
  int32_t m = 0;            // MDP: selected-set size of the data set; MaxBS: floor(n/2)
  int64_t declared_edges = 0;
  std::vector<int32_t> u, v, w;
  int64_t scale = 1;        // weights are value * scale
  int32_t max_decimals = 0;
  bool rounded = false;     // some weight had more than 3 decimals
};

// MDP data sets (read_instance, src/mdp/GPU-MDP-CSR.cu:255-367):
//   MDG-a/b/c   "n m" header, 0-based "i j d_ij" lines, m from the header
//   b2500       "n pairs", 1-based, m = 1000, weights doubled
//   p30005000   "n pairs", 1-based, m = n/2
//   nenad       "n pairs", 0-based, m = 100
//   sparse      '%' comment lines, "n n nnz", 1-based, m = 100
// Self-loops are dropped.  Throws std::runtime_error with the reason.
Instance read_mdp(const std::string& path, const std::string& dataset);

// MaxBS / converter format (load, src/maxbisection/GPU-MAXBS-CSR.cu:145-173):
// "n n E" then E lines "u v w", 1-based; self-loops kept.
Instance read_maxbs(const std::string& path);

// Decimal string -> value * 10^decimals (round half away from zero past 3).
int64_t parse_fixed(const std::string& tok, int32_t decimals, bool* rounded);
// Number of decimals of a decimal string.
int32_t decimals_of(const std::string& tok);

// "%.*f" of value / scale.
std::string format_scaled(int64_t value, int64_t scale, int digits);

}  // namespace tscli
