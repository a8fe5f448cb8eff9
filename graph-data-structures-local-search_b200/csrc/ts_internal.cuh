// ts_internal.cuh -- device-side layout of graphs and solver state.
//
// HBM layout (all arrays 256-byte aligned by cudaMalloc):
//   graph   rowptr int64[n+1], adj int2[entries] = (neighbour, weight), rows sorted
//           by neighbour id.  Bitset: uint64[n][wpr] (wpr even, so rows start on 16 B).
//           Hash: per-vertex open-addressing tables int2 (key, weight), key -1 = empty,
//           offsets int64[n+1] (table sizes are powers of two >= 2).
//   solver  position-indexed arrays split into the inside side (rows i in [0,m))
//           and the outside side (columns j in [0,n-m), padded to ldc = multiple of 4
//           so a lane reads 4 columns with one 16 B load):
//             sol_in/sol_out (vertex ids), vg_in/vg_out (contribution, KeyT),
//             tab_in/tab_out (tabu expiry), pos[n] (vertex -> global position).
//           WSwap: W int32[m][ldc], W[i][j] = w(sol_in[i], sol_out[j]).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace tsb {

constexpr int32_t kHashEmpty = -1;
constexpr int64_t kMdpSentinel = -99999;                 // GPU-MDP-CSR.cu:59,:581
constexpr int64_t kMaxbsInf = 9999999999LL;              // -INF, GPU-MAXBS-CSR.cu:7
constexpr int64_t kMaxbsRecoverBelow = -2500000000LL;    // value < INF/4, :456

enum Struct : int32_t { S_CSR = 0, S_HASH = 1, S_WSWAP = 2, S_BITSET = 3, S_BB = 4, S_BITSET_BB = 5 };
enum Problem : int32_t { P_MDP = 0, P_MAXBS = 1 };

// Device error word bits.
enum : int32_t {
  E_LOG_FULL = 1,
  E_PERTURB_WINDOW = 2,
  E_BAD_INDEX = 4,
  E_BAD_EDGE = 8,
  E_HASH_FULL = 16,
  E_BULK_TIMEOUT = 32,  // a bulk copy into shared memory did not complete in time
};

struct DevGraph {
  int32_t n;
  int32_t kind;
  int64_t entries;
  const int64_t* rowptr;
  const int2* adj;
  const uint64_t* bits;
  int64_t wpr;
  const int64_t* hoff;
  const int32_t* hkey;  // Hash: per-vertex tables, keys (neighbour id, -1 empty) ...
  const int32_t* hval;  // ... and weights, same slots
  const int64_t* rev;   // CSR only: index of the mirrored entry (z->y) of every entry (y->z)
};

struct alignas(16) CtaRec {
  long long key;
  long long idx;
};

struct TraceRec {
  int64_t iter, idx, key, cur, best;
  int32_t kind, tenure, tenure2, pad;
};

// Mutable per-solver scalars, one device struct read at every kernel entry.
struct DevState {
  long long iter;
  long long target;       // stop when iter reaches it
  long long cur;
  long long best;
  long long evaluations;
  long long isi;          // MaxBS iterations since improvement
  long long log_n;        // applied moves
  long long best_log_n;   // log length at the last improvement
  long long trace_n;
  long long pert_events;  // perturbation events consumed
  long long pert_base;    // first event held in the device draw window
  long long pert_limit;   // events of the window that hold draws (from pert_base)
  long long pert_moves;
  unsigned int counter;   // last-CTA-done ticket
  int32_t mode;           // 0 fast sweep, 1 exact sweep
  int32_t done;
  int32_t stopped;
  int32_t err;
  int32_t pad;
};

template <class KeyT>
struct DevSolver {
  int32_t n, m, delta, ldc;
  int32_t problem;
  int32_t tenure_policy, tenure, maxt, piter, num_pert;
  int32_t c2_tab[4];      // C2 for C1 = 15, 30, 60, 120 (reference schedule)
  int32_t c2_fixed;
  int32_t n_row_blocks, n_chunks, chunk_cols, stage_bytes;
  // CSR: adjacent pairs are left out of the w-free sweep (a per-column mask
  // in shared memory) and evaluated exactly by the join.  Always for MDP; for
  // MaxBS only when a weight is negative (with w >= 0 the w-free gain of an
  // adjacent pair under-estimates it and cannot win).
  int32_t adj_mask;
  // Tile geometry: inside positions per tile; the fast pass (32-bit keys:
  // one structure query per column for all the tile's rows) and its index
  // capacity in row entries.
  int32_t tile_rows;
  int32_t fast;
  int32_t fast_ecap;
  // Plain kernel, fast pass: CTAs per tile (each takes every n_slices-th of
  // the tile's work units); 1 (or 0: unset) = one CTA per tile.
  int32_t n_slices;
  // WSwap: 1 when the matrix holds 16-bit weights (every |w| <= 32767), read
  // through W as int16_t; 0: 32-bit.
  int32_t w16;
  int64_t P;
  int32_t* sol_in;
  int32_t* sol_out;
  KeyT* vg_in;
  KeyT* vg_out;
  int32_t* tab_in;
  int32_t* tab_out;
  int32_t* pos;
  int32_t* W;
  int32_t* cpos;          // CSR only: cpos[k] = pos[adj[k].x], patched on every move
  DevState* st;
  CtaRec* recs;
  int2* movelog;
  long long log_cap;
  TraceRec* trace;
  long long trace_cap;
  const long long* draws;
  long long draw_events;  // events held in the window
};

// Hash structure: one open-addressing table per vertex, keyed by the
// neighbour id.  The reference keeps one global table at load <= 0.6 with a
// MurmurHash3 finaliser (GPU-MDP-Hash.cu:151-158,430-440); here the per-vertex
// tables keep every probe short: capacity = power of two >= 2*degree
// (load <= 0.5, at least 8 slots), split into 4-slot buckets read with one
// 16-byte load; the home bucket is a Fibonacci multiplicative hash and a full
// bucket spills to the next one.  A lookup that meets an empty slot in a
// bucket without the key is a miss (no deletions ever happen).  The sweep
// reads a tile's tables once to build its own shared-memory index, so the
// table size is also the structure's HBM traffic per row.
__host__ __device__ __forceinline__ int64_t hash_capacity(int64_t deg) {
  int64_t cap = 8;
  while (cap < 2 * deg) cap <<= 1;
  return cap;
}
__host__ __device__ __forceinline__ uint32_t hash_gshift(int64_t cap) {  // 32 - log2(cap / 4)
  uint32_t l = 0;
  while ((4LL << l) < cap) l++;
  return 32u - l;
}
__host__ __device__ __forceinline__ uint32_t hash_group(int32_t v, uint32_t gshift) {
  return ((uint32_t)v * 2654435769u) >> gshift;
}

// IEEE binary32 round-to-nearest-even of an integer, returned as the exact
// integer value of the nearest float (24 significant bits).
__host__ __device__ __forceinline__ long long round_to_f32(long long x) {
  if (x == 0) return 0;
  bool neg = x < 0;
  unsigned long long a = neg ? 0ull - (unsigned long long)x : (unsigned long long)x;
#ifdef __CUDA_ARCH__
  int msb = 63 - __clzll((long long)a);
#else
  int msb = 63 - __builtin_clzll(a);
#endif
  if (msb <= 23) return x;
  int shift = msb - 23;
  unsigned long long q = a >> shift, rem = a & ((1ull << shift) - 1), half = 1ull << (shift - 1);
  if (rem > half || (rem == half && (q & 1))) q++;
  unsigned long long r = q << shift;
  return neg ? -(long long)r : (long long)r;
}

// Penalty key of a tabu, non-aspirated MaxBS move: the float result of
// double(-9999999999) + g (GPU-MAXBS-CSR.cu:350).
__host__ __device__ __forceinline__ long long maxbs_penalty(long long g) {
  return round_to_f32(g - kMaxbsInf);
}

__host__ __device__ __forceinline__ int32_t mdp_ref_tenure(long long iter) {
  // determine_tabu_tenure, GPU-MDP-CSR.cu:461-476 (alpha 15, T 1500).
  int temp = (int)(iter % 1500);
  if (temp > 700 && temp <= 800) return 120;
  if ((temp > 300 && temp <= 400) || (temp > 1100 && temp <= 1200)) return 60;
  if ((temp > 100 && temp <= 200) || (temp > 500 && temp <= 600) ||
      (temp > 900 && temp <= 1000) || (temp > 1300 && temp <= 1400))
    return 30;
  return 15;
}

__host__ __device__ __forceinline__ int32_t maxbs_ref_tenure(long long iter, int32_t maxt) {
  // tabuTenure, GPU-MAXBS-CSR.cu:248-263 (C++ remainder truncates toward zero).
  const int b[15] = {1, 2, 1, 4, 1, 2, 1, 8, 1, 2, 1, 4, 1, 2, 1};
  long long period = 16LL * maxt;
  long long it = ((iter - 1) % period) + 1;
  long long p = 1;
  for (int i = 0; i < 15; i++) {
    long long tenure = (1LL * maxt * b[i]) / 8;
    long long length = 4LL * tenure;
    if (it < p + length) return (int32_t)tenure;
    p += length;
  }
  return maxt / 8;
}

}  // namespace tsb
