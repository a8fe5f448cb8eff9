// ts_host.h -- host-side objects behind the C-ABI handles.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "ts_b200.h"
#include "ts_internal.cuh"

namespace tsb {

// Names the span of a C-ABI call on a profiler's timeline (NVTX range: ncu
// --nvtx filters, Nsight Systems); a no-op unless a tool is attached.
struct TraceRange {
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};

// Thread-local message of the last failing call.
void set_error(const std::string& msg);
const char* last_error();

// Records the failure and returns TS_ERR_CUDA (or TS_ERR_OUT_OF_MEMORY).
ts_status cuda_fail(cudaError_t e, const char* what);

#define TS_CUDA(call)                                     \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return ::tsb::cuda_fail(e_, #call); \
  } while (0)

// Owning device buffer.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  ts_status alloc(size_t nbytes, const char* what) {
    release();
    if (nbytes == 0) nbytes = 16;
    cudaError_t e = cudaMalloc(&p, nbytes);
    if (e != cudaSuccess) {
      p = nullptr;
      return cuda_fail(e, what);
    }
    bytes = nbytes;
    return TS_OK;
  }
  template <class T> T* as() const { return static_cast<T*>(p); }
};

}  // namespace tsb

struct ts_graph {
  int32_t n = 0;
  int32_t kind = 0;
  int32_t drop_self_loops = 0;
  int32_t device = 0;
  cudaStream_t stream = nullptr;
  int64_t num_edges = 0;
  int64_t entries = 0;
  int64_t max_wdeg = 0;
  bool neg_w = false;  // some edge weight is negative
  int64_t max_abs_w = 0;  // largest |w| of an entry
  int64_t wpr = 0;
  int64_t hash_slots = 0;
  tsb::DevBuf rowptr, adj, bits, hoff, hkey, hval, rev;
  // Host copy of the CSR row pointers/degrees (for footprint planning and the
  // solver's staging budgets); small: n+1 int64.
  std::vector<int64_t> h_rowptr;
  tsb::DevGraph dev() const {
    tsb::DevGraph g;
    g.n = n;
    g.kind = kind;
    g.entries = entries;
    g.rowptr = rowptr.as<int64_t>();
    g.adj = adj.as<int2>();
    g.bits = bits.as<uint64_t>();
    g.wpr = wpr;
    g.hoff = hoff.as<int64_t>();
    g.hkey = hkey.as<int32_t>();
    g.hval = hval.as<int32_t>();
    g.rev = rev.as<int64_t>();
    return g;
  }
  int64_t device_bytes() const {
    return (int64_t)(rowptr.bytes + adj.bytes + bits.bytes + hoff.bytes + hkey.bytes + hval.bytes + rev.bytes);
  }
  mutable int64_t deg90 = -1;  // 90th-percentile degree, computed on first use
};

namespace tsb {

// Shared by the plain solver and the batched form (solver.cu).
// Reference-compatible random streams: the MDP start (srand/rand rejection),
// the MaxBS shuffle partition (side0[v] = 1: part 0) and one perturbation
// event of k distinct flat move indices.
void mdp_random_set(int32_t n, int32_t m, uint32_t seed, std::vector<int32_t>& ids);
void maxbs_random_part(std::mt19937& rng, int32_t n, std::vector<uint8_t>& side0);
void draw_event(std::mt19937& rng, int64_t P, int k, std::vector<long long>& out);
// Dynamic shared memory for staging R rows of a lookup structure (the pass
// with per-row registers).
int32_t staging_bytes(const ts_graph* g, int R);

// Tile shape of a solve, shared by the plain and the persistent (batched,
// served; `persist`: 256-thread CTAs) forms: rows per tile, whether the fast pass runs (32-bit keys) and its index capacity,
// the CSR adjacency mask, column chunks (a multiple of one pass of the CTA, at
// least `min_tiles` tiles where the columns allow) and the dynamic shared
// memory one tile needs.
struct TileGeom {
  int32_t rows = 0, n_row_blocks = 0, chunk_cols = 0, n_chunks = 0;
  int32_t fast = 0, fast_ecap = 0, adj_mask = 0, stage_bytes = 0;
  size_t smem = 16;
};
TileGeom tile_geometry(const ts_graph* g, int32_t problem, int32_t m, bool wide, int64_t min_tiles,
                       int32_t pass, bool persist);
// WSwap: the matrix holds 16-bit weights when every |w| fits (the patch of a
// move clears and sets elements, so an element only ever holds one weight).
bool wswap_w16(const ts_graph* g);
// Opts kernel `fn` in to `smem` bytes of dynamic shared memory on the current
// device.  The limit only grows (under a lock), so a launch planned earlier
// with a larger size stays valid when a smaller one is planned later.
cudaError_t allow_dyn_smem(const void* fn, size_t smem);

}  // namespace tsb
