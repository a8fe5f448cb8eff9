// noalloc.cu -- best admissible swap of a caller-held state, with no device
// allocation.
//
// Who needs it: callers that may not allocate device memory -- plugins whose
// host application owns all of HBM through its own pool allocator, and
// services that run under a fixed device-memory budget.  They keep the graph
// and the tabu state in their own buffers and get one iteration's decision:
// every swap evaluated with the reference's key rule (tabu/aspiration filter,
// MDP -99999 sentinel, MaxBS float-quantised penalty) and the ArgMax with its
// lowest-index tie rule.  This entry point has no counterpart in the reference.
//
// Scratch: one file-scope device array (kScratchBytes, about 3 MiB) holding the
// position-ordered contributions and tabu flags, the per-CTA records and the
// last-CTA ticket.  Every GPU that loads the library keeps it until the process
// exits.  All calls share it and it keeps the last call's contents: the ticket
// is cleared by the staging kernel of every call, and calls that overlap on the
// GPU (from other streams or host threads) race on it.
//
// Cost: one thread per swap pair, each with its own binary search of the
// inside vertex's CSR row in global memory -- about log2(degree) + 2 dependent
// loads per pair, so a call over P pairs takes roughly P / 1e10 seconds on a
// B200 (n = 262,144 with m = n/2 is ~1.7e10 pairs: seconds per call).  It is
// meant for modest instances, not as the fast path.
#include <climits>
#include <cstdint>
#include <mutex>

#include "sweep.cuh"
#include "ts_host.h"

namespace tsb {
namespace {

constexpr int32_t kNaMaxN = TS_NOALLOC_MAX_N;
constexpr int kNaTPB = 256;
constexpr int kNaMaxCtas = 4096;
constexpr size_t kNaPvgOff = 0;                                        // long long[kNaMaxN]
constexpr size_t kNaTabOff = kNaPvgOff + sizeof(long long) * kNaMaxN;  // int32[kNaMaxN]
constexpr size_t kNaRecOff = kNaTabOff + sizeof(int32_t) * kNaMaxN;    // CtaRec[kNaMaxCtas]
constexpr size_t kNaCntOff = kNaRecOff + sizeof(CtaRec) * kNaMaxCtas;  // unsigned
constexpr size_t kScratchBytes = kNaCntOff + 256;

static __device__ __align__(256) unsigned char g_na_scratch[kScratchBytes];

struct NaView {
  long long* pvg;
  int32_t* ptab;
  CtaRec* recs;
  unsigned int* counter;
};

NaView view_of(void* base) {
  unsigned char* b = static_cast<unsigned char*>(base);
  NaView v;
  v.pvg = reinterpret_cast<long long*>(b + kNaPvgOff);
  v.ptab = reinterpret_cast<int32_t*>(b + kNaTabOff);
  v.recs = reinterpret_cast<CtaRec*>(b + kNaRecOff);
  v.counter = reinterpret_cast<unsigned int*>(b + kNaCntOff);
  return v;
}

// Position order: pvg[p] = vg[sol[p]], ptab[p] = tab[sol[p]] > iter.
__global__ void k_na_stage(int32_t n, long long iter, const int32_t* __restrict__ sol,
                           const long long* __restrict__ vg, const int32_t* __restrict__ tab,
                           NaView sc) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *sc.counter = 0u;
  for (int32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int32_t v = sol[p];
    sc.pvg[p] = vg[v];
    sc.ptab[p] = tab[v] > iter;
  }
}

// First entry of u's sorted row with neighbour v (lower_bound), else 0.
__device__ __forceinline__ int32_t na_lookup(const int64_t* rowptr, const int32_t* col,
                                             const int32_t* w, int32_t u, int32_t v) {
  long long lo = rowptr[u], len = rowptr[u + 1] - lo;
  const long long end = lo + len;
  while (len > 0) {
    const long long half = len >> 1;
    if (col[lo + half] < v) { lo += half + 1; len -= half + 1; }
    else len = half;
  }
  return (lo < end && col[lo] == v) ? w[lo] : 0;
}

__global__ void __launch_bounds__(kNaTPB)
k_na_sweep(int32_t problem, int32_t n, int32_t m, long long cur, long long best,
           const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
           const int32_t* __restrict__ w, const int32_t* __restrict__ sol, NaView sc,
           int64_t* __restrict__ out) {
  __shared__ CtaRec red[kNaTPB / 32];
  __shared__ int32_t s_last;
  const int32_t delta = n - m;
  const long long P = (long long)m * delta;
  const long long D = best - cur;
  long long bk = LLONG_MIN, bi = LLONG_MAX;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < P;
       idx += (long long)gridDim.x * blockDim.x) {
    const int32_t i = (int32_t)(idx / delta), j = (int32_t)(idx % delta) + m;
    const int32_t wt = na_lookup(rowptr, col, w, sol[i], sol[j]);
    const long long x = problem == P_MDP ? sc.pvg[j] - sc.pvg[i] - wt
                                         : sc.pvg[i] + sc.pvg[j] + 2LL * wt;
    long long key = x;
    if (!allowed(sc.ptab[i] != 0, sc.ptab[j] != 0, x, D))
      key = problem == P_MDP ? kMdpSentinel : maxbs_penalty(x);
    better_rec(bk, bi, key, idx);
  }
  block_best(bk, bi, red);
  if (threadIdx.x == 0) {
    sc.recs[blockIdx.x].key = bk;
    sc.recs[blockIdx.x].idx = bi;
    __threadfence();
    s_last = atomicAdd(sc.counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  bk = LLONG_MIN;
  bi = LLONG_MAX;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
    better_rec(bk, bi, __ldcg(&sc.recs[b].key), __ldcg(&sc.recs[b].idx));
  block_best(bk, bi, red);
  if (threadIdx.x == 0) {
    out[0] = bk;
    out[1] = bi;
    *sc.counter = 0u;
  }
}

constexpr int kMaxDevices = 64;
std::mutex g_na_mu;
// The scratch array has one address per CUDA context: cached per device
// together with the context it was looked up in, and looked up again when the
// caller's current context on that device is another one (a context the caller
// created itself, or a new primary context after a device reset).
struct NaAddr {
  void* ctx;
  void* addr;
};
NaAddr g_na_addr[kMaxDevices];

// cuCtxGetCurrent, reached through the runtime so the library needs no
// link-time dependency on the driver library.
using CtxGetCurrentFn = int (*)(void**);
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      f = nullptr;
    }
    return reinterpret_cast<CtxGetCurrentFn>(f);
  }();
  return fn;
}

}  // namespace
}  // namespace tsb

using namespace tsb;

extern "C" ts_status ts_best_swap_noalloc(int32_t problem, int32_t n, int32_t m, int64_t iter,
                                          int64_t cur, int64_t best, const int64_t* d_rowptr,
                                          const int32_t* d_col, const int32_t* d_w,
                                          const int32_t* d_sol, const int64_t* d_vg,
                                          const int32_t* d_tab, int64_t* d_out, void* stream) {
  if (problem != TS_PROBLEM_MDP && problem != TS_PROBLEM_MAXBS) {
    set_error("ts_best_swap_noalloc: unknown problem");
    return TS_ERR_INVALID_ARG;
  }
  if (n < 2 || n > kNaMaxN) {
    set_error("ts_best_swap_noalloc: n must be in [2, " + std::to_string(kNaMaxN) +
              "]; the fixed scratch area holds that many positions");
    return TS_ERR_INVALID_ARG;
  }
  if (m < 1 || m >= n) { set_error("ts_best_swap_noalloc: need 1 <= m < n"); return TS_ERR_INVALID_ARG; }
  if (!d_rowptr || !d_col || !d_w || !d_sol || !d_vg || !d_tab || !d_out) {
    set_error("ts_best_swap_noalloc: NULL device pointer");
    return TS_ERR_INVALID_ARG;
  }
  int dev = 0;
  TS_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) { set_error("ts_best_swap_noalloc: device index out of range"); return TS_ERR_UNSUPPORTED; }
  void* base = nullptr;
  {
    // With the caller's device current: the scratch array's device address in
    // the current context (its name in host code is only a host-side
    // stand-in).  The first call in a context looks it up; later calls in the
    // same context reuse it.
    CtxGetCurrentFn get_ctx = ctx_get_current();
    if (!get_ctx) {
      set_error("ts_best_swap_noalloc: cuCtxGetCurrent is not available from the driver");
      return TS_ERR_UNSUPPORTED;
    }
    void* ctx = nullptr;
    if (get_ctx(&ctx) != 0 || !ctx) {
      // No context bound to this thread yet: bind the device's primary context
      // (cudaSetDevice initialises it) -- the one the runtime would use.
      TS_CUDA(cudaSetDevice(dev));
      if (get_ctx(&ctx) != 0 || !ctx) {
        set_error("ts_best_swap_noalloc: no current CUDA context on the calling thread");
        return TS_ERR_CUDA;
      }
    }
    std::lock_guard<std::mutex> lock(g_na_mu);
    if (g_na_addr[dev].ctx != ctx || !g_na_addr[dev].addr) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_na_scratch);
      if (e != cudaSuccess) return cuda_fail(e, "ts_best_swap_noalloc: cudaGetSymbolAddress");
      g_na_addr[dev].ctx = ctx;
      g_na_addr[dev].addr = p;
    }
    base = g_na_addr[dev].addr;
  }
  const NaView sc = view_of(base);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const long long P = (long long)m * (n - m);
  long long grid = (P + kNaTPB - 1) / kNaTPB;
  if (grid > kNaMaxCtas) grid = kNaMaxCtas;
  int sgrid = (n + kNaTPB - 1) / kNaTPB;
  k_na_stage<<<sgrid, kNaTPB, 0, st>>>(n, (long long)iter, d_sol, reinterpret_cast<const long long*>(d_vg),
                                       d_tab, sc);
  TS_CUDA(cudaGetLastError());
  k_na_sweep<<<(int)grid, kNaTPB, 0, st>>>(problem, n, m, (long long)cur, (long long)best, d_rowptr,
                                           d_col, d_w, d_sol, sc, d_out);
  TS_CUDA(cudaGetLastError());
  return TS_OK;
}
