// graph.cu -- device-side graph builders for the six lookup structures and
// the single lookup interface.
//
// Reference builders replaced: read_instance/createCSR (src/mdp/GPU-MDP-CSR.cu:
// 210-367, host sort + H2D), load/createCSR (src/maxbisection/GPU-MAXBS-CSR.cu:
// 112-173), the host bitmap (src/mdp/GPU-MDP-CSR-Bitset-BuscaBinaria.cu:321-378),
// and the uint32-keyed global hash table (src/mdp/GPU-MDP-Hash.cu:140-217,413-440),
// whose (u<<16)|v key aliases once n > 65,536.  Here everything is built on the
// device from the edge list: one stable radix sort of 64-bit (row, neighbour)
// keys produces the CSR; bitset rows and per-vertex hash tables are filled from
// it.  The hash tables are keyed by (row vertex, neighbour) -- the row selects
// the table, the neighbour id is the key -- so no aliasing at any n; keys and
// weights are stored as separate arrays so a probe reads 4 bytes.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "ts_host.h"

namespace tsb {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

ts_status cuda_fail(cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  set_error(m);
  cudaGetLastError();  // clear sticky-free errors
  return e == cudaErrorMemoryAllocation ? TS_ERR_OUT_OF_MEMORY : TS_ERR_CUDA;
}

cudaError_t allow_dyn_smem(const void* fn, size_t smem) {
  // The default limit is 48 KB minus the kernel's static shared memory, so
  // even a request below 48 KB may need the attribute raised.
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, fn);
  if (e != cudaSuccess) return e;
  if ((size_t)fa.maxDynamicSharedSizeBytes >= smem) return cudaSuccess;
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

namespace {

constexpr int kTPB = 256;

inline int blocks_for(int64_t n, int tpb = kTPB) {
  int64_t b = (n + tpb - 1) / tpb;
  if (b < 1) b = 1;
  if (b > 148LL * 64) b = 148 * 64;  // grid-stride loops cover the rest
  return (int)b;
}

// Directed entries: 2 per edge ((u,v) at 2e, (v,u) at 2e+1), key = row<<32|col.
// Dropped self-loops and out-of-range endpoints get row n (sorted past the end).
__global__ void k_make_keys(int32_t n, int64_t E, const int32_t* __restrict__ u,
                            const int32_t* __restrict__ v, const int32_t* __restrict__ w,
                            int drop_self, unsigned long long* __restrict__ keys,
                            int32_t* __restrict__ vals, int32_t* __restrict__ err) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
       e += (int64_t)gridDim.x * blockDim.x) {
    int32_t a = u[e], b = v[e];
    bool bad = a < 0 || a >= n || b < 0 || b >= n;
    if (bad) atomicOr(err, E_BAD_EDGE);
    bool skip = bad || (drop_self && a == b);
    unsigned long long ra = skip ? (unsigned long long)n : (unsigned long long)a;
    unsigned long long rb = skip ? (unsigned long long)n : (unsigned long long)b;
    keys[2 * e] = (ra << 32) | (unsigned)(skip ? 0 : b);
    keys[2 * e + 1] = (rb << 32) | (unsigned)(skip ? 0 : a);
    vals[2 * e] = w[e];
    vals[2 * e + 1] = w[e];
  }
}

// rowptr[r] = first sorted entry whose row >= r; entries with row == n are past the end.
__global__ void k_rowptr(int32_t n, int64_t N, const unsigned long long* __restrict__ keys,
                         int64_t* __restrict__ rowptr) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k <= N;
       k += (int64_t)gridDim.x * blockDim.x) {
    int64_t rp = k == 0 ? -1 : (int64_t)(keys[k - 1] >> 32);
    int64_t rc = k == N ? n : (int64_t)(keys[k] >> 32);
    if (rp > n) rp = n;
    if (rc > n) rc = n;
    for (int64_t r = rp + 1; r <= rc; r++) rowptr[r] = k;
  }
}

__global__ void k_pack_adj(int64_t N, const unsigned long long* __restrict__ keys,
                           const int32_t* __restrict__ vals, int2* __restrict__ adj) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < N;
       k += (int64_t)gridDim.x * blockDim.x)
    adj[k] = make_int2((int32_t)(keys[k] & 0xffffffffu), vals[k]);
}

// Per-row sum |w|: bounds |contribution| and decides the 32-bit key path
// (out[0]); out[1] != 0 when some weight is negative; out[2] = max |w| (the
// WSwap matrix holds 16-bit weights when it fits).
__global__ void k_max_wdeg(int32_t n, const int64_t* __restrict__ rowptr,
                           const int2* __restrict__ adj, unsigned long long* __restrict__ out) {
  for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    unsigned long long s = 0, mx = 0;
    bool neg = false;
    for (int64_t k = rowptr[r]; k < rowptr[r + 1]; k++) {
      int32_t x = adj[k].y;
      const unsigned long long a = (unsigned long long)(x < 0 ? -(long long)x : (long long)x);
      s += a;
      mx = a > mx ? a : mx;
      neg |= x < 0;
    }
    atomicMax(out, s);
    if (neg) atomicMax(out + 1, 1ull);
    if (mx) atomicMax(out + 2, mx);
  }
}

__device__ __forceinline__ int32_t row_of(const int64_t* rowptr, int32_t n, int64_t k) {
  int32_t lo = 0, hi = n - 1;  // last row r with rowptr[r] <= k
  while (lo < hi) {
    int32_t mid = (lo + hi + 1) >> 1;
    if (rowptr[mid] <= k) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__global__ void k_fill_bits(int32_t n, int64_t N, const int64_t* __restrict__ rowptr,
                            const int2* __restrict__ adj, int64_t wpr,
                            unsigned long long* __restrict__ bits) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < N;
       k += (int64_t)gridDim.x * blockDim.x) {
    int32_t r = row_of(rowptr, n, k);
    int32_t c = adj[k].x;
    atomicOr(&bits[r * wpr + (c >> 6)], 1ull << (c & 63));
  }
}

__global__ void k_hash_caps(int32_t n, const int64_t* __restrict__ rowptr, int64_t* __restrict__ caps) {
  for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    caps[r] = hash_capacity(rowptr[r + 1] - rowptr[r]);
  if (blockIdx.x == 0 && threadIdx.x == 0) caps[n] = 0;
}

__global__ void k_hash_clear(int64_t slots, int32_t* __restrict__ keys, int32_t* __restrict__ vals) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < slots;
       k += (int64_t)gridDim.x * blockDim.x) {
    keys[k] = kHashEmpty;
    vals[k] = 0;
  }
}

// Inserts the first entry of every (row, neighbour) pair with linear probing.
__global__ void k_hash_insert(int32_t n, int64_t N, const int64_t* __restrict__ rowptr,
                              const int2* __restrict__ adj, const int64_t* __restrict__ hoff,
                              int32_t* __restrict__ keys, int32_t* __restrict__ vals,
                              int32_t* __restrict__ err) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < N;
       k += (int64_t)gridDim.x * blockDim.x) {
    int32_t r = row_of(rowptr, n, k);
    int2 e = adj[k];
    if (k > rowptr[r] && adj[k - 1].x == e.x) continue;  // duplicate pair: first wins
    const int64_t base = hoff[r];
    const int64_t cap = hoff[r + 1] - base;
    const uint32_t gmask = (uint32_t)(cap / 4 - 1);
    uint32_t grp = hash_group(e.x, hash_gshift(cap));
    bool ok = false;
    for (uint32_t t = 0; t <= gmask && !ok; t++) {
      for (int sl = 0; sl < 4; sl++) {
        const int64_t at = base + 4LL * grp + sl;
        if (atomicCAS(&keys[at], kHashEmpty, e.x) == kHashEmpty) {
          vals[at] = e.y;
          ok = true;
          break;
        }
      }
      grp = (grp + 1) & gmask;
    }
    if (!ok) atomicOr(err, E_HASH_FULL);
  }
}

// rev[k] for entry k = (y -> z): the entry (z -> y) in row z with the same
// duplicate rank (a self-loop's entries map to themselves).
__global__ void k_reverse_index(int32_t n, int64_t N, const int64_t* __restrict__ rowptr,
                                const int2* __restrict__ adj, int64_t* __restrict__ rev) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < N;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t y = row_of(rowptr, n, k);
    const int32_t z = adj[k].x;
    auto lower = [&](int32_t row, int32_t key) {
      int64_t lo = rowptr[row], len = rowptr[row + 1] - lo;
      while (len > 0) {
        int64_t half = len >> 1;
        if (adj[lo + half].x < key) { lo += half + 1; len -= half + 1; }
        else len = half;
      }
      return lo;
    };
    const int64_t t = k - lower(y, z);
    rev[k] = lower(z, y) + t;
  }
}

}  // namespace

// ------------------------------------------------------------- lookups
// First entry of row u with neighbour v (gpu_edge semantics, GPU-MDP-CSR.cu:555-564).
__device__ __forceinline__ int32_t csr_scan(const DevGraph& g, int32_t u, int32_t v) {
  for (int64_t k = g.rowptr[u]; k < g.rowptr[u + 1]; k++) {
    int2 e = g.adj[k];
    if (e.x == v) return e.y;
  }
  return 0;
}

// lower_bound over the sorted row (binary-search variant,
// GPU-MDP-CSR-BuscaBinaria.cu:554-566, returning the first duplicate).
__device__ __forceinline__ int32_t csr_bsearch(const DevGraph& g, int32_t u, int32_t v) {
  int64_t lo = g.rowptr[u], len = g.rowptr[u + 1] - lo;
  while (len > 0) {
    int64_t half = len >> 1;
    if (g.adj[lo + half].x < v) { lo += half + 1; len -= half + 1; }
    else len = half;
  }
  if (lo < g.rowptr[u + 1] && g.adj[lo].x == v) return g.adj[lo].y;
  return 0;
}

__device__ __forceinline__ int32_t lookup_any(const DevGraph& g, int32_t u, int32_t v) {
  switch (g.kind) {
    case S_HASH: {
      const int64_t base = g.hoff[u];
      const int64_t cap = g.hoff[u + 1] - base;
      const uint32_t gmask = (uint32_t)(cap / 4 - 1);
      uint32_t grp = hash_group(v, hash_gshift(cap));
      for (uint32_t t = 0; t <= gmask; t++) {
        const int4 k4 = *reinterpret_cast<const int4*>(g.hkey + base + 4LL * grp);
        const int32_t ks[4] = {k4.x, k4.y, k4.z, k4.w};
        bool empty = false;
        for (int sl = 0; sl < 4; sl++) {
          if (ks[sl] == v) return g.hval[base + 4LL * grp + sl];
          empty |= ks[sl] == kHashEmpty;
        }
        if (empty) return 0;
        grp = (grp + 1) & gmask;
      }
      return 0;
    }
    case S_BITSET:
    case S_BITSET_BB: {
      uint64_t word = g.bits[u * g.wpr + (v >> 6)];
      if (!((word >> (v & 63)) & 1ull)) return 0;
      return g.kind == S_BITSET ? csr_scan(g, u, v) : csr_bsearch(g, u, v);
    }
    case S_BB:
      return csr_bsearch(g, u, v);
    default:  // CSR and WSwap (whose matrix belongs to a solver)
      return csr_scan(g, u, v);
  }
}

__global__ void k_lookup(DevGraph g, int64_t count, const int32_t* __restrict__ u,
                         const int32_t* __restrict__ v, int32_t* __restrict__ w) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < count;
       k += (int64_t)gridDim.x * blockDim.x) {
    int32_t a = u[k], b = v[k];
    w[k] = (a >= 0 && a < g.n && b >= 0 && b < g.n) ? lookup_any(g, a, b) : 0;
  }
}

// ------------------------------------------------------------- build
static ts_status build_graph(ts_graph* G, int64_t E, const int32_t* d_u, const int32_t* d_v,
                             const int32_t* d_w) {
  cudaStream_t st = G->stream;
  const int32_t n = G->n;
  const int64_t N2 = 2 * E;
  DevBuf keys, keys_alt, vals, vals_alt, err, tmp, cnt;
  TS_CUDA(cudaSetDevice(G->device));
  ts_status s;
  if ((s = keys.alloc(sizeof(unsigned long long) * N2, "alloc keys")) != TS_OK) return s;
  if ((s = keys_alt.alloc(sizeof(unsigned long long) * N2, "alloc keys")) != TS_OK) return s;
  if ((s = vals.alloc(sizeof(int32_t) * N2, "alloc vals")) != TS_OK) return s;
  if ((s = vals_alt.alloc(sizeof(int32_t) * N2, "alloc vals")) != TS_OK) return s;
  if ((s = err.alloc(sizeof(int32_t) * 2, "alloc err")) != TS_OK) return s;
  if ((s = cnt.alloc(3 * sizeof(unsigned long long), "alloc cnt")) != TS_OK) return s;
  TS_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int32_t) * 2, st));
  if (E > 0) {
    k_make_keys<<<blocks_for(E), kTPB, 0, st>>>(n, E, d_u, d_v, d_w, G->drop_self_loops,
                                                keys.as<unsigned long long>(), vals.as<int32_t>(),
                                                err.as<int32_t>());
    TS_CUDA(cudaGetLastError());
  }
  int row_bits = 1;
  while ((1LL << row_bits) <= (int64_t)n) row_bits++;
  cub::DoubleBuffer<unsigned long long> dk(keys.as<unsigned long long>(), keys_alt.as<unsigned long long>());
  cub::DoubleBuffer<int32_t> dv(vals.as<int32_t>(), vals_alt.as<int32_t>());
  if (N2 > 0) {
    size_t tbytes = 0;
    TS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tbytes, dk, dv, N2, 0, 32 + row_bits, st));
    if ((s = tmp.alloc(tbytes, "alloc sort temp")) != TS_OK) return s;
    TS_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tbytes, dk, dv, N2, 0, 32 + row_bits, st));
  }
  if ((s = G->rowptr.alloc(sizeof(int64_t) * (n + 1), "alloc rowptr")) != TS_OK) return s;
  k_rowptr<<<blocks_for(N2 + 1), kTPB, 0, st>>>(n, N2, dk.Current(), G->rowptr.as<int64_t>());
  TS_CUDA(cudaGetLastError());
  G->h_rowptr.assign(n + 1, 0);
  TS_CUDA(cudaMemcpyAsync(G->h_rowptr.data(), G->rowptr.p, sizeof(int64_t) * (n + 1),
                          cudaMemcpyDeviceToHost, st));
  int32_t h_err[2] = {0, 0};
  TS_CUDA(cudaMemcpyAsync(h_err, err.p, sizeof(int32_t) * 2, cudaMemcpyDeviceToHost, st));
  TS_CUDA(cudaStreamSynchronize(st));
  if (h_err[0] & E_BAD_EDGE) {
    set_error("ts_graph_create: edge endpoint outside [0, n)");
    return TS_ERR_INVALID_ARG;
  }
  const int64_t N = G->h_rowptr[n];
  G->entries = N;
  G->num_edges = N / 2;
  // Two spare entries: the sweep bulk-copies rows from an even entry to an
  // even end (16-byte aligned), which can reach one entry past the last row.
  if ((s = G->adj.alloc(sizeof(int2) * (N + 2), "alloc adj")) != TS_OK) return s;
  if (N > 0) {
    k_pack_adj<<<blocks_for(N), kTPB, 0, st>>>(N, dk.Current(), dv.Current(), G->adj.as<int2>());
    TS_CUDA(cudaGetLastError());
  }
  keys.release();
  keys_alt.release();
  vals.release();
  vals_alt.release();
  tmp.release();
  TS_CUDA(cudaMemsetAsync(cnt.p, 0, 3 * sizeof(unsigned long long), st));
  if (n > 0) {
    k_max_wdeg<<<blocks_for(n), kTPB, 0, st>>>(n, G->rowptr.as<int64_t>(), G->adj.as<int2>(),
                                               cnt.as<unsigned long long>());
    TS_CUDA(cudaGetLastError());
  }
  unsigned long long mw[3] = {0, 0, 0};
  TS_CUDA(cudaMemcpyAsync(mw, cnt.p, sizeof(mw), cudaMemcpyDeviceToHost, st));

  if (G->kind == TS_STRUCT_CSR_BITSET || G->kind == TS_STRUCT_CSR_BITSET_BB) {
    int64_t words = ((int64_t)n + 63) / 64;
    G->wpr = (words + 1) & ~1LL;  // even: every row starts on a 16 B boundary
    size_t bytes = sizeof(uint64_t) * (size_t)n * (size_t)G->wpr;
    if ((s = G->bits.alloc(bytes, "alloc bitset")) != TS_OK) return s;
    TS_CUDA(cudaMemsetAsync(G->bits.p, 0, bytes, st));
    if (N > 0) {
      k_fill_bits<<<blocks_for(N), kTPB, 0, st>>>(n, N, G->rowptr.as<int64_t>(), G->adj.as<int2>(),
                                                  G->wpr, G->bits.as<unsigned long long>());
      TS_CUDA(cudaGetLastError());
    }
  }
  if (G->kind == TS_STRUCT_HASH) {
    if ((s = G->hoff.alloc(sizeof(int64_t) * (n + 1), "alloc hash offsets")) != TS_OK) return s;
    DevBuf caps;
    if ((s = caps.alloc(sizeof(int64_t) * (n + 1), "alloc hash caps")) != TS_OK) return s;
    k_hash_caps<<<blocks_for(n), kTPB, 0, st>>>(n, G->rowptr.as<int64_t>(), caps.as<int64_t>());
    TS_CUDA(cudaGetLastError());
    size_t tbytes = 0;
    TS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tbytes, caps.as<int64_t>(), G->hoff.as<int64_t>(),
                                          n + 1, st));
    if ((s = tmp.alloc(tbytes, "alloc scan temp")) != TS_OK) return s;
    TS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tbytes, caps.as<int64_t>(), G->hoff.as<int64_t>(),
                                          n + 1, st));
    int64_t slots = 0;
    TS_CUDA(cudaMemcpyAsync(&slots, G->hoff.as<int64_t>() + n, sizeof(int64_t),
                            cudaMemcpyDeviceToHost, st));
    TS_CUDA(cudaStreamSynchronize(st));
    G->hash_slots = slots;
    if ((s = G->hkey.alloc(sizeof(int32_t) * slots, "alloc hash keys")) != TS_OK) return s;
    if ((s = G->hval.alloc(sizeof(int32_t) * slots, "alloc hash weights")) != TS_OK) return s;
    k_hash_clear<<<blocks_for(slots), kTPB, 0, st>>>(slots, G->hkey.as<int32_t>(), G->hval.as<int32_t>());
    TS_CUDA(cudaGetLastError());
    if (N > 0) {
      k_hash_insert<<<blocks_for(N), kTPB, 0, st>>>(n, N, G->rowptr.as<int64_t>(), G->adj.as<int2>(),
                                                    G->hoff.as<int64_t>(), G->hkey.as<int32_t>(),
                                                    G->hval.as<int32_t>(), err.as<int32_t>());
      TS_CUDA(cudaGetLastError());
    }
    TS_CUDA(cudaMemcpyAsync(h_err, err.p, sizeof(int32_t) * 2, cudaMemcpyDeviceToHost, st));
  }
  TS_CUDA(cudaStreamSynchronize(st));
  if (h_err[0] & E_HASH_FULL) {
    set_error("ts_graph_create: hash table overflow");
    return TS_ERR_DEVICE;
  }
  if (G->kind == TS_STRUCT_CSR) {
    if ((s = G->rev.alloc(sizeof(int64_t) * (size_t)(N > 0 ? N : 1), "alloc reverse index")) != TS_OK) return s;
    if (N > 0) {
      k_reverse_index<<<blocks_for(N), kTPB, 0, st>>>(n, N, G->rowptr.as<int64_t>(), G->adj.as<int2>(),
                                                      G->rev.as<int64_t>());
      TS_CUDA(cudaGetLastError());
    }
    TS_CUDA(cudaStreamSynchronize(st));
  }
  G->max_wdeg = (int64_t)mw[0];
  G->neg_w = mw[1] != 0;
  G->max_abs_w = (int64_t)mw[2];
  return TS_OK;
}

}  // namespace tsb

using namespace tsb;

static ts_status make_graph(int32_t n, int64_t E, const int32_t* d_u, const int32_t* d_v,
                            const int32_t* d_w, int32_t kind, int32_t drop, void* stream,
                            ts_graph** out) {
  if (!out) { set_error("ts_graph_create: out is NULL"); return TS_ERR_INVALID_ARG; }
  *out = nullptr;
  if (n < 2 || E < 0 || kind < 0 || kind >= TS_STRUCT_COUNT) {
    set_error("ts_graph_create: need n >= 2, num_edges >= 0 and a valid structure");
    return TS_ERR_INVALID_ARG;
  }
  if (E > 0 && (!d_u || !d_v || !d_w)) { set_error("ts_graph_create: NULL edge array"); return TS_ERR_INVALID_ARG; }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("no CUDA device visible");
    return TS_ERR_NO_DEVICE;
  }
  auto* G = new ts_graph;
  G->n = n;
  G->kind = kind;
  G->drop_self_loops = drop ? 1 : 0;
  G->stream = (cudaStream_t)stream;
  cudaGetDevice(&G->device);
  ts_status s = build_graph(G, E, d_u, d_v, d_w);
  if (s != TS_OK) { delete G; return s; }
  *out = G;
  return TS_OK;
}

extern "C" {

int32_t ts_abi_version(void) { return TS_ABI_VERSION; }

const char* ts_status_string(ts_status s) {
  switch (s) {
    case TS_OK: return "ok";
    case TS_ERR_INVALID_ARG: return "invalid argument";
    case TS_ERR_CUDA: return "CUDA error";
    case TS_ERR_OUT_OF_MEMORY: return "out of device memory";
    case TS_ERR_UNSUPPORTED: return "unsupported";
    case TS_ERR_DEVICE: return "device-side error";
    case TS_ERR_STATE: return "invalid call order";
    case TS_ERR_NO_DEVICE: return "no CUDA device";
  }
  return "unknown status";
}

const char* ts_last_error(void) { return tsb::last_error(); }

static const char* kNames[TS_STRUCT_COUNT] = {"csr", "hash", "wswap", "csr-bitset", "csr-bb", "csr-bitset-bb"};

int32_t ts_struct_from_name(const char* name) {
  if (!name) return -1;
  for (int i = 0; i < TS_STRUCT_COUNT; i++)
    if (std::strcmp(name, kNames[i]) == 0) return i;
  return -1;
}

const char* ts_struct_name(int32_t kind) {
  return (kind >= 0 && kind < TS_STRUCT_COUNT) ? kNames[kind] : "unknown";
}

ts_status ts_graph_create_device(int32_t n, int64_t num_edges, const int32_t* d_u, const int32_t* d_v,
                                 const int32_t* d_w, int32_t kind, int32_t drop_self_loops,
                                 void* stream, ts_graph** out) {
  tsb::TraceRange tr_("ts_graph_create_device");
  return make_graph(n, num_edges, d_u, d_v, d_w, kind, drop_self_loops, stream, out);
}

ts_status ts_graph_create(int32_t n, int64_t num_edges, const int32_t* u, const int32_t* v,
                          const int32_t* w, int32_t kind, int32_t drop_self_loops, void* stream,
                          ts_graph** out) {
  tsb::TraceRange tr_("ts_graph_create");
  if (!out) { set_error("ts_graph_create: out is NULL"); return TS_ERR_INVALID_ARG; }
  *out = nullptr;
  if (num_edges < 0 || (num_edges > 0 && (!u || !v || !w))) {
    set_error("ts_graph_create: bad edge arrays");
    return TS_ERR_INVALID_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("no CUDA device visible");
    return TS_ERR_NO_DEVICE;
  }
  cudaStream_t st = (cudaStream_t)stream;
  DevBuf du, dv, dw;
  ts_status s;
  size_t b = sizeof(int32_t) * (size_t)num_edges;
  if ((s = du.alloc(b, "alloc u")) != TS_OK) return s;
  if ((s = dv.alloc(b, "alloc v")) != TS_OK) return s;
  if ((s = dw.alloc(b, "alloc w")) != TS_OK) return s;
  if (num_edges > 0) {
    TS_CUDA(cudaMemcpyAsync(du.p, u, b, cudaMemcpyHostToDevice, st));
    TS_CUDA(cudaMemcpyAsync(dv.p, v, b, cudaMemcpyHostToDevice, st));
    TS_CUDA(cudaMemcpyAsync(dw.p, w, b, cudaMemcpyHostToDevice, st));
  }
  s = make_graph(n, num_edges, du.as<int32_t>(), dv.as<int32_t>(), dw.as<int32_t>(), kind,
                 drop_self_loops, stream, out);
  cudaStreamSynchronize(st);
  return s;
}

ts_status ts_graph_info_get(const ts_graph* g, ts_graph_info* out) {
  if (!g || !out) { set_error("ts_graph_info_get: NULL argument"); return TS_ERR_INVALID_ARG; }
  std::memset(out, 0, sizeof(*out));
  out->n = g->n;
  out->kind = g->kind;
  out->num_edges = g->num_edges;
  out->num_entries = g->entries;
  out->max_weighted_degree = g->max_wdeg;
  out->device_bytes = g->device_bytes();
  out->hash_slots = g->hash_slots;
  out->bitset_words_per_row = g->wpr;
  return TS_OK;
}

ts_status ts_graph_destroy(ts_graph* g) {
  if (!g) return TS_OK;
  cudaSetDevice(g->device);
  cudaStreamSynchronize(g->stream);
  delete g;
  return TS_OK;
}

ts_status ts_lookup(const ts_graph* g, int64_t count, const int32_t* d_u, const int32_t* d_v,
                    int32_t* d_w_out) {
  tsb::TraceRange tr_("ts_lookup");
  if (!g || count < 0 || (count > 0 && (!d_u || !d_v || !d_w_out))) {
    set_error("ts_lookup: bad argument");
    return TS_ERR_INVALID_ARG;
  }
  if (count == 0) return TS_OK;
  TS_CUDA(cudaSetDevice(g->device));
  int64_t b = (count + 255) / 256;
  if (b > 148 * 64) b = 148 * 64;
  k_lookup<<<(int)b, 256, 0, g->stream>>>(g->dev(), count, d_u, d_v, d_w_out);
  TS_CUDA(cudaGetLastError());
  return TS_OK;
}

ts_status ts_lookup_host(const ts_graph* g, int64_t count, const int32_t* u, const int32_t* v,
                         int32_t* w_out) {
  if (!g || count < 0 || (count > 0 && (!u || !v || !w_out))) {
    set_error("ts_lookup_host: bad argument");
    return TS_ERR_INVALID_ARG;
  }
  if (count == 0) return TS_OK;
  TS_CUDA(cudaSetDevice(g->device));
  DevBuf a, b, c;
  size_t bytes = sizeof(int32_t) * (size_t)count;
  ts_status s;
  if ((s = a.alloc(bytes, "alloc")) != TS_OK) return s;
  if ((s = b.alloc(bytes, "alloc")) != TS_OK) return s;
  if ((s = c.alloc(bytes, "alloc")) != TS_OK) return s;
  TS_CUDA(cudaMemcpyAsync(a.p, u, bytes, cudaMemcpyHostToDevice, g->stream));
  TS_CUDA(cudaMemcpyAsync(b.p, v, bytes, cudaMemcpyHostToDevice, g->stream));
  s = ts_lookup(g, count, a.as<int32_t>(), b.as<int32_t>(), c.as<int32_t>());
  if (s != TS_OK) return s;
  TS_CUDA(cudaMemcpyAsync(w_out, c.p, bytes, cudaMemcpyDeviceToHost, g->stream));
  TS_CUDA(cudaStreamSynchronize(g->stream));
  return TS_OK;
}

}  // extern "C"
