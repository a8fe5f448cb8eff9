// sweep.cuh -- one tabu iteration as ONE kernel launch.
//
// Replaces, per iteration, the reference's calculateSwapGain / calculateMoveGain
// (src/mdp/GPU-MDP-CSR.cu:567-584, src/maxbisection/GPU-MAXBS-CSR.cu:337-353 and
// their five structure variants), cub::DeviceReduce::ArgMax + the 8-byte D2H
// copy (:651-652 / :450-451), updateVertexEdgeGain/updateMoveGain (:523-541 /
// :355-375, WSwap :524-562 / :367-409), updateSolution/finalizeMove
// (:544-553 / :377-399), best tracking (:671-674 / :469-476) and the MaxBS
// perturbation (:480-501).
//
// Each CTA owns a tile of R inside positions (rows) x chunk_cols outside
// positions (columns) of the m x (n-m) pair space.  It evaluates every pair's
// gain in 32-bit (or 64-bit) integers, applies the tabu/aspiration filter and
// keeps a per-row maximum; no gain array exists.  The CTA then resolves the
// lowest flat index achieving its maximum (the CUB ArgMax tie rule,
// cub/thread/thread_operators.cuh:103-121) by rescanning one row, and writes one
// (key, index) record.  The last CTA to finish reduces the records, decides the
// move and applies it -- so an iteration needs no host round trip.
//
// The fast pass only tracks allowed pairs (non-tabu, or aspirated).  When no
// allowed pair exists (or, for MDP, the best allowed gain is not above the
// -99999 sentinel), the last CTA switches the state to "exact" and the next
// launch re-evaluates every pair with the reference's full key rule (MDP
// sentinel, MaxBS float-quantised penalty) in int64.
#pragma once
#include <climits>
#include <cstdint>
#include <type_traits>

#include "ts_internal.cuh"

namespace tsb {

constexpr int kColsPerLane = 4;
constexpr int kMaxTPB = 512;
// Threads per CTA: the bitmap structures stage ~n/8 bytes per row, so they run
// one large CTA per SM and need more warps in it to hide shared-memory latency.
// The index structures (Hash, BB, bitmaps) build a shared-memory index per
// tile and run two 512-thread CTAs per SM.
template <int ST> struct Tpb { static constexpr int v = 512; };
template <> struct Tpb<S_CSR> { static constexpr int v = 256; };
template <> struct Tpb<S_WSWAP> { static constexpr int v = 256; };
// The persistent kernels (batched and served forms) run 256 threads for every
// structure: a cluster CTA also holds the solve's init/finish code, and at
// 512 threads its register budget would not fit an SM.
template <int ST, bool PERSIST> struct TpbOf { static constexpr int v = PERSIST ? 256 : Tpb<ST>::v; };
__host__ __device__ inline int tpb_of(int st, bool persist = false) {
  return (persist || st == S_CSR || st == S_WSWAP) ? 256 : 512;
}
__host__ __device__ inline int pass_cols_of(int st, bool persist = false) {
  return tpb_of(st, persist) * kColsPerLane;
}

template <int ST> struct Rows { static constexpr int R = 16; };
template <> struct Rows<S_CSR> { static constexpr int R = 32; };
// The bitmap structures: 4 rows per tile.  On the 2,000-vertex MDP case
// (m = 200) 8-row tiles made 25 CTAs and 4-row tiles 50: 39k -> 57k
// iterations/s (CSR+Bitset), 36k -> 53k (CSR+Bitset+BB).
template <> struct Rows<S_BITSET> { static constexpr int R = 4; };
template <> struct Rows<S_BITSET_BB> { static constexpr int R = 4; };
// Hash and CSR+BB: 4 rows per tile.  48 registers and ~16 KB of staged rows
// per tile let five CTAs share an SM; on the MaxBS conflict graph
// (n = 100,000) that is 1.4x (Hash) and 1.8x (CSR+BB) over 16 rows, the
// column loads shared by fewer rows notwithstanding.
template <> struct Rows<S_HASH> { static constexpr int R = 4; };
template <> struct Rows<S_BB> { static constexpr int R = 4; };
constexpr int kMaxTileRows = 32;
// Rows per tile of the pass with per-row registers (64-bit keys, or a graph
// too large for the fast pass's index), by structure id.
__host__ __device__ inline int rows_of(int st) {
  return st == S_CSR ? Rows<S_CSR>::R
       : st == S_BITSET ? Rows<S_BITSET>::R
       : st == S_BITSET_BB ? Rows<S_BITSET_BB>::R
       : st == S_HASH ? Rows<S_HASH>::R
       : st == S_BB ? Rows<S_BB>::R
       : Rows<S_WSWAP>::R;
}

template <class KeyT> struct KeyLim;
template <> struct KeyLim<int32_t> {
  static constexpr int32_t none = INT32_MIN;
  __device__ static int32_t clampD(long long d) {
    return d > INT32_MAX ? INT32_MAX : (d < INT32_MIN + 1 ? INT32_MIN + 1 : (int32_t)d);
  }
};
template <> struct KeyLim<long long> {
  static constexpr long long none = LLONG_MIN;
  __device__ static long long clampD(long long d) { return d; }
};

template <int PROB, class KeyT>
__device__ __forceinline__ KeyT pair_gain(KeyT rowv, KeyT colv, int32_t w) {
  if (PROB == P_MDP) return colv - rowv - (KeyT)w;  // vg[v] - vg[u] - w(u,v)
  return rowv + colv + (KeyT)2 * (KeyT)w;           // vg[u] + vg[v] + 2 w(u,v)
}

// WSwap sweep: the gain split into a column part, maximised per row over the
// thread's columns, and the row's own term added once afterwards:
// MaxBS vg[u] + (vg[v] + 2w), MDP (vg[v] - w) - vg[u].
template <int PROB, class KeyT>
__device__ __forceinline__ KeyT wsw_col_term(KeyT colv, int32_t w) {
  if (PROB == P_MDP) return colv - (KeyT)w;
  return colv + (KeyT)2 * (KeyT)w;
}
template <int PROB, class KeyT>
__device__ __forceinline__ KeyT wsw_row_term(KeyT rowv, KeyT col_term) {
  if (PROB == P_MDP) return col_term - rowv;
  return rowv + col_term;
}

__device__ __forceinline__ bool allowed(bool row_tabu, bool col_tabu, long long x, long long D) {
  return !(row_tabu || col_tabu) || x > D;  // GPU-MDP-CSR.cu:580, GPU-MAXBS-CSR.cu:349
}

__device__ __forceinline__ int32_t warp_max(int32_t v) { return __reduce_max_sync(0xffffffffu, v); }
__device__ __forceinline__ long long warp_max(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    long long t = __shfl_xor_sync(0xffffffffu, v, o);
    v = t > v ? t : v;
  }
  return v;
}

__device__ __forceinline__ void better_rec(long long& k, long long& i, long long k2, long long i2) {
  if (k2 > k || (k2 == k && i2 < i)) { k = k2; i = i2; }
}

// Block-wide (key desc, index asc) reduction; result valid in thread 0.
__device__ __forceinline__ void block_best(long long& k, long long& i, CtaRec* scratch) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    long long k2 = __shfl_xor_sync(0xffffffffu, k, o);
    long long i2 = __shfl_xor_sync(0xffffffffu, i, o);
    better_rec(k, i, k2, i2);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) { scratch[warp].key = k; scratch[warp].idx = i; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) better_rec(k, i, scratch[w].key, scratch[w].idx);
  }
  __syncthreads();
}

// Solver-state loads.  The plain kernel (one launch per iteration) reads state
// through the read-only path: it only changes between launches.  The batched
// kernel's CTAs read state that their cluster leader changed earlier in the
// same launch (plain stores and atomics), so they use ordinary coherent loads
// (L1-cached; PERSIST): the CTA barrier, and the cluster barrier's
// release/acquire, make the leader's writes visible to them.
template <bool PERSIST, class T>
__device__ __forceinline__ T ld_st(const T* p) {
  if constexpr (PERSIST) return *p;
  else return __ldg(p);
}

// WSwap matrix rows are streamed once per iteration: evict-first in L2 so they
// do not push the small per-column arrays out.  The batched form also keeps
// them out of L1 (never allocated there, so never stale).
template <bool PERSIST>
__device__ __forceinline__ int4 ld_w4(const int32_t* p) {
  if constexpr (PERSIST) {
    int4 r;
    asm volatile(
        "{\n\t.reg .b64 pol;\n\t"
        "createpolicy.fractional.L2::evict_first.b64 pol, 1.0;\n\t"
        "ld.global.L1::no_allocate.L2::cache_hint.v4.s32 {%0,%1,%2,%3}, [%4], pol;\n\t}"
        : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
        : "l"(p));
    return r;
  } else {
    return __ldcs(reinterpret_cast<const int4*>(p));
  }
}
template <bool PERSIST>
__device__ __forceinline__ int32_t ld_w1(const int32_t* p) {
  if constexpr (PERSIST) return __ldcg(p);
  else return *p;
}
// 16-bit matrix: four weights of a row in one 8-byte load, same policies;
// kept packed until used (unpack_w16) so all rows' loads stay in flight.
template <bool PERSIST>
__device__ __forceinline__ int2 ld_w4_16(const int16_t* p) {
  int2 r;
  if constexpr (PERSIST) {
    asm volatile(
        "{\n\t.reg .b64 pol;\n\t"
        "createpolicy.fractional.L2::evict_first.b64 pol, 1.0;\n\t"
        "ld.global.L1::no_allocate.L2::cache_hint.v2.s32 {%0,%1}, [%2], pol;\n\t}"
        : "=r"(r.x), "=r"(r.y)
        : "l"(p));
  } else {
    r = __ldcs(reinterpret_cast<const int2*>(p));
  }
  return r;
}
__device__ __forceinline__ int4 unpack_w16(int2 r) {
  return make_int4((r.x << 16) >> 16, r.x >> 16, (r.y << 16) >> 16, r.y >> 16);
}

// WSwap matrix element access for either element width.
template <bool PERSIST, class KeyT>
__device__ __forceinline__ int32_t w_get(const DevSolver<KeyT>& s, long long at) {
  if (s.w16) {
    const int16_t* W16 = reinterpret_cast<const int16_t*>(s.W);
    if constexpr (PERSIST) return (int32_t)__ldcg(W16 + at);
    else return (int32_t)W16[at];
  }
  return ld_w1<PERSIST>(s.W + at);
}
template <class KeyT>
__device__ __forceinline__ void w_set(const DevSolver<KeyT>& s, long long at, int32_t v) {
  if (s.w16) reinterpret_cast<int16_t*>(s.W)[at] = (int16_t)v;
  else s.W[at] = v;
}

// Column loads: 4 contiguous columns per lane (16 B aligned since ldc % 4 == 0).
template <bool PERSIST>
__device__ __forceinline__ void load4(const int32_t* p, int32_t (&o)[4]) {
  const int4 t = ld_st<PERSIST>(reinterpret_cast<const int4*>(p));
  o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w;
}
template <bool PERSIST>
__device__ __forceinline__ void load4(const long long* p, long long (&o)[4]) {
  const longlong2 a = ld_st<PERSIST>(reinterpret_cast<const longlong2*>(p));
  const longlong2 b = ld_st<PERSIST>(reinterpret_cast<const longlong2*>(p) + 1);
  o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}

// Per-row lookup data of the staged structures.  Keys and weights are int32
// arrays read with a stride: 1 when staged in shared memory (split into a key
// array and a weight array), 2 when left in the global CSR (interleaved
// (neighbour, weight) pairs) because the row did not fit the staging budget.
struct RowDesc {
  const int32_t* key;  // BB: CSR keys; Hash: table keys; Bitset: CSR keys (hit path)
  const int32_t* wt;   // matching weights
  const uint64_t* bits;  // Bitset: bitmap words of the row
  int32_t len;         // BB / Bitset: CSR degree
  int32_t stride;      // 1 staged, 2 global CSR
  uint32_t mask;       // Hash: number of 4-slot buckets - 1
  uint32_t shift;      // Hash: 32 - log2(buckets)
  const int32_t* dir;  // BB rows in shared memory: bucket directory (nullptr: none)
  int32_t bshift;      // BB: vertex id >> bshift = directory bucket
};

// Branch-free lower_bound; the trip count depends on len only (uniform per row).
template <int STRIDE>
__device__ __forceinline__ int32_t bb_lower(const int32_t* key, const int32_t* wt, int32_t len, int32_t v) {
  int32_t lo = 0;
  int32_t step = len > 0 ? (1 << (31 - __clz(len))) : 0;
  for (; step > 0; step >>= 1)
    if (lo + step <= len && key[(lo + step - 1) * STRIDE] < v) lo += step;
  return (lo < len && key[lo * STRIDE] == v) ? wt[lo * STRIDE] : 0;
}
// Binary search of a staged row guided by its bucket directory: dir[b] is the
// lower bound of the first id of bucket b (ids split into power-of-two
// ranges, about one row entry per two buckets), so the search starts on the
// few entries that can hold v.  Same answer as a lower_bound over the
// whole row: the first entry of v, or 0.
__device__ __forceinline__ int32_t dir_lower(const RowDesc& d, int32_t v) {
  const int32_t b = v >> d.bshift;
  int32_t lo = d.dir[b], hi = d.dir[b + 1];
  while (lo < hi) {
    const int32_t mid = (lo + hi) >> 1;
    if (d.key[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return (lo < d.len && d.key[lo] == v) ? d.wt[lo] : 0;
}

__device__ __forceinline__ int32_t bb_lower(const RowDesc& d, int32_t v) {
  if (d.dir) return dir_lower(d, v);
  return d.stride == 1 ? bb_lower<1>(d.key, d.wt, d.len, v) : bb_lower<2>(d.key, d.wt, d.len, v);
}

// Bucketed probe: one 16-byte load reads a whole 4-slot bucket.
__device__ __forceinline__ int32_t hash_probe(const int32_t* key, const int32_t* wt, uint32_t gmask,
                                              uint32_t gshift, int32_t v) {
  uint32_t grp = hash_group(v, gshift);
  for (uint32_t t = 0; t <= gmask; t++) {
    const int4 k4 = *reinterpret_cast<const int4*>(key + 4u * grp);
    if (k4.x == v) return wt[4u * grp];
    if (k4.y == v) return wt[4u * grp + 1u];
    if (k4.z == v) return wt[4u * grp + 2u];
    if (k4.w == v) return wt[4u * grp + 3u];
    if (k4.x == kHashEmpty || k4.y == kHashEmpty || k4.z == kHashEmpty || k4.w == kHashEmpty) return 0;
    grp = (grp + 1u) & gmask;
  }
  return 0;
}

template <int STRIDE>
__device__ __forceinline__ int32_t scan_first(const int32_t* key, const int32_t* wt, int32_t len, int32_t v) {
  for (int32_t k = 0; k < len; k++)
    if (key[k * STRIDE] == v) return wt[k * STRIDE];
  return 0;
}

// Whole-warp linear scan of a CSR row for v (every lane passes the same v):
// 32 entries per step, the first match found with a ballot.
__device__ __forceinline__ int32_t warp_scan_first(const RowDesc& d, int32_t v) {
  const int lane = threadIdx.x & 31;
  for (int32_t base = 0; base < d.len; base += 32) {
    const int32_t k = base + lane;
    const bool hit = k < d.len && d.key[k * d.stride] == v;
    const unsigned b = __ballot_sync(0xffffffffu, hit);
    if (b) return d.wt[(base + __ffs(b) - 1) * d.stride];
  }
  return 0;
}

__device__ __forceinline__ bool bit_test(const uint64_t* words, int32_t v) {
  return (words[v >> 6] >> (v & 63)) & 1ull;
}

// One lane's lookup in a staged row (the rescan path).
template <int ST>
__device__ __forceinline__ int32_t staged_lookup(const RowDesc& d, int32_t v) {
  if (ST == S_BB) return bb_lower(d, v);
  if (ST == S_HASH) return hash_probe(d.key, d.wt, d.mask, d.shift, v);
  // Bitset guard, then the CSR row on a hit (GPU-MDP-CSR-Bitset-BuscaBinaria.cu:598-604).
  if (!bit_test(d.bits, v)) return 0;
  if (ST == S_BITSET_BB) return bb_lower(d, v);
  return d.stride == 1 ? scan_first<1>(d.key, d.wt, d.len, v) : scan_first<2>(d.key, d.wt, d.len, v);
}

// Compact descriptor of a binary-search row staged in shared memory, kept at
// the start of the staging area (one 16-byte load per row and pass): byte
// offsets from the dynamic shared-memory base, so the directory and row reads
// compile to shared-memory loads (x keys, y weights, z directory,
// w = bshift | len << 5).  x == kNotStaged: the row stayed in global memory
// (RowDesc path).  Measured on the MaxBS conflict graph (n = 100,000): 1.2x
// for CSR+BB; the same form for Hash and the bitmaps was slower than their
// RowDesc path, so they keep it.
constexpr uint32_t kNotStaged = 0xffffffffu;

template <int ST>
__device__ __forceinline__ int32_t lite_lookup(const unsigned char* base, const uint4 L, int32_t v) {
  const int32_t* key = reinterpret_cast<const int32_t*>(base + L.x);
  const int32_t* wt = reinterpret_cast<const int32_t*>(base + L.y);
  // the same search as dir_lower
  const int32_t* dir = reinterpret_cast<const int32_t*>(base + L.z);
  const int32_t b = v >> (L.w & 31u);
  int32_t lo = dir[b], hi = dir[b + 1];
  const int32_t end = hi;  // entries of bucket b: [dir[b], dir[b+1]); v can only be there
  while (lo < hi) {
    const int32_t mid = (lo + hi) >> 1;
    if (key[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return (lo < end && key[lo] == v) ? wt[lo] : 0;
}

// Generic global-memory lookup used by the exact pass.
template <int ST, class KeyT, bool PERSIST>
__device__ __forceinline__ int32_t global_lookup(const DevGraph& g, const DevSolver<KeyT>& s,
                                                 int32_t row, int32_t col, int32_t u, int32_t v) {
  if (ST == S_WSWAP) return w_get<PERSIST>(s, (long long)row * s.ldc + col);
  const long long st = g.rowptr[u];
  const int32_t deg = (int32_t)(g.rowptr[u + 1] - st);
  const int32_t* ck = reinterpret_cast<const int32_t*>(g.adj + st);
  if (ST == S_CSR) return scan_first<2>(ck, ck + 1, deg, v);
  if (ST == S_BB) return bb_lower<2>(ck, ck + 1, deg, v);
  if (ST == S_HASH) {
    const long long b = g.hoff[u];
    const long long cap = g.hoff[u + 1] - b;
    return hash_probe(g.hkey + b, g.hval + b, (uint32_t)(cap / 4 - 1), hash_gshift(cap), v);
  }
  if (!bit_test(g.bits + (long long)u * g.wpr, v)) return 0;
  return ST == S_BITSET ? scan_first<2>(ck, ck + 1, deg, v) : bb_lower<2>(ck, ck + 1, deg, v);
}

}  // namespace tsb
#include "fast.cuh"
namespace tsb {

template <class KeyT>
__device__ __forceinline__ KeyT* vg_at(const DevSolver<KeyT>& s, int32_t p) {
  return p < s.m ? s.vg_in + p : s.vg_out + (p - s.m);
}

__device__ __forceinline__ void atomic_add_key(int32_t* a, int32_t d) { atomicAdd(a, d); }
__device__ __forceinline__ void atomic_add_key(long long* a, long long d) {
  atomicAdd(reinterpret_cast<unsigned long long*>(a), (unsigned long long)d);
}

// ------------------------------------------------------------------ tail
struct TailShared {
  CtaRec red[kMaxTPB / 32];
  long long key, idx;
  int32_t action;
  int32_t wuv;
};

// Applies one swap (tabu move or perturbation move) with the whole CTA.
// Returns (in thread 0) the perturbation gain aux read after the contribution
// update, before negation (finalizeMove GPU-MAXBS-CSR.cu:381-384).
template <int PROB, int ST, class KeyT>
__device__ long long apply_swap(const DevGraph& g, const DevSolver<KeyT>& s, int32_t iu, int32_t jv,
                                long long iter, int32_t t_u, int32_t t_v, bool set_tabu,
                                TailShared& sh) {
  const int32_t m = s.m;
  const int32_t u = __ldcg(s.sol_in + iu), v = __ldcg(s.sol_out + jv);
  const long long su = g.rowptr[u], sv = g.rowptr[v];
  const int32_t nu = (int32_t)(g.rowptr[u + 1] - su), nv = (int32_t)(g.rowptr[v + 1] - sv);
  if (threadIdx.x == 0) sh.wuv = 0;
  __syncthreads();
  // The moved vertices' adjacency, kApplyBatch entries per thread in flight:
  // every load of a batch is issued before any is used (a hub row of
  // thousands of entries is a few dependent round trips, not one per 256
  // entries).  The updates are integer atomics: their order does not matter.
  // (One per thread for MaxBS WSwap, whose sweep would lose a resident CTA
  // per SM to the extra registers.)
  constexpr int kApplyBatch = (PROB == P_MAXBS && ST == S_WSWAP) ? 1 : 3;
  const int32_t total = nu + nv;
  for (int32_t base = 0; base < total; base += kApplyBatch * (int32_t)blockDim.x) {
    int2 e[kApplyBatch];
    int32_t prev[kApplyBatch];
    long long rv[kApplyBatch];
#pragma unroll
    for (int j = 0; j < kApplyBatch; j++) {
      const int32_t k = base + j * (int32_t)blockDim.x + (int32_t)threadIdx.x;
      const bool from_u = k < nu;
      const long long at = from_u ? su + k : sv + (k - nu);
      const long long rs = from_u ? su : sv;
      e[j] = make_int2(-1, 0);
      prev[j] = -1;
      rv[j] = 0;
      if (k < total) {
        e[j] = g.adj[at];
        if (at != rs) prev[j] = g.adj[at - 1].x;
        if (ST == S_CSR) rv[j] = g.rev[at];
      }
    }
    int32_t pz[kApplyBatch];
#pragma unroll
    for (int j = 0; j < kApplyBatch; j++) pz[j] = e[j].x >= 0 ? s.pos[e[j].x] : 0;
#pragma unroll
    for (int j = 0; j < kApplyBatch; j++) {
      const int32_t k = base + j * (int32_t)blockDim.x + (int32_t)threadIdx.x;
      if (k >= total) continue;
      const bool from_u = k < nu;
      const int32_t z = e[j].x, w = e[j].y, p = pz[j];
      KeyT d;
      if (PROB == P_MDP) {
        d = from_u ? -(KeyT)w : (KeyT)w;
      } else {
        const bool z_in = p < m;
        d = (from_u == z_in) ? -(KeyT)2 * (KeyT)w : (KeyT)2 * (KeyT)w;
      }
      atomic_add_key(vg_at(s, p), d);
      if (ST == S_CSR) s.cpos[rv[j]] = from_u ? m + jv : iu;  // new position of u / v
      const bool first = prev[j] != z;
      if (PROB == P_MAXBS && from_u && z == v && first) sh.wuv = w;
      if (ST == S_WSWAP && z != u && z != v) {
        // Row iu now describes v, column jv now describes u
        // (updateVertexEdgeGain, GPU-MDP-WSwap.cu:535-560).  First the
        // entries that stop being edges are cleared: row iu at u's outside
        // neighbours, column jv at v's inside neighbours ...
        if (from_u && p >= m) w_set(s, (long long)iu * s.ldc + (p - m), 0);
        if (!from_u && p < m) w_set(s, (long long)p * s.ldc + jv, 0);
      }
    }
  }
  if (ST == S_WSWAP) {
    // ... then the new edges are set: row iu at v's outside neighbours,
    // column jv at u's inside neighbours, each with the first entry of a
    // duplicated pair.  The element (iu, jv) -- w(u, v) either way -- and
    // self-loop entries (kept by the MaxBS loader) are left alone, so W keeps
    // returning the CSR lookup's w(u, v).  Plain stores: every element is
    // written by one entry, after the barrier that ends the clearing.
    __syncthreads();
    for (int32_t base = 0; base < total; base += kApplyBatch * (int32_t)blockDim.x) {
      int2 e[kApplyBatch];
      int32_t prev[kApplyBatch], pz[kApplyBatch];
#pragma unroll
      for (int j = 0; j < kApplyBatch; j++) {  // the batch's loads before any use
        const int32_t k = base + j * (int32_t)blockDim.x + (int32_t)threadIdx.x;
        const bool from_u = k < nu;
        const long long at = from_u ? su + k : sv + (k - nu);
        e[j] = make_int2(-1, 0);
        prev[j] = -1;
        if (k < total) {
          e[j] = g.adj[at];
          if (at != (from_u ? su : sv)) prev[j] = g.adj[at - 1].x;
        }
      }
#pragma unroll
      for (int j = 0; j < kApplyBatch; j++) pz[j] = e[j].x >= 0 ? s.pos[e[j].x] : 0;
#pragma unroll
      for (int j = 0; j < kApplyBatch; j++) {
        const int32_t k = base + j * (int32_t)blockDim.x + (int32_t)threadIdx.x;
        if (k >= total || e[j].x == u || e[j].x == v || prev[j] == e[j].x) continue;
        const bool from_u = k < nu;
        const int32_t p = pz[j];
        if (!from_u && p >= m) w_set(s, (long long)iu * s.ldc + (p - m), e[j].y);
        if (from_u && p < m) w_set(s, (long long)p * s.ldc + jv, e[j].y);
      }
    }
  }
  __syncthreads();
  long long aux = 0;
  if (threadIdx.x == 0) {
    // L2 reads: the contributions were just changed by atomics, and this CTA's
    // sweep may hold older copies of them in L1.
    KeyT a = __ldcg(s.vg_in + iu), b = __ldcg(s.vg_out + jv);
    if (PROB == P_MAXBS) {
      aux = (long long)a + (long long)b - 2LL * sh.wuv;
      a = -a;
      b = -b;
    }
    s.vg_in[iu] = b;   // v now inside at iu
    s.vg_out[jv] = a;  // u now outside at jv
    s.sol_in[iu] = v;
    s.sol_out[jv] = u;
    s.pos[u] = m + jv;
    s.pos[v] = iu;
    if (set_tabu) {
      s.tab_out[jv] = (int32_t)(iter + t_u);
      s.tab_in[iu] = (int32_t)(iter + t_v);
    } else {
      int32_t t = s.tab_in[iu];
      s.tab_in[iu] = s.tab_out[jv];
      s.tab_out[jv] = t;
    }
    long long ln = s.st->log_n;
    if (ln < s.log_cap) s.movelog[ln] = make_int2(iu, jv);
    else s.st->err |= E_LOG_FULL;
    s.st->log_n = ln + 1;
  }
  __syncthreads();
  return aux;
}

template <class KeyT>
__device__ __forceinline__ void trace_rec(const DevSolver<KeyT>& s, long long iter, long long idx,
                                          long long key, int32_t kind, int32_t t1, int32_t t2) {
  DevState* st = s.st;
  long long tn = st->trace_n;
  if (s.trace && tn < s.trace_cap) {
    TraceRec r;
    r.iter = iter; r.idx = idx; r.key = key; r.cur = st->cur; r.best = st->best;
    r.kind = kind; r.tenure = t1; r.tenure2 = t2; r.pad = 0;
    s.trace[tn] = r;
  }
  st->trace_n = tn + 1;
}

// Decision on the iteration's reduced (key, index) -- valid in thread 0 -- and
// application of the move by the whole CTA: switch to the exact pass, MDP
// break, or move + tabu + bookkeeping (+ MaxBS perturbation).
template <int PROB, int ST, class KeyT>
__device__ void decide_apply(const DevGraph& g, const DevSolver<KeyT>& s, int mode, long long k,
                             long long i, TailShared& sh) {
  DevState* st = s.st;
  if (threadIdx.x == 0) {
    int action = 0;  // 0: switch to exact, 1: move, 2: MDP break
    if (mode == 0) {
      if (k != LLONG_MIN && (PROB == P_MAXBS || k > kMdpSentinel)) action = 1;
    } else {
      action = (PROB == P_MDP && k == kMdpSentinel) ? 2 : 1;
    }
    if (action != 0 && (i < 0 || i >= s.P)) {  // cannot happen; never index with it
      st->err |= E_BAD_INDEX;
      st->done = 1;
      action = 3;
    }
    sh.action = action;
    sh.key = k;
    sh.idx = i;
    st->mode = action == 0 ? 1 : 0;
    if (action == 2) {
      st->evaluations += s.P;
      st->done = 1;
      st->stopped = 1;
      trace_rec(s, st->iter, i, k, 1, 0, 0);
    }
  }
  __syncthreads();
  if (sh.action != 1) return;
  const long long key = sh.key, idx = sh.idx;
  const long long iter = st->iter;
  const int32_t iu = (int32_t)(idx / s.delta), jv = (int32_t)(idx % s.delta);
  int32_t t_u, t_v, t2 = 0;
  if (PROB == P_MDP) {
    const int32_t c1 = s.tenure_policy == 0 ? mdp_ref_tenure(iter) : s.tenure;
    int32_t c2 = s.c2_fixed;
    if (s.tenure_policy == 0) c2 = s.c2_tab[c1 == 15 ? 0 : c1 == 30 ? 1 : c1 == 60 ? 2 : 3];
    t_u = c1;  // tab[u] = iter + C1 (GPU-MDP-CSR.cu:549)
    t_v = c2;  // tab[v] = iter + C2 (:550)
    t2 = c2;
  } else {
    const int32_t tt = s.tenure_policy == 0 ? maxbs_ref_tenure(iter, s.maxt) : s.tenure;
    t_u = tt;
    t_v = tt;
  }
  apply_swap<PROB, ST, KeyT>(g, s, iu, jv, iter, t_u, t_v, true, sh);
  if (threadIdx.x == 0) {
    long long cur = st->cur;
    if (PROB == P_MAXBS && key < kMaxbsRecoverBelow) cur += key + kMaxbsInf;  // :456-460
    else cur += key;
    st->cur = cur;
    st->evaluations += s.P;
    if (cur > st->best) {
      st->best = cur;
      st->best_log_n = st->log_n;
      st->isi = 0;
    } else {
      st->isi += 1;
    }
    trace_rec(s, iter, idx, key, 0, t_u, t2);
    st->iter = iter + 1;
    sh.action = (PROB == P_MAXBS && st->isi >= s.piter) ? 3 : 1;
  }
  __syncthreads();
  if (PROB == P_MAXBS && sh.action == 3) {
    const long long ev = st->pert_events - st->pert_base;
    if (ev < 0 || ev >= s.draw_events || ev >= st->pert_limit) {
      if (threadIdx.x == 0) { st->err |= E_PERTURB_WINDOW; st->done = 1; }
    } else {
      for (int32_t q = 0; q < s.num_pert; q++) {
        const long long mv = s.draws[ev * s.num_pert + q];
        if (mv < 0 || mv >= s.P) {  // never index with a bad draw (the same value in every thread)
          if (threadIdx.x == 0) { st->err |= E_BAD_INDEX; st->done = 1; }
          break;
        }
        const int32_t pu = (int32_t)(mv / s.delta), pv = (int32_t)(mv % s.delta);
        const long long aux = apply_swap<PROB, ST, KeyT>(g, s, pu, pv, iter + 1, 0, 0, false, sh);
        if (threadIdx.x == 0) {
          st->cur += aux;
          st->pert_moves += 1;
          trace_rec(s, iter + 1, mv, aux, 2, 0, 0);
        }
        __syncthreads();
      }
      if (threadIdx.x == 0) {
        st->pert_events += 1;
        st->isi = 0;
      }
    }
  }
  __syncthreads();
}

// ------------------------------------------------------------------ tile
// Best allowed pair of one tile (row block rb, column chunk ch) in the fast
// pass (mode 0), or best pair under the full reference key rule (mode 1);
// (out_key, out_idx) valid in thread 0, (LLONG_MIN, LLONG_MAX) if none.
// Used once per CTA by the plain kernel and in a loop by the batched one
// (PERSIST: state written earlier in the same launch, see ld_st).  floor_key:
// the best key the caller holds from earlier tiles; a tile whose maximum is
// below it returns no record.
// W16K (WSwap, plain kernel only): the kernel is compiled for the 16-bit
// matrix alone, so its registers are that pass's; otherwise the width is
// read from the solver at run time.
template <int PROB, int ST, class KeyT, bool PERSIST, bool W16K = false>
__device__ void tile_eval(const DevGraph& g, const DevSolver<KeyT>& s, int mode, long long iter,
                          long long D64, int rb, int ch, long long& out_key, long long& out_idx,
                          TailShared& sh, long long floor_key = LLONG_MIN, int slice = 0,
                          int nslices = 1) {
  if constexpr (std::is_same<KeyT, int32_t>::value && ST != S_WSWAP) {
    if (mode == 0 && s.fast) {
      tile_fast<PROB, ST, PERSIST>(g, s, iter, D64, rb, ch, out_key, out_idx, slice, nslices);
      return;
    }
  }
  if (slice != 0) {  // the other passes take a tile in one CTA: slice 0's
    out_key = LLONG_MIN;
    out_idx = LLONG_MAX;
    return;
  }
  constexpr int R = Rows<ST>::R;
  constexpr int TPB = TpbOf<ST, PERSIST>::v;
  using Lim = KeyLim<KeyT>;
  const KeyT D = Lim::clampD(D64);
  const int tid = threadIdx.x, lane = tid & 31;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ KeyT s_rv[kMaxTileRows];
  __shared__ int32_t s_ru[kMaxTileRows];
  __shared__ int32_t s_rtab[kMaxTileRows];
  __shared__ KeyT s_rowbest[R];
  __shared__ RowDesc s_desc[R];
  __shared__ long long s_rstart[R];
  __shared__ int32_t s_off[R + 1];
  __shared__ long long s_mc;
  __shared__ int32_t s_rstar;
  __shared__ uint32_t s_cmin;

  // the exact pass takes the solver's tile height (the fast pass's 32 rows
  // when that pass is on); the per-row-register pass below is compiled for R
  const int Rt = mode == 1 ? s.tile_rows : R;
  const int32_t r0 = rb * Rt;
  const int32_t nr = min(Rt, s.m - r0);
  const int32_t c0 = ch * s.chunk_cols;
  const int32_t c_end = min(c0 + s.chunk_cols, s.delta);

  if (tid < Rt) {
    const bool ok = tid < nr;
    s_rv[tid] = ok ? ld_st<PERSIST>(s.vg_in + r0 + tid) : (KeyT)0;
    s_ru[tid] = ok ? ld_st<PERSIST>(s.sol_in + r0 + tid) : 0;
    s_rtab[tid] = ok ? (ld_st<PERSIST>(s.tab_in + r0 + tid) > iter) : 0;
    if (tid < R) s_rowbest[tid] = Lim::none;
  }
  __syncthreads();

  long long my_key = LLONG_MIN, my_idx = LLONG_MAX;

  if (mode == 1) {
    // ---------------- exact pass: the reference's full key rule, int64.
    for (int32_t r = 0; r < nr; r++) {
      const int32_t u = s_ru[r];
      const long long rv = (long long)s_rv[r];
      const bool rt = s_rtab[r] != 0;
      const long long base = (long long)(r0 + r) * s.delta;
      for (int32_t c = c0 + tid; c < c_end; c += blockDim.x) {
        const int32_t v = ld_st<PERSIST>(s.sol_out + c);
        const long long cv = (long long)ld_st<PERSIST>(s.vg_out + c);
        const bool ct = ld_st<PERSIST>(s.tab_out + c) > iter;
        const int32_t w = global_lookup<ST, KeyT, PERSIST>(g, s, r0 + r, c, u, v);
        const long long x = pair_gain<PROB, long long>(rv, cv, w);
        long long key = x;
        if (!allowed(rt, ct, x, D64)) key = PROB == P_MDP ? kMdpSentinel : maxbs_penalty(x);
        better_rec(my_key, my_idx, key, base + c);
      }
    }
    block_best(my_key, my_idx, sh.red);
  } else {
    // ---------------- fast pass
    uint32_t* s_mask = reinterpret_cast<uint32_t*>(smem_raw);  // CSR + MDP: adjacency per column
    uint4* s_lite = reinterpret_cast<uint4*>(smem_raw);       // CSR+BB: row descriptors
    // CSR: adjacent pairs leave the w-free sweep (MDP always; MaxBS when a
    // weight is negative) and are evaluated exactly by the join below
    const bool masked = PROB == P_MDP || s.adj_mask != 0;
    if (ST == S_CSR) {
      if (masked)
        for (int32_t c = tid; c < s.chunk_cols; c += blockDim.x) s_mask[c] = 0u;
      if (tid < 32) {
        // row segments and their prefix (one lane per row)
        long long a0 = 0;
        int32_t d = 0;
        if (lane < nr) {
          a0 = g.rowptr[s_ru[lane]];
          d = (int32_t)(g.rowptr[s_ru[lane] + 1] - a0);
          s_rstart[lane] = a0;
        }
        int32_t incl = d;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += t;
        }
        if (lane < R) s_off[lane + 1] = incl;
        if (lane == 0) s_off[0] = 0;
      }
    } else if (ST != S_WSWAP) {
      if (tid == 0) {
        // CSR+BB: the rows' compact descriptors take the first 16 * R bytes
        long long off = ST == S_BB ? 16LL * R : 0;  // bytes used in the staging area, 16 B aligned
        for (int r = 0; r < R; r++) {
          RowDesc d;
          d.key = nullptr; d.wt = nullptr; d.bits = nullptr;
          d.len = 0; d.stride = 2; d.mask = 0; d.shift = 0; d.dir = nullptr; d.bshift = 0;
          if (r < nr) {
            const int32_t u = s_ru[r];
            const long long rs = g.rowptr[u];
            const int32_t* ck = reinterpret_cast<const int32_t*>(g.adj + rs);
            d.len = (int32_t)(g.rowptr[u + 1] - rs);
            if (ST == S_HASH) {
              const long long hb = g.hoff[u];
              const long long cap = g.hoff[u + 1] - hb;
              d.mask = (uint32_t)(cap / 4 - 1);
              d.shift = hash_gshift(cap);
              d.key = g.hkey + hb;
              d.wt = g.hval + hb;
              d.stride = 1;
              const long long b = (4LL * cap + 15) & ~15LL;  // per array
              if (off + 2 * b <= s.stage_bytes) {
                d.key = reinterpret_cast<const int32_t*>(smem_raw + off);
                d.wt = reinterpret_cast<const int32_t*>(smem_raw + off + b);
                off += 2 * b;
              }
            } else {
              d.key = ck;  // BB rows, and the Bitset hit path
              d.wt = ck + 1;
              if (ST == S_BITSET || ST == S_BITSET_BB) {
                d.bits = g.bits + (long long)u * g.wpr;
                const long long b = 8LL * g.wpr;
                if (off + b <= s.stage_bytes) {
                  d.bits = reinterpret_cast<const uint64_t*>(smem_raw + off);
                  off += b;
                }
              }
            }
          }
          s_desc[r] = d;
        }
        if (ST != S_HASH) {  // CSR rows after the bitmaps, split into keys and weights
          int32_t lg_n = 0;
          while ((1LL << lg_n) < (long long)g.n) lg_n++;
          for (int r = 0; r < nr; r++) {
            const int32_t len = s_desc[r].len;
            const long long b = (4LL * len + 15) & ~15LL;
            // binary-search rows also get a bucket directory (~0.5 entries per
            // bucket: most absent neighbours land in an empty bucket)
            int32_t lg_nb = 0;
            if (ST == S_BB || ST == S_BITSET_BB) {
              lg_nb = 4;
              while ((1 << lg_nb) < 2 * len && lg_nb < 12) lg_nb++;
            }
            const long long bd = (ST == S_BB || ST == S_BITSET_BB) ? ((4LL * ((1 << lg_nb) + 1) + 15) & ~15LL) : 0;
            if (off + 2 * b + bd <= s.stage_bytes) {
              s_desc[r].key = reinterpret_cast<const int32_t*>(smem_raw + off);
              s_desc[r].wt = reinterpret_cast<const int32_t*>(smem_raw + off + b);
              s_desc[r].stride = 1;
              if (bd) {
                s_desc[r].dir = reinterpret_cast<const int32_t*>(smem_raw + off + 2 * b);
                s_desc[r].bshift = lg_n > lg_nb ? lg_n - lg_nb : 0;
                s_desc[r].mask = (uint32_t)(1 << lg_nb);  // buckets (directory has one more entry)
              }
              off += 2 * b + bd;
            }
          }
        }
        auto soff = [](const void* p) {
          return (uint32_t)(reinterpret_cast<const unsigned char*>(p) - smem_raw);
        };
        if (ST == S_BB)
          for (int r = 0; r < R; r++) {
            uint4 L = make_uint4(kNotStaged, 0u, 0u, 0u);
            const RowDesc& d = s_desc[r];
            if (r < nr && d.dir)
              L = make_uint4(soff(d.key), soff(d.wt), soff(d.dir), (uint32_t)d.bshift | ((uint32_t)d.len << 5));
            s_lite[r] = L;
          }
      }
    }
    __syncthreads();
    if (ST == S_CSR) {
      // Join the rows' CSR segments with the chunk by position: cpos[k] is the
      // current position of entry k's neighbour, so adjacent pairs of the tile
      // are found with contiguous reads.  They are evaluated exactly here; for
      // MDP they are also masked out of the sweep (their w-free gain would be
      // an over-estimate).  For MaxBS with every weight >= 0 the w-free gain
      // is an under-estimate and harmless; a graph with a negative weight
      // masks them too.
      const int32_t total = s_off[nr];
      for (int32_t f = tid; f < total; f += blockDim.x) {
        int32_t lo = 0, hi = nr - 1;  // row r with s_off[r] <= f < s_off[r+1]
        while (lo < hi) {
          const int32_t mid = (lo + hi + 1) >> 1;
          if (s_off[mid] <= f) lo = mid; else hi = mid - 1;
        }
        const int32_t r = lo;
        const long long k = s_rstart[r] + (f - s_off[r]);
        const int32_t c = ld_st<PERSIST>(s.cpos + k) - s.m;
        if (c < c0 || c >= c_end) continue;
        const int2 e = g.adj[k];
        if (k > s_rstart[r] && g.adj[k - 1].x == e.x) continue;  // duplicate pair: first entry wins
        if (masked) atomicOr(&s_mask[c - c0], 1u << r);
        const KeyT x = pair_gain<PROB, KeyT>(s_rv[r], ld_st<PERSIST>(s.vg_out + c), e.y);
        if (allowed(s_rtab[r] != 0, ld_st<PERSIST>(s.tab_out + c) > iter, (long long)x, (long long)D))
          atomicMax(&s_rowbest[r], x);
      }
    } else if (ST != S_WSWAP) {
      for (int r = 0; r < nr; r++) {
        const RowDesc d = s_desc[r];
        const int32_t u = s_ru[r];
        if ((ST == S_BITSET || ST == S_BITSET_BB) && __isShared(d.bits)) {
          // bitmap rows start on 16 B (wpr is even)
          const uint4* src = reinterpret_cast<const uint4*>(g.bits + (long long)u * g.wpr);
          uint4* dst = reinterpret_cast<uint4*>(const_cast<uint64_t*>(d.bits));
          for (long long q = tid; q < g.wpr / 2; q += TPB) dst[q] = __ldg(src + q);
        }
        if (__isShared(d.key)) {
          int32_t* dk = const_cast<int32_t*>(d.key);
          int32_t* dw = const_cast<int32_t*>(d.wt);
          if (ST == S_HASH) {
            const long long hb = g.hoff[u];
            const long long slots = 4LL * ((long long)d.mask + 1);
            for (long long q = tid; q < slots; q += TPB) {
              dk[q] = __ldg(g.hkey + hb + q);
              dw[q] = __ldg(g.hval + hb + q);
            }
          } else {
            const int2* src = g.adj + g.rowptr[u];
            for (int32_t q = tid; q < d.len; q += TPB) {
              const int2 e = __ldg(src + q);
              dk[q] = e.x;
              dw[q] = e.y;
            }
          }
        }
      }
    }
    __syncthreads();
    if (ST == S_BB || ST == S_BITSET_BB) {
      // bucket directories of the staged rows: dir[b] = lower_bound(b << bshift)
      for (int r = 0; r < nr; r++) {
        const RowDesc d = s_desc[r];
        if (!d.dir) continue;
        int32_t* dd = const_cast<int32_t*>(d.dir);
        for (int32_t b = tid; b <= (int32_t)d.mask; b += TPB) {
          const long long lim = (long long)b << d.bshift;
          int32_t lo = 0, len = d.len;
          while (len > 0) {
            const int32_t half = len >> 1;
            if ((long long)d.key[lo + half] < lim) { lo += half + 1; len -= half + 1; }
            else len = half;
          }
          dd[b] = lo;
        }
      }
      __syncthreads();
    }

    KeyT best[R];  // this thread's maximum per row
#pragma unroll
    for (int r = 0; r < R; r++) best[r] = Lim::none;

    // Bitmap structures with every row's bitmap staged: the rows' shared
    // offsets stay in registers and each pair is one 32-bit shared load and a
    // bit extract (lean path below).
    uint32_t rbase[R];
    bool bm_staged = false;
    if (ST == S_BITSET || ST == S_BITSET_BB) {
      bm_staged = true;
#pragma unroll
      for (int r = 0; r < R; r++) {
        const uint64_t* b = s_desc[r].bits;
        const bool in_smem = r < nr && __isShared(b);
        bm_staged &= r >= nr || in_smem;
        rbase[r] = in_smem ? (uint32_t)(reinterpret_cast<const unsigned char*>(b) - smem_raw) : 0u;
      }
    }

    const int passes = s.chunk_cols / (TPB * kColsPerLane);
    // The WSwap matrix element width is a compile-time choice of the pass
    // loop, so each width gets its own register allocation.
    auto sweep_passes = [&](auto w16_tag) {
      constexpr bool W16 = decltype(w16_tag)::value;
      for (int pass = 0; pass < passes; pass++) {
        const int32_t cb = c0 + (pass * TPB + tid) * kColsPerLane;
        const bool lane_on = cb < c_end;
        if (ST == S_BITSET || ST == S_BITSET_BB) {
          // the bitmap paths vote across the warp: leave the loop together
          if (__all_sync(0xffffffffu, !lane_on)) break;
        } else if (!lane_on) {
          break;
        }
        KeyT cv[4];
        int32_t ct4[4];
        bool valid[4], ct[4];
        if (ST == S_WSWAP) {
          // Issue every row's W load of this pass before using any: the matrix
          // streams from HBM once per iteration.
          int4 wv[W16 ? 1 : R];
          int2 wp[W16 ? R : 1];
          if constexpr (W16) {
            const int16_t* W16p = reinterpret_cast<const int16_t*>(s.W);
  #pragma unroll
            for (int r = 0; r < R; r++) wp[r] = ld_w4_16<PERSIST>(W16p + (long long)(r0 + r) * s.ldc + cb);
          } else {
  #pragma unroll
            for (int r = 0; r < R; r++) wv[r] = ld_w4<PERSIST>(s.W + (long long)(r0 + r) * s.ldc + cb);
          }
          load4<PERSIST>(s.vg_out + cb, cv);
          load4<PERSIST>(s.tab_out + cb, ct4);
  #pragma unroll
          for (int q = 0; q < 4; q++) {
            valid[q] = cb + q < c_end;
            ct[q] = ct4[q] > iter;
          }
          // best[r] holds the row's maximum of the column part of the gain
          // (MaxBS vg[v] + 2w, MDP vg[v] - w); the row's own term is added
          // once per row after the sweep (wsw_row_term)
          const bool plain4 = valid[0] && valid[1] && valid[2] && valid[3] && !(ct[0] || ct[1] || ct[2] || ct[3]);
  #pragma unroll
          for (int r = 0; r < R; r++) {
            int4 wr;
            if constexpr (W16) wr = unpack_w16(wp[r]);
            else wr = wv[r];
            const int32_t w4[4] = {wr.x, wr.y, wr.z, wr.w};
            if (plain4) {
              KeyT m = wsw_col_term<PROB, KeyT>(cv[0], w4[0]);
  #pragma unroll
              for (int q = 1; q < 4; q++) {
                const KeyT y = wsw_col_term<PROB, KeyT>(cv[q], w4[q]);
                m = y > m ? y : m;
              }
              best[r] = m > best[r] ? m : best[r];
            } else {
              const KeyT t = s_rv[r];
  #pragma unroll
              for (int q = 0; q < 4; q++) {
                const KeyT y = wsw_col_term<PROB, KeyT>(cv[q], w4[q]);
                const KeyT x = wsw_row_term<PROB, KeyT>(t, y);
                if (valid[q] && (!ct[q] || x > D)) best[r] = y > best[r] ? y : best[r];
              }
            }
          }
          continue;
        }
        if (lane_on) {
          load4<PERSIST>(s.vg_out + cb, cv);
          load4<PERSIST>(s.tab_out + cb, ct4);
        } else {
  #pragma unroll
          for (int q = 0; q < 4; q++) { cv[q] = 0; ct4[q] = 0; }
        }
  #pragma unroll
        for (int q = 0; q < 4; q++) {
          valid[q] = lane_on && cb + q < c_end;
          ct[q] = ct4[q] > iter;
        }
        if (ST == S_CSR) {
          uint32_t mk[4];
  #pragma unroll
          for (int q = 0; q < 4; q++) {
            mk[q] = valid[q] ? (masked ? s_mask[cb + q - c0] : 0u) : 0xffffffffu;
            if (valid[q] && ct[q]) {
              // Tabu column: a pair is allowed only when aspirated (gain > best - cur).
  #pragma unroll
              for (int r = 0; r < R; r++)
                if (!(pair_gain<PROB, KeyT>(s_rv[r], cv[q], 0) > D)) mk[q] |= 1u << r;
            }
          }
          if ((mk[0] | mk[1] | mk[2] | mk[3]) == 0u) {
  #pragma unroll
            for (int r = 0; r < R; r++) {
              const KeyT t = s_rv[r];
  #pragma unroll
              for (int q = 0; q < 4; q++) {
                const KeyT x = pair_gain<PROB, KeyT>(t, cv[q], 0);
                best[r] = x > best[r] ? x : best[r];
              }
            }
          } else {
  #pragma unroll
            for (int r = 0; r < R; r++) {
              const KeyT t = s_rv[r];
  #pragma unroll
              for (int q = 0; q < 4; q++) {
                const KeyT x = pair_gain<PROB, KeyT>(t, cv[q], 0);
                if (!((mk[q] >> r) & 1u)) best[r] = x > best[r] ? x : best[r];
              }
            }
          }
        } else {
          int32_t vx[4] = {0, 0, 0, 0};
          if (lane_on) load4<PERSIST>(s.sol_out + cb, vx);
          if ((ST == S_BITSET || ST == S_BITSET_BB) && bm_staged) {
            // Lean bitmap path.  Columns past the chunk read word 0 of the row
            // and are masked by `valid`.  Pairs that hit
            // (rare: deg / n) get their weight from the row in a warp-uniform
            // branch; when every lane's four columns are valid and non-tabu the
            // gain goes straight into the maximum.
            uint32_t wofs[4], bsh[4];
  #pragma unroll
            for (int q = 0; q < 4; q++) {
              const uint32_t vv = valid[q] ? (uint32_t)vx[q] : 0u;  // in-bounds word for any lane
              wofs[q] = (vv >> 5) << 2;
              bsh[q] = vv & 31u;
            }
            const bool simple = valid[0] && valid[1] && valid[2] && valid[3] && !(ct[0] || ct[1] || ct[2] || ct[3]);
            const bool wsimple = __all_sync(0xffffffffu, simple);
  #pragma unroll
            for (int r = 0; r < R; r++) {
              if (r >= nr) continue;
              const KeyT t = s_rv[r];
              const unsigned char* rb = smem_raw + rbase[r];
              bool hq[4];
  #pragma unroll
              for (int q = 0; q < 4; q++)
                hq[q] = valid[q] && ((*reinterpret_cast<const uint32_t*>(rb + wofs[q]) >> bsh[q]) & 1u);
              int32_t wq[4] = {0, 0, 0, 0};
              unsigned any = __ballot_sync(0xffffffffu, hq[0] | hq[1] | hq[2] | hq[3]);
              if (any) {
                const RowDesc d = s_desc[r];
                if (ST == S_BITSET) {
                  // each hit resolved by the whole warp scanning the row 32 entries at a time
                  while (any) {
                    const int L = __ffs(any) - 1;
                    any &= any - 1;
  #pragma unroll
                    for (int q = 0; q < 4; q++) {
                      const int32_t hv = __shfl_sync(0xffffffffu, hq[q] ? vx[q] : -1, L);
                      if (hv >= 0) {
                        const int32_t ww = warp_scan_first(d, hv);
                        if (lane == L) wq[q] = ww;
                      }
                    }
                  }
                } else {
  #pragma unroll
                  for (int q = 0; q < 4; q++)
                    if (hq[q]) wq[q] = bb_lower(d, vx[q]);
                }
              }
              if (wsimple) {
  #pragma unroll
                for (int q = 0; q < 4; q++) {
                  const KeyT x = pair_gain<PROB, KeyT>(t, cv[q], wq[q]);
                  best[r] = x > best[r] ? x : best[r];
                }
              } else {
  #pragma unroll
                for (int q = 0; q < 4; q++) {
                  const KeyT x = pair_gain<PROB, KeyT>(t, cv[q], wq[q]);
                  if (valid[q] && (!ct[q] || x > D)) best[r] = x > best[r] ? x : best[r];
                }
              }
            }
            continue;
          }
  #pragma unroll
          for (int r = 0; r < R; r++) {
            if (r >= nr) continue;
            const KeyT t = s_rv[r];
            int32_t wq[4];
            if (ST == S_BB && s_lite[r].x != kNotStaged) {
              const uint4 L = s_lite[r];  // the same for the whole CTA: a uniform branch
  #pragma unroll
              for (int q = 0; q < 4; q++) wq[q] = valid[q] ? lite_lookup<ST>(smem_raw, L, vx[q]) : 0;
            } else if (ST == S_BITSET) {
              const RowDesc d = s_desc[r];
              // Bit test per pair; each hit is resolved by the whole warp
              // scanning the row 32 entries at a time (first match by ballot).
              bool hq[4];
  #pragma unroll
              for (int q = 0; q < 4; q++) {
                hq[q] = valid[q] && bit_test(d.bits, vx[q]);
                wq[q] = 0;
              }
              unsigned any = __ballot_sync(0xffffffffu, hq[0] | hq[1] | hq[2] | hq[3]);
              while (any) {
                const int L = __ffs(any) - 1;
                any &= any - 1;
  #pragma unroll
                for (int q = 0; q < 4; q++) {
                  const int32_t hv = __shfl_sync(0xffffffffu, hq[q] ? vx[q] : -1, L);
                  if (hv >= 0) {
                    const int32_t ww = warp_scan_first(d, hv);
                    if (lane == L) wq[q] = ww;
                  }
                }
              }
            } else {
              const RowDesc d = s_desc[r];
  #pragma unroll
              for (int q = 0; q < 4; q++) wq[q] = valid[q] ? staged_lookup<ST>(d, vx[q]) : 0;
            }
  #pragma unroll
            for (int q = 0; q < 4; q++) {
              const KeyT x = pair_gain<PROB, KeyT>(t, cv[q], wq[q]);
              if (valid[q] && (!ct[q] || x > D)) best[r] = x > best[r] ? x : best[r];
            }
          }
        }
      }
    };
    if constexpr (ST == S_WSWAP && W16K) {
      sweep_passes(std::true_type{});
    } else if constexpr (ST == S_WSWAP) {
      if (s.w16) sweep_passes(std::true_type{});
      else sweep_passes(std::false_type{});
    } else {
      sweep_passes(std::false_type{});
    }

    if (ST == S_WSWAP) {
#pragma unroll
      for (int r = 0; r < R; r++)
        if (best[r] != Lim::none) best[r] = wsw_row_term<PROB, KeyT>(s_rv[r], best[r]);
    }
    // Per-row block maximum.
#pragma unroll
    for (int r = 0; r < R; r++) {
      const KeyT v = warp_max(best[r]);
      if (lane == 0 && v != Lim::none) atomicMax(&s_rowbest[r], v);
    }
    __syncthreads();
    if (tid == 0) {
      long long mc = LLONG_MIN;
      int32_t rstar = -1;
      for (int r = 0; r < nr; r++) {
        const KeyT v = s_rowbest[r];
        if (v == Lim::none) continue;
        if (s_rtab[r] && !(v > D)) continue;  // tabu row: only aspirated pairs
        if ((long long)v > mc) { mc = (long long)v; rstar = r; }
      }
      s_mc = mc;
      // A tile whose maximum is below what the caller already holds cannot
      // win the iteration: skip its rescan.
      s_rstar = mc < floor_key ? -1 : rstar;
      s_cmin = 0xffffffffu;
    }
    __syncthreads();
    if (s_rstar >= 0) {
      // Rescan the winning row: lowest column whose allowed gain equals the maximum.
      const int32_t r = s_rstar;
      const KeyT target = (KeyT)s_mc;
      const KeyT t = s_rv[r];
      const bool rt = s_rtab[r] != 0;
      // Only a thread whose own maximum of this row equals the target swept a
      // matching column, so only such threads (usually one) hold the answer.
      // Each one's columns (pass-major, then the four of a pass: ascending)
      // are rescanned by its whole warp, one column per lane, 32 at a time,
      // so the loads of a round are all in flight together; the lowest
      // matching lane of the first round with a match is that thread's
      // lowest matching column.
      KeyT mine = Lim::none;
#pragma unroll
      for (int rr = 0; rr < R; rr++)
        if (rr == r) mine = best[rr];
      uint32_t cmin = 0xffffffffu;
      unsigned who = __ballot_sync(0xffffffffu, mine == target);
      const int32_t ncols = passes * kColsPerLane;
      while (who) {
        const int32_t tt = (tid & ~31) + (__ffs(who) - 1);
        who &= who - 1;
        for (int32_t j0 = 0; j0 < ncols; j0 += 32) {
          const int32_t j = j0 + lane;
          const int32_t c = c0 + ((j / kColsPerLane) * TPB + tt) * kColsPerLane + (j % kColsPerLane);
          bool hit = false;
          if (j < ncols && c < c_end) {
            int32_t w = 0;
            bool skip = false;
            if (ST == S_CSR) {
              // adjacent pairs are matched below from the row's entries; when
              // not masked (MaxBS, w >= 0) an adjacent pair's w-free gain never
              // exceeds its exact gain, so it cannot equal the row maximum alone.
              skip = masked && ((s_mask[c - c0] >> r) & 1u);
            } else if (ST == S_WSWAP) {
              w = w_get<PERSIST>(s, (long long)(r0 + r) * s.ldc + c);
            } else {
              w = staged_lookup<ST>(s_desc[r], ld_st<PERSIST>(s.sol_out + c));
            }
            const KeyT x = pair_gain<PROB, KeyT>(t, ld_st<PERSIST>(s.vg_out + c), w);
            hit = !skip && x == target &&
                  allowed(rt, ld_st<PERSIST>(s.tab_out + c) > iter, (long long)x, (long long)D);
          }
          const unsigned hb = __ballot_sync(0xffffffffu, hit);
          if (hb) {
            const uint32_t cc = (uint32_t)__shfl_sync(0xffffffffu, c, __ffs(hb) - 1);
            cmin = cc < cmin ? cc : cmin;
            break;
          }
        }
      }
      if (ST == S_CSR) {
        const long long a0 = s_rstart[r], a1 = a0 + (s_off[r + 1] - s_off[r]);
        for (long long k = a0 + tid; k < a1; k += blockDim.x) {
          const int32_t c = ld_st<PERSIST>(s.cpos + k) - s.m;
          if (c < c0 || c >= c_end) continue;
          const int2 e = g.adj[k];
          if (k > a0 && g.adj[k - 1].x == e.x) continue;
          const KeyT x = pair_gain<PROB, KeyT>(t, ld_st<PERSIST>(s.vg_out + c), e.y);
          if (x == target && allowed(rt, ld_st<PERSIST>(s.tab_out + c) > iter, (long long)x, (long long)D) &&
              (uint32_t)c < cmin)
            cmin = (uint32_t)c;
        }
      }
      cmin = __reduce_min_sync(0xffffffffu, cmin);
      if (lane == 0 && cmin != 0xffffffffu) atomicMin(&s_cmin, cmin);
      __syncthreads();
      if (tid == 0 && s_cmin != 0xffffffffu) {
        my_key = s_mc;
        my_idx = (long long)(r0 + r) * s.delta + s_cmin;
      }
    }
  }

  out_key = my_key;
  out_idx = my_idx;
  __syncthreads();  // the tile's shared arrays are reused by the next call
}

// ------------------------------------------------------------------ kernel
// Plain form: one launch = one iteration; CTA b evaluates tile b, the last
// CTA to finish reduces the records and applies the move.
// Minimum resident CTAs per SM the plain kernel is compiled for (0: left to
// the compiler).  The 512-thread index structures are held to two CTAs per SM
// (at most 64 registers): their sweep hides latency with warps.  WSwap is
// left to the compiler (holding its 32-bit matrix kernel to 64-80 registers
// spilled its 16 rows of packed matrix loads), except the Max Bisection
// kernel for the 16-bit matrix: held to four CTAs per SM (64 registers) it
// keeps more matrix loads in flight and streams the n = 100,000 matrix at
// 0.81 of measured HBM instead of 0.73.  The MDP one lost there (0.60 instead
// of 0.65 on the Chung-Lu n = 200,000 case) and stays at three.
template <int PROB, int ST, class KeyT, bool W16K = false> struct IterMinBlocks {
  static constexpr int v = (ST == S_WSWAP && W16K && PROB == P_MAXBS) ? 4
                           : (ST == S_CSR || ST == S_WSWAP) ? 0 : 2;
};

template <int PROB, int ST, class KeyT, bool W16K = false>
__global__ void __launch_bounds__(Tpb<ST>::v, (IterMinBlocks<PROB, ST, KeyT, W16K>::v))
iter_kernel(const DevGraph g, const DevSolver<KeyT> s) {
  // Small grids are launched with programmatic stream serialization: the
  // previous iteration's grid may still be finishing.  Wait for it (all of
  // its memory visible), then let the next iteration's grid be scheduled.
  // (Both are no-ops for a grid launched without that attribute.)
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  DevState* st = s.st;
  if (st->done || st->iter >= st->target) return;
  const int mode = st->mode;
  const long long iter = st->iter;
  const long long D64 = st->best - st->cur;
  __shared__ TailShared sh;
  __shared__ int32_t s_last;
  long long k, i;
  // CTA -> (tile, slice): the slices of a tile are adjacent CTAs
  const int ns = s.n_slices > 1 ? s.n_slices : 1;
  const int tile = (int)blockIdx.x / ns, slice = (int)blockIdx.x % ns;
  tile_eval<PROB, ST, KeyT, false, W16K>(g, s, mode, iter, D64, tile / s.n_chunks, tile % s.n_chunks, k, i, sh,
                                         LLONG_MIN, slice, ns);
  if (threadIdx.x == 0) {
    CtaRec rec;
    rec.key = k;
    rec.idx = i;
    s.recs[blockIdx.x] = rec;
    __threadfence();
    const unsigned prev = atomicAdd(&st->counter, 1u);
    s_last = prev == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  k = LLONG_MIN;
  i = LLONG_MAX;
  // Grids of more CTAs than threads: kRecBatch records per thread in flight
  // per round (thousands of tiles are otherwise a chain of dependent L2
  // round trips); smaller ones read one record per thread.
  constexpr int kRecBatch = 8;
  if ((int)gridDim.x <= (int)blockDim.x) {
    if ((int)threadIdx.x < (int)gridDim.x)
      better_rec(k, i, __ldcg(&s.recs[threadIdx.x].key), __ldcg(&s.recs[threadIdx.x].idx));
  } else {
    for (int b0 = threadIdx.x; b0 < (int)gridDim.x; b0 += kRecBatch * blockDim.x) {
      longlong2 r[kRecBatch];
#pragma unroll
      for (int j = 0; j < kRecBatch; j++) {
        const int b = b0 + j * (int)blockDim.x;
        r[j] = b < (int)gridDim.x ? __ldcg(reinterpret_cast<const longlong2*>(&s.recs[b]))
                                  : make_longlong2(LLONG_MIN, LLONG_MAX);
      }
#pragma unroll
      for (int j = 0; j < kRecBatch; j++) better_rec(k, i, r[j].x, r[j].y);
    }
  }
  block_best(k, i, sh.red);
  decide_apply<PROB, ST, KeyT>(g, s, mode, k, i, sh);
  if (threadIdx.x == 0) st->counter = 0;
}

}  // namespace tsb
