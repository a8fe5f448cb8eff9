// fast.cuh -- the fast pass of a tile with 32-bit keys: one structure query
// per column for all 32 rows of the tile, and the per-row maximum factored out.
//
// The reference evaluates every pair (u, v) with its own lookup of w(u, v)
// (calculateSwapGain / calculateMoveGain, src/mdp/GPU-MDP-CSR.cu:567-584,
// src/maxbisection/GPU-MAXBS-CSR.cu:337-353, and the lookups of the five
// other structures).  Here a tile of 32 inside positions (rows) first builds,
// in shared memory and from its own structure, an index of the rows'
// adjacency:
//   Hash          a multimap of (neighbour -> row, weight) records, filled from
//                 the rows' per-vertex hash tables; probed by hashing;
//   CSR+BB        the rows' CSR entries (bulk-copied into shared memory) sorted
//                 into a bucket directory; probed by directory + binary search;
//   CSR+Bitset(+BB) the union of the rows' bitmap rows (one bit per vertex),
//                 a rank directory and per-vertex row masks; probed by one bit
//                 test; a hit resolves the weight in the row's bulk-copied CSR
//                 entries by a linear scan (CSR+Bitset) or a binary search
//                 (CSR+Bitset+BB), as the two reference structures do;
//   CSR           the join of the rows' CSR entries with the columns through
//                 cpos (no per-column query: adjacent columns are marked).
// Each column v is then queried once for the whole tile.  A non-adjacent,
// non-tabu column gives every row the w-free gain, whose maximum over such
// columns is the row's value plus the largest column contribution -- so the
// sweep keeps, per thread, only the two largest column contributions (with
// the rows each column is adjacent to).  Adjacent columns go to a queue and
// their pairs are evaluated exactly; tabu columns are evaluated for every row
// on the spot (allowed only when aspirated).  Each row's result is the best of
// its exact pairs and its first top entry it is not adjacent to; a row adjacent
// to every top entry is swept again alone.  Results per row are packed
// (key, column) records, so ties go to the lowest column as in the CUB ArgMax
// tie rule; rows are merged in order, so ties across rows go to the lowest
// flat index.
#pragma once
#include <climits>
#include <cstdint>

#include "ts_internal.cuh"

namespace tsb {

constexpr int kFastRows = 32;  // rows per tile: one bit each in a 32-bit mask
constexpr int kTabuQueue = 1024;  // tabu columns a tile evaluates warp-wide (more: per lane)
constexpr int kTrack = 4;          // high-degree rows whose own best free column the sweep tracks
constexpr int32_t kTrackDeg = 256; // ... from this degree up
constexpr int kTopK = 2;       // column candidates kept per thread and per tile (the
                               // per-thread insertion below is written out for two)

// ---------------------------------------------------------------- layout
// Dynamic shared memory of the fast pass (byte offsets), the same on the host
// (launch size) and the device.  ecap: index capacity in row entries per
// group of rows; wpr: bitmap words per row.
struct FastLayout {
  uint32_t keys, recs, queue, stage, dir, uni, rank, masks, total;
  int32_t ecap, hslots, dirmax, uwords;
};

__host__ __device__ inline uint32_t al16(uint64_t b) { return (uint32_t)((b + 15) & ~15ull); }

__host__ __device__ inline FastLayout fast_layout(int st, int32_t ecap, int64_t wpr) {
  FastLayout L;
  L.keys = L.recs = L.queue = L.stage = L.dir = L.uni = L.rank = L.masks = 0;
  L.ecap = ecap;
  L.hslots = 4 * ((3 * ecap / 2 + 3) / 4 + 1);
  int32_t d = 16;
  while (d < 2 * ecap) d <<= 1;
  L.dirmax = d;
  L.uwords = (int32_t)(2 * wpr);
  const uint32_t stage_b = al16(8ull * (ecap + 2 * kFastRows + 2));
  uint32_t off = 0;
  if (st == S_HASH) {
    L.keys = off; off += al16(4ull * L.hslots);
    L.recs = off; off += al16(8ull * L.hslots);
    L.queue = off; off += al16(4ull * ecap);
  } else if (st == S_BB) {
    L.stage = off; L.queue = off; off += stage_b;  // the queue reuses the staging area
    L.keys = off; off += al16(4ull * ecap);
    L.recs = off; off += al16(8ull * ecap);
    L.dir = off; off += al16(2ull * (d + 2));
  } else if (st == S_BITSET || st == S_BITSET_BB) {
    L.uni = off; off += al16(4ull * L.uwords);
    L.rank = off; off += al16(2ull * L.uwords);
    L.masks = off; off += al16(4ull * ecap);
    L.stage = off; off += stage_b;
    L.queue = off; off += al16(4ull * ecap);
  }
  L.total = off;
  return L;
}

// Largest index capacity whose layout fits `budget` bytes (0: none fits).
__host__ inline int32_t fast_ecap_for(int st, int64_t wpr, uint32_t budget) {
  for (int32_t e = 4096; e >= 256; e >>= 1)
    if (fast_layout(st, e, wpr).total <= budget) return e;
  return 0;
}

// ---------------------------------------------------------------- helpers
// (key, column) of a row packed so that a larger key, then a smaller column,
// compares larger; 0 is below every record of a real pair (|key| < 2^30).
__device__ __forceinline__ unsigned long long pack_kc(int32_t x, int32_t c) {
  return ((unsigned long long)((uint32_t)x ^ 0x80000000u) << 32) | (unsigned long long)(~(uint32_t)c);
}
__device__ __forceinline__ int32_t unpack_key(unsigned long long p) {
  return (int32_t)((uint32_t)(p >> 32) ^ 0x80000000u);
}
__device__ __forceinline__ int32_t unpack_col(unsigned long long p) { return (int32_t)(~(uint32_t)p); }

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
  const uint32_t hi = __reduce_max_sync(0xffffffffu, (uint32_t)(v >> 32));
  const uint32_t lo = __reduce_max_sync(0xffffffffu, (uint32_t)(v >> 32) == hi ? (uint32_t)v : 0u);
  return ((unsigned long long)hi << 32) | lo;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// mbarrier + 1-D bulk copy global -> shared (single GPU, no multicast).
__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// Waits for phase 0 of the barrier for at most `limit_ns`; false on timeout.
__device__ __forceinline__ bool mbar_wait0(unsigned long long* bar, unsigned long long limit_ns) {
  const unsigned long long t0 = global_ns();
  for (;;) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar))
        : "memory");
    if (ok) return true;
    if (global_ns() - t0 > limit_ns) return false;
  }
}

__device__ __forceinline__ uint32_t fast_bucket(int32_t v, uint32_t nb) {
  return (uint32_t)(((unsigned long long)((uint32_t)v * 2654435769u) * nb) >> 32);
}

// Tile state of the fast pass (static shared memory).
struct FastSh {
  int32_t ru[kFastRows];
  int32_t rv[kFastRows];
  int32_t rtab[kFastRows];
  int32_t rdeg[kFastRows];      // CSR degree of each row
  long long rrow[kFastRows];    // rowptr[u] of each row
  long long rhb[kFastRows];     // Hash: first slot of each row's table
  int32_t rcap[kFastRows];      // Hash: slots of each row's table
  int32_t soff[kFastRows + 1];  // staged rows: first entry of each row in the staging area
  unsigned long long best[kFastRows];  // packed best (key, column) per row, column-allowed pairs
  unsigned long long wtop[kTopK * (kMaxTPB / 32)];
  uint32_t wtopm[kTopK * (kMaxTPB / 32)];
  unsigned long long top[kTopK];
  uint32_t topm[kTopK];
  unsigned long long red[kMaxTPB / 32];
  unsigned long long mbar;
  int32_t qn;
  int32_t trk[kTrack];          // tracked rows of the group (see kTrack)
  int32_t ntrk;
  uint32_t trk_mask;
  unsigned long long trkbest[kTrack];  // packed (contribution, column) per tracked row
  int32_t tqn;                  // tabu columns queued for the warp-wide evaluation
  int32_t lqn;                  // CSR+Bitset: hits on long rows queued for a warp-wide scan (reuses tq)
  int32_t tq[kTabuQueue];
  int32_t ntop;
  int32_t nb;        // Hash: buckets; BB: directory buckets
  int32_t bshift;    // BB: v >> bshift = directory bucket
  int32_t total;     // entries staged / keys indexed
  uint32_t rescan;   // rows swept again alone
  uint32_t group;    // rows of the current group
  uint32_t done_rows;
  int32_t ngroups;   // groups formed so far (this tile's work units, in order)
  int32_t gsel;      // the current group is this CTA's (its slice of the tile)
  int32_t ok;        // bulk copies completed
};

// ---------------------------------------------------------------- the index
template <int ST>
struct FastIndex {
  const FastLayout L;
  unsigned char* base;
  FastSh& sh;
  __device__ FastIndex(const FastLayout& l, unsigned char* b, FastSh& s) : L(l), base(b), sh(s) {}
  __device__ int32_t* keys() const { return reinterpret_cast<int32_t*>(base + L.keys); }
  __device__ int2* recs() const { return reinterpret_cast<int2*>(base + L.recs); }
  __device__ int32_t* queue() const { return reinterpret_cast<int32_t*>(base + L.queue); }
  __device__ int2* stage() const { return reinterpret_cast<int2*>(base + L.stage); }
  __device__ uint16_t* dir() const { return reinterpret_cast<uint16_t*>(base + L.dir); }
  __device__ uint32_t* uni() const { return reinterpret_cast<uint32_t*>(base + L.uni); }
  __device__ uint16_t* rank() const { return reinterpret_cast<uint16_t*>(base + L.rank); }
  __device__ uint32_t* masks() const { return reinterpret_cast<uint32_t*>(base + L.masks); }

  // Does any row of the group have v as a neighbour?
  __device__ __forceinline__ bool query(int32_t v) const {
    if (ST == S_HASH) {
      const int32_t* k = keys();
      const uint32_t nb = (uint32_t)sh.nb;
      uint32_t b = fast_bucket(v, nb);
      for (uint32_t t = 0; t < nb; t++) {
        const int4 k4 = *reinterpret_cast<const int4*>(k + 4u * b);
        if (k4.x == v || k4.y == v || k4.z == v || k4.w == v) return true;
        if ((k4.x | k4.y | k4.z | k4.w) < 0) return false;  // an empty slot (-1) ends the chain
        b = b + 1 == nb ? 0 : b + 1;
      }
      return false;
    } else if (ST == S_BB) {
      const uint16_t* d = dir();
      const uint32_t b = (uint32_t)v >> sh.bshift;
      int32_t lo = d[b], hi = d[b + 1];
      if (lo == hi) return false;
      const int32_t* k = keys();
      while (lo < hi) {
        const int32_t mid = (lo + hi) >> 1;
        if (k[mid] < v) lo = mid + 1;
        else hi = mid;
      }
      return lo < (int32_t)d[b + 1] && k[lo] == v;
    } else {
      return (uni()[(uint32_t)v >> 5] >> (v & 31)) & 1u;
    }
  }

  // Weight of (row r, v) in row r's staged CSR entries (bitmap hit path):
  // the first entry of v, found by a linear scan (CSR+Bitset,
  // GPU-MDP-CSR-Bitset.cu edge lookup) or a lower_bound (CSR+Bitset+BB).
  __device__ __forceinline__ int32_t staged_weight(int r, int32_t v) const {
    const int32_t o = (int32_t)(sh.rrow[r] & 1);
    const int2* e = stage() + sh.soff[r] + o;
    const int32_t len = sh.rdeg[r];
    if (ST == S_BITSET) {
      // two entries per 16-byte load: the row's slot starts on an even entry
      // (16 bytes), the row itself at entry o of it
      const int4* p = reinterpret_cast<const int4*>(stage() + sh.soff[r]);
      const int32_t end = o + len;
      const int32_t pairs = (end + 1) >> 1;  // 16-byte words holding the row
      int32_t j = 0;
      for (; j + 1 < pairs; j += 2) {  // two words per trip, both loads first
        const int4 q0 = p[j], q1 = p[j + 1];
        if (q0.x == v && 2 * j >= o) return q0.y;
        if (q0.z == v) return q0.w;
        if (q1.x == v) return q1.y;
        if (q1.z == v && 2 * j + 3 < end) return q1.w;
      }
      if (j < pairs) {
        const int4 q = p[j];
        if (q.x == v && 2 * j >= o) return q.y;
        if (q.z == v && 2 * j + 1 < end) return q.w;
      }
      return 0;
    }
    int32_t lo = 0, n = len;
    while (n > 0) {
      const int32_t half = n >> 1;
      if (e[lo + half].x < v) { lo += half + 1; n -= half + 1; }
      else n = half;
    }
    return (lo < len && e[lo].x == v) ? e[lo].y : 0;
  }

  // staged_weight for a whole warp (every lane passes the same r and v):
  // the lanes read 32 of the row's 16-byte words at a time, the first
  // matching entry in row order wins.  For rows of hundreds of entries.
  __device__ __forceinline__ int32_t staged_weight_warp(int r, int32_t v, int lane) const {
    const int32_t o = (int32_t)(sh.rrow[r] & 1);
    const int4* p = reinterpret_cast<const int4*>(stage() + sh.soff[r]);
    const int32_t end = o + sh.rdeg[r];
    const int32_t words = (end + 1) >> 1;
    for (int32_t j0 = 0; j0 < words; j0 += 32) {
      const int32_t j = j0 + lane;
      bool h0 = false, h1 = false;
      int32_t hw = 0;
      if (j < words) {
        const int4 q = p[j];
        h0 = q.x == v && 2 * j >= o;
        h1 = q.z == v && 2 * j + 1 < end;
        hw = h0 ? q.y : q.w;
      }
      const unsigned b = __ballot_sync(0xffffffffu, h0 || h1);
      if (b) return __shfl_sync(0xffffffffu, hw, __ffs(b) - 1);
    }
    return 0;
  }

  // Calls f(r, w) for every row r of the group adjacent to v, with w(u_r, v).
  template <class F>
  __device__ __forceinline__ void for_rows(int32_t v, F&& f) const {
    if (ST == S_HASH) {
      const int32_t* k = keys();
      const int2* rc = recs();
      const uint32_t nb = (uint32_t)sh.nb;
      uint32_t b = fast_bucket(v, nb);
      for (uint32_t t = 0; t < nb; t++) {
        bool empty = false;
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const int32_t kk = k[4u * b + j];
          if (kk == v) { const int2 e = rc[4u * b + j]; f(e.x, e.y); }
          empty |= kk < 0;
        }
        if (empty) return;
        b = b + 1 == nb ? 0 : b + 1;
      }
    } else if (ST == S_BB) {
      const uint16_t* d = dir();
      const uint32_t b = (uint32_t)v >> sh.bshift;
      int32_t lo = d[b], hi = d[b + 1];
      const int32_t end = hi;
      const int32_t* k = keys();
      while (lo < hi) {
        const int32_t mid = (lo + hi) >> 1;
        if (k[mid] < v) lo = mid + 1;
        else hi = mid;
      }
      const int2* rc = recs();
      for (; lo < end && k[lo] == v; lo++) f(rc[lo].x, rc[lo].y);
    } else {
      const uint32_t* U = uni();
      const uint32_t wi = (uint32_t)v >> 5;
      const uint32_t word = U[wi];
      if (!((word >> (v & 31)) & 1u)) return;
      const int32_t rk = rank()[wi] + __popc(word & ((1u << (v & 31)) - 1u));
      uint32_t mk = masks()[rk];
      while (mk) {
        const int r = __ffs(mk) - 1;
        mk &= mk - 1;
        f(r, staged_weight(r, v));
      }
    }
  }

  // w(u_r, v) and whether row r is adjacent to v (one row of the group).
  __device__ __forceinline__ int32_t weight_of(int r, int32_t v, bool& adj) const {
    adj = false;
    int32_t w = 0;
    if (ST == S_BITSET || ST == S_BITSET_BB) {
      if ((mask_of(v) >> r) & 1u) { adj = true; w = staged_weight(r, v); }
      return w;
    }
    for_rows(v, [&](int rr, int32_t ww) {
      if (rr == r) { adj = true; w = ww; }
    });
    return w;
  }

  __device__ __forceinline__ uint32_t mask_of(int32_t v) const {
    if (ST == S_BITSET || ST == S_BITSET_BB) {
      const uint32_t* U = uni();
      const uint32_t wi = (uint32_t)v >> 5;
      const uint32_t word = U[wi];
      if (!((word >> (v & 31)) & 1u)) return 0u;
      return masks()[rank()[wi] + __popc(word & ((1u << (v & 31)) - 1u))];
    }
    uint32_t mk = 0;
    for_rows(v, [&](int r, int32_t) { mk |= 1u << r; });
    return mk;
  }
};

// Block-wide exclusive prefix sum of cnt[0..len) in place (len <= 8192);
// returns the total in every thread.
template <class T>
__device__ int32_t block_exclusive_scan(T* cnt, int32_t len, FastSh& sh) {
  const int tid = threadIdx.x, T_ = blockDim.x;
  const int32_t per = (len + T_ - 1) / T_;
  const int32_t a0 = min(len, tid * per), a1 = min(len, a0 + per);
  int32_t run = 0;
  for (int32_t i = a0; i < a1; i++) run += (int32_t)cnt[i];
  // exclusive scan of the per-thread sums
  const int lane = tid & 31, warp = tid >> 5;
  int32_t incl = run;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  __syncthreads();
  if (lane == 31) sh.red[warp] = (unsigned long long)incl;
  __syncthreads();
  int32_t wbase = 0, total = 0;
  for (int w = 0; w < (int)(T_ >> 5); w++) {
    const int32_t v = (int32_t)sh.red[w];
    if (w < warp) wbase += v;
    total += v;
  }
  int32_t x = wbase + incl - run;
  for (int32_t i = a0; i < a1; i++) {
    const int32_t c = (int32_t)cnt[i];
    cnt[i] = (T)x;
    x += c;
  }
  __syncthreads();
  return total;
}

// Bulk-copies the CSR entries of the group's rows into the staging area (each
// row from an even entry, so every copy starts and ends on 16 bytes) and waits.
template <int ST>
__device__ bool fast_stage_rows(const DevGraph& g, const FastIndex<ST>& ix, FastSh& sh, uint32_t grp,
                                DevState* st) {
  const int tid = threadIdx.x;
  if (tid == 0) {
    int32_t off = 0;
    for (int r = 0; r < kFastRows; r++) {
      sh.soff[r] = off;
      if ((grp >> r) & 1u) {
        const long long a = sh.rrow[r] & ~1LL, b = (sh.rrow[r] + sh.rdeg[r] + 1) & ~1LL;
        off += (int32_t)(b - a);
      }
    }
    sh.soff[kFastRows] = off;
    sh.ok = 1;
    mbar_init(&sh.mbar);
  }
  __syncthreads();
  const uint32_t bytes = 8u * (uint32_t)sh.soff[kFastRows];
  if (bytes == 0) return true;
  if (tid < 32) {
    if (tid == 0) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(&sh.mbar, bytes);
    }
    __syncwarp();
    const int r = tid;
    if ((grp >> r) & 1u) {
      const long long a = sh.rrow[r] & ~1LL, b = (sh.rrow[r] + sh.rdeg[r] + 1) & ~1LL;
      if (b > a) bulk_g2s(ix.stage() + sh.soff[r], g.adj + a, (uint32_t)(8 * (b - a)), &sh.mbar);
    }
  }
  const bool ok = mbar_wait0(&sh.mbar, 2000000000ull);
  if (!ok) {
    // bounded: record the failure, wait once more for the copies in flight
    if (tid == 0) { atomicOr(&st->err, E_BULK_TIMEOUT); st->done = 1; sh.ok = 0; }
    mbar_wait0(&sh.mbar, 2000000000ull);
  }
  __syncthreads();
  return sh.ok != 0;
}

// Builds the group's index.  Returns false if the bulk copies failed.
template <int ST>
__device__ bool fast_build(const DevGraph& g, const FastIndex<ST>& ix, FastSh& sh, uint32_t grp, DevState* st) {
  const int tid = threadIdx.x, T = blockDim.x;
  if (ST == S_HASH) {
    // entries of the group (distinct neighbours <= degree) -> buckets
    if (tid == 0) {
      int32_t e = 0, off = 0;
      for (int r = 0; r < kFastRows; r++) {
        sh.soff[r] = off;  // per-row slot offsets of the flattened table read
        if ((grp >> r) & 1u) {
          e += sh.rdeg[r];
          off += sh.rcap[r];
        }
      }
      sh.soff[kFastRows] = off;
      // every slot the layout reserves: at most 2/3 full, and about 1/3 for a
      // group of average rows, so most absent neighbours end in the home bucket
      sh.nb = ix.L.hslots / 4;
      (void)e;
    }
    __syncthreads();
    int32_t* k = ix.keys();
    int2* rc = ix.recs();
    const int32_t slots = 4 * sh.nb;
    for (int32_t q = tid; q < slots; q += T) k[q] = kHashEmpty;
    __syncthreads();
    const uint32_t nb = (uint32_t)sh.nb;
    const int32_t total = sh.soff[kFastRows];
    // the rows' table slots, kB per thread per round, every load issued first
    constexpr int kB = 4;
    for (int32_t f0 = tid; f0 < total; f0 += T * kB) {
      int32_t key[kB], w[kB], rr[kB];
#pragma unroll
      for (int j = 0; j < kB; j++) {
        const int32_t f = f0 + j * T;
        key[j] = kHashEmpty;
        w[j] = 0;
        rr[j] = 0;
        if (f < total) {
          int32_t lo = 0, hi = kFastRows - 1;  // row r with soff[r] <= f < soff[r+1]
          while (lo < hi) {
            const int32_t mid = (lo + hi + 1) >> 1;
            if (sh.soff[mid] <= f) lo = mid; else hi = mid - 1;
          }
          rr[j] = lo;
          const long long at = sh.rhb[lo] + (f - sh.soff[lo]);
          key[j] = __ldg(g.hkey + at);
          w[j] = __ldg(g.hval + at);
        }
      }
#pragma unroll
      for (int j = 0; j < kB; j++) {
        if (key[j] < 0) continue;
        uint32_t b = fast_bucket(key[j], nb);
        for (uint32_t t = 0; t < nb; t++) {
          bool put = false;
#pragma unroll
          for (int q = 0; q < 4; q++) {
            if (!put && atomicCAS(&k[4u * b + q], kHashEmpty, key[j]) == kHashEmpty) {
              rc[4u * b + q] = make_int2(rr[j], w[j]);
              put = true;
            }
          }
          if (put) break;
          b = b + 1 == nb ? 0 : b + 1;
        }
      }
    }
    __syncthreads();
    return true;
  } else {
    if (!fast_stage_rows<ST>(g, ix, sh, grp, st)) return false;
    const int2* sg = ix.stage();
    const int32_t total = sh.soff[kFastRows];
    auto row_of = [&](int32_t f) {
      int32_t lo = 0, hi = kFastRows - 1;
      while (lo < hi) {
        const int32_t mid = (lo + hi + 1) >> 1;
        if (sh.soff[mid] <= f) lo = mid; else hi = mid - 1;
      }
      return lo;
    };
    if (ST == S_BB) {
      // Directory over id ranges, ~2 buckets per entry so most absent
      // neighbours meet an empty bucket.  D[0] = 0 and, once built,
      // D[b + 1] = end of bucket b: bucket b holds records [D[b], D[b+1]).
      if (tid == 0) {
        int32_t e = 0;
        for (int r = 0; r < kFastRows; r++)
          if ((grp >> r) & 1u) e += sh.rdeg[r];
        int32_t lg_nb = 4;
        while ((1 << lg_nb) < 2 * e && (1 << lg_nb) < ix.L.dirmax) lg_nb++;
        int32_t lg_n = 0;
        while ((1LL << lg_n) < (long long)g.n) lg_n++;
        sh.nb = 1 << lg_nb;
        sh.bshift = lg_n > lg_nb ? lg_n - lg_nb : 0;
      }
      __syncthreads();
      uint16_t* D = ix.dir();
      uint32_t* D32 = reinterpret_cast<uint32_t*>(D);
      const int32_t nbk = sh.nb, bsh = sh.bshift;
      for (int32_t q = tid; q < (nbk + 3) / 2; q += T) D32[q] = 0u;  // D[0 .. nbk+1]
      __syncthreads();
      // 16-bit counters updated with 32-bit atomics (a count never exceeds
      // the index capacity, so no carry crosses into the neighbour half)
      auto add16 = [&](int32_t i) -> int32_t {
        const uint32_t old = atomicAdd(D32 + (i >> 1), (i & 1) ? 0x10000u : 1u);
        return (int32_t)((old >> ((i & 1) * 16)) & 0xffffu);
      };
      // first entry of every (row, neighbour), counted per bucket
      for (int32_t f = tid; f < total; f += T) {
        const int r = row_of(f);
        const int32_t e = f - sh.soff[r] - (int32_t)(sh.rrow[r] & 1);
        if (e < 0 || e >= sh.rdeg[r]) continue;
        const int32_t v = sg[f].x;
        if (e > 0 && sg[f - 1].x == v) continue;
        add16(1 + (int32_t)((uint32_t)v >> bsh));
      }
      __syncthreads();
      block_exclusive_scan<uint16_t>(D + 1, nbk, sh);  // D[1 + b] = start of bucket b
      int32_t* k = ix.keys();
      int2* rc = ix.recs();
      for (int32_t f = tid; f < total; f += T) {
        const int r = row_of(f);
        const int32_t e = f - sh.soff[r] - (int32_t)(sh.rrow[r] & 1);
        if (e < 0 || e >= sh.rdeg[r]) continue;
        const int2 x = sg[f];
        if (e > 0 && sg[f - 1].x == x.x) continue;
        const int32_t at = add16(1 + (int32_t)((uint32_t)x.x >> bsh));
        k[at] = x.x;
        rc[at] = make_int2(r, x.y);
      }
      __syncthreads();
      // sort each bucket by neighbour id (a few entries each)
      for (int32_t b = tid; b < nbk; b += T) {
        const int32_t lo = D[b], hi = D[b + 1];
        for (int32_t i = lo + 1; i < hi; i++) {
          const int32_t kv = k[i];
          const int2 rv = rc[i];
          int32_t j = i - 1;
          while (j >= lo && k[j] > kv) { k[j + 1] = k[j]; rc[j + 1] = rc[j]; j--; }
          k[j + 1] = kv;
          rc[j + 1] = rv;
        }
      }
      __syncthreads();
      return true;
    }
    // Bitmap structures: union of the rows' bitmap rows, rank directory,
    // per-vertex row masks from the staged CSR entries.
    uint32_t* U = ix.uni();
    const int32_t uw = (int32_t)(2 * g.wpr);
    for (int32_t q = tid; q < (int32_t)(g.wpr / 2); q += T) {
      uint4 acc = make_uint4(0u, 0u, 0u, 0u);
      uint32_t gm = grp;
      while (gm) {  // eight rows per round, their loads in flight together
        uint4 x[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
          x[j] = make_uint4(0u, 0u, 0u, 0u);
          if (gm) {
            const int r = __ffs(gm) - 1;
            gm &= gm - 1;
            x[j] = __ldg(reinterpret_cast<const uint4*>(g.bits + (long long)sh.ru[r] * g.wpr) + q);
          }
        }
#pragma unroll
        for (int j = 0; j < 8; j++) { acc.x |= x[j].x; acc.y |= x[j].y; acc.z |= x[j].z; acc.w |= x[j].w; }
      }
      reinterpret_cast<uint4*>(U)[q] = acc;
    }
    __syncthreads();
    uint16_t* RK = ix.rank();
    for (int32_t q = tid; q < uw; q += T) RK[q] = (uint16_t)__popc(U[q]);
    __syncthreads();
    const int32_t keys_n = block_exclusive_scan<uint16_t>(RK, uw, sh);
    uint32_t* MK = ix.masks();
    for (int32_t q = tid; q < keys_n; q += T) MK[q] = 0u;
    __syncthreads();
    for (int32_t f = tid; f < total; f += T) {
      const int r = row_of(f);
      const int32_t e = f - sh.soff[r] - (int32_t)(sh.rrow[r] & 1);
      if (e < 0 || e >= sh.rdeg[r]) continue;
      const int32_t v = sg[f].x;
      const uint32_t wi = (uint32_t)v >> 5, word = U[wi];
      if (!((word >> (v & 31)) & 1u)) continue;  // cannot happen: the bitmap holds every entry
      atomicOr(MK + RK[wi] + __popc(word & ((1u << (v & 31)) - 1u)), 1u << r);
    }
    __syncthreads();
    return true;
  }
}

// Exact-by-column best of one row over the tile's columns, every pair
// evaluated with w from `wfn(c, v)`: the row's record is merged into
// sh.best[r].  Used for rows adjacent to every top column (rescan) and for
// rows too large for the index (heavy rows, wfn = a global lookup).
template <int PROB, bool PERSIST, class WFn>
__device__ void fast_row_sweep(const DevSolver<int32_t>& s, FastSh& sh, int r, int32_t c0, int32_t c_end,
                               long long iter, int32_t D, bool skip_tabu_cols, WFn&& wfn) {
  const int tid = threadIdx.x, T = blockDim.x;
  const int32_t rv = sh.rv[r];
  unsigned long long mine = 0;
  for (int32_t c = c0 + tid; c < c_end; c += T) {
    const bool ct = ld_st<PERSIST>(s.tab_out + c) > iter;
    if (ct && skip_tabu_cols) continue;
    const int32_t v = ld_st<PERSIST>(s.sol_out + c);
    int32_t w = 0;
    if (!wfn(c, v, w)) continue;  // pair handled elsewhere
    const int32_t x = pair_gain<PROB, int32_t>(rv, ld_st<PERSIST>(s.vg_out + c), w);
    if (ct && !(x > D)) continue;
    const unsigned long long p = pack_kc(x, c);
    mine = p > mine ? p : mine;
  }
  mine = warp_max_u64(mine);
  if ((tid & 31) == 0 && mine) atomicMax(&sh.best[r], mine);
}

// The fast pass of one tile (32-bit keys, mode 0).  (out_key, out_idx) valid
// in thread 0; (LLONG_MIN, LLONG_MAX) when the tile has no allowed pair.
// Work units of a tile: its groups, then its heavy rows, in order.  With
// nslices > 1 several CTAs share the tile: slice k takes the units whose
// index is k mod nslices (every slice forms the same groups from the rows'
// degrees), so a tile whose rows hold far more entries than one index is
// spread over CTAs instead of running its units one after another.
template <int PROB, int ST, bool PERSIST>
__device__ void tile_fast(const DevGraph& g, const DevSolver<int32_t>& s, long long iter, long long D64, int rb,
                          int ch, long long& out_key, long long& out_idx, int slice = 0, int nslices = 1) {
  __shared__ FastSh sh;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int tid = threadIdx.x, T = blockDim.x, lane = tid & 31, warp = tid >> 5;
  const int32_t D = KeyLim<int32_t>::clampD(D64);
  const int32_t r0 = rb * kFastRows;
  const int32_t nr = min(kFastRows, s.m - r0);
  const int32_t c0 = ch * s.chunk_cols;
  const int32_t c_end = min(c0 + s.chunk_cols, s.delta);
  const FastLayout L = fast_layout(ST, s.fast_ecap, g.wpr);
  const FastIndex<ST> ix(L, smem_raw, sh);

  if (tid < kFastRows) {
    const bool ok = tid < nr;
    const int32_t u = ok ? ld_st<PERSIST>(s.sol_in + r0 + tid) : 0;
    sh.ru[tid] = u;
    sh.rv[tid] = ok ? ld_st<PERSIST>(s.vg_in + r0 + tid) : 0;
    sh.rtab[tid] = ok ? (ld_st<PERSIST>(s.tab_in + r0 + tid) > iter) : 0;
    const long long a = ok ? g.rowptr[u] : 0;
    const long long a1 = ok ? g.rowptr[u + 1] : 0;
    long long hb = 0, hb1 = 0;
    if (ST == S_HASH && ok) { hb = g.hoff[u]; hb1 = g.hoff[u + 1]; }
    sh.rrow[tid] = a;
    sh.rdeg[tid] = (int32_t)(a1 - a);
    sh.rhb[tid] = hb;
    sh.rcap[tid] = (int32_t)(hb1 - hb);
    sh.best[tid] = 0ull;
  }
  if (tid == 0) { sh.done_rows = 0u; sh.ngroups = 0; }
  __syncthreads();

  const uint32_t all_rows = nr >= 32 ? 0xffffffffu : ((1u << nr) - 1u);
  const bool masked_csr = ST == S_CSR && (PROB == P_MDP || s.adj_mask != 0);

  // ---------------- rows per group: the index holds at most ecap entries
  for (;;) {
    if (tid == 0) {
      uint32_t grp = 0;
      if (ST == S_CSR) {
        grp = all_rows & ~sh.done_rows;
      } else {
        int32_t e = 0;
        for (int r = 0; r < nr; r++) {
          if ((sh.done_rows >> r) & 1u) continue;
          const int32_t d = sh.rdeg[r];
          if (d > s.fast_ecap) continue;  // heavy row: swept alone below
          if (e + d > s.fast_ecap) break;
          e += d;
          grp |= 1u << r;
        }
      }
      sh.group = grp;
      sh.done_rows |= grp;
      sh.gsel = grp != 0u && sh.ngroups % nslices == slice;
      if (grp != 0u) sh.ngroups++;
      sh.qn = 0;
      sh.tqn = 0;
      sh.lqn = 0;
      // Hub rows are adjacent to every top column (hubs are adjacent to each
      // other), so the shared top-2 rarely serves them: the sweep tracks the
      // best free column of up to kTrack of the group's highest-degree rows.
      // (CSR without the adjacency mask needs none: its w-free gains only
      // under-estimate adjacent pairs.)
      int32_t nt = 0;
      uint32_t tm = 0u;
      if (sh.gsel && (ST != S_CSR || masked_csr)) {
        for (int t = 0; t < kTrack; t++) {
          int best_r = -1;
          for (int r = 0; r < nr; r++)
            if (((grp >> r) & 1u) && !((tm >> r) & 1u) && sh.rdeg[r] >= kTrackDeg &&
                (best_r < 0 || sh.rdeg[r] > sh.rdeg[best_r]))
              best_r = r;
          if (best_r < 0) break;
          tm |= 1u << best_r;
          sh.trk[nt] = best_r;
          sh.trkbest[nt] = 0ull;
          nt++;
        }
      }
      sh.ntrk = nt;
      sh.trk_mask = tm;
      sh.rescan = 0u;
    }
    __syncthreads();
    const uint32_t grp = sh.group;
    if (grp == 0u) break;
    if (!sh.gsel) {  // another slice's group
      __syncthreads();
      continue;
    }

    // ---------------- index of the group
    uint32_t* s_mask = reinterpret_cast<uint32_t*>(smem_raw);  // CSR: rows adjacent to each column
    if (ST == S_CSR) {
      if (masked_csr)
        for (int32_t c = tid; c < s.chunk_cols; c += T) s_mask[c] = 0u;
      if (tid < 32) {
        int32_t d = tid < nr ? sh.rdeg[tid] : 0;
        int32_t incl = d;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += t;
        }
        sh.soff[tid + 1] = incl;
        if (tid == 0) sh.soff[0] = 0;
      }
      __syncthreads();
      // join: entries of the rows whose neighbour sits in this chunk, exact.
      // Four entries per thread per round (loads first); the lanes of a warp
      // mostly hold entries of one row, so their maxima are combined in the
      // warp before one atomic per row.
      const int32_t total = sh.soff[nr];
      constexpr int kJ = 4;
      for (int32_t f0 = tid - lane; f0 < total; f0 += T * kJ) {  // uniform per warp
        int rj[kJ];
        long long kj[kJ];
        int32_t cj[kJ];
        int2 ej[kJ];
        bool dj[kJ];
#pragma unroll
        for (int j = 0; j < kJ; j++) {  // first loads: cpos and the entries
          const int32_t f = f0 + j * T + lane;
          rj[j] = -1;
          kj[j] = 0;
          cj[j] = -1;
          ej[j] = make_int2(0, 0);
          dj[j] = true;
          if (f < total) {
            int32_t lo = 0, hi = nr - 1;
            while (lo < hi) {
              const int32_t mid = (lo + hi + 1) >> 1;
              if (sh.soff[mid] <= f) lo = mid; else hi = mid - 1;
            }
            rj[j] = lo;
            kj[j] = sh.rrow[lo] + (f - sh.soff[lo]);
            cj[j] = ld_st<PERSIST>(s.cpos + kj[j]) - s.m;
            ej[j] = g.adj[kj[j]];
            dj[j] = kj[j] > sh.rrow[lo] && g.adj[kj[j] - 1].x == ej[j].x;  // first entry wins
          }
        }
        int32_t cvj[kJ], ctj[kJ];
#pragma unroll
        for (int j = 0; j < kJ; j++) {  // second loads: the columns' state
          const bool in = rj[j] >= 0 && !dj[j] && cj[j] >= c0 && cj[j] < c_end;
          if (!in) rj[j] = -1;
          cvj[j] = in ? ld_st<PERSIST>(s.vg_out + cj[j]) : 0;
          ctj[j] = in ? ld_st<PERSIST>(s.tab_out + cj[j]) : 0;
        }
#pragma unroll
        for (int j = 0; j < kJ; j++) {
          unsigned long long p = 0ull;
          const int r = rj[j];
          if (r >= 0) {
            if (masked_csr) atomicOr(&s_mask[cj[j] - c0], 1u << r);
            const int32_t x = pair_gain<PROB, int32_t>(sh.rv[r], cvj[j], ej[j].y);
            if (!(ctj[j] > iter) || x > D) p = pack_kc(x, cj[j]);
          }
          // per distinct row of the warp: its lanes' maximum, one atomic
          unsigned todo = __ballot_sync(0xffffffffu, p != 0ull);
          while (todo) {
            const int leader = __ffs(todo) - 1;
            const int rr = __shfl_sync(0xffffffffu, r, leader);
            const bool mine = r == rr && p != 0ull;
            const unsigned long long mx = warp_max_u64(mine ? p : 0ull);
            if (lane == leader) atomicMax(&sh.best[rr], mx);
            todo &= ~__ballot_sync(0xffffffffu, mine);
          }
        }
      }
      __syncthreads();
    } else {
      if (!fast_build<ST>(g, ix, sh, grp, s.st)) {
        if (tid == 0) { out_key = LLONG_MIN; out_idx = LLONG_MAX; }
        __syncthreads();
        return;
      }
    }

    // ---------------- sweep: one query per column, per-thread top columns
    int32_t tcv[kTopK], tc[kTopK];
    uint32_t tmk[kTopK];
#pragma unroll
    for (int k = 0; k < kTopK; k++) { tcv[k] = INT32_MIN; tc[k] = INT32_MAX; tmk[k] = 0u; }
    int32_t* Q = ix.queue();
    const int ntrk = sh.ntrk;
    int trk[kTrack];
    unsigned long long hb[kTrack];
#pragma unroll
    for (int h = 0; h < kTrack; h++) { trk[h] = sh.trk[h]; hb[h] = 0ull; }
    // one pass of loads in flight ahead of the pass being evaluated
    const int32_t it32 = iter > (long long)INT32_MAX ? INT32_MAX : (int32_t)iter;  // tabu stamps are int32
    int32_t cb = c0 + tid * kColsPerLane;
    int32_t cv[4] = {0, 0, 0, 0}, ct4[4] = {0, 0, 0, 0}, vx[4] = {0, 0, 0, 0};
    if (cb < c_end) {
      load4<PERSIST>(s.vg_out + cb, cv);
      load4<PERSIST>(s.tab_out + cb, ct4);
      if (ST != S_CSR) load4<PERSIST>(s.sol_out + cb, vx);
    }
    for (; cb < c_end; cb += T * kColsPerLane) {
      const int32_t nb_ = cb + T * kColsPerLane;
      int32_t ncv[4], nct[4], nvx[4];
      if (nb_ < c_end) {
        load4<PERSIST>(s.vg_out + nb_, ncv);
        load4<PERSIST>(s.tab_out + nb_, nct);
        if (ST != S_CSR) load4<PERSIST>(s.sol_out + nb_, nvx);
      }
      // the four columns at once: validity, tabu, adjacency, best contribution
      bool ok[4], tb[4], adj[4];
      int32_t m4 = INT32_MIN;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        ok[q] = cb + q < c_end;
        tb[q] = ok[q] && ct4[q] > it32;
        adj[q] = (ST != S_CSR) && ok[q] && ix.query(vx[q]);
        if (ok[q] && !tb[q]) m4 = cv[q] > m4 ? cv[q] : m4;
      }
      if (tb[0] | tb[1] | tb[2] | tb[3]) {
        // tabu columns: evaluated after the sweep by a warp, one lane per row
#pragma unroll
        for (int q = 0; q < 4; q++)
          if (tb[q]) {
            const int32_t at = atomicAdd(&sh.tqn, 1);
            if (at < kTabuQueue) {
              sh.tq[at] = cb + q;
            } else {  // queue full (very long tenures): this lane evaluates every row
              const int32_t c = cb + q;
              uint32_t rowsleft = grp;
              while (rowsleft) {
                const int r = __ffs(rowsleft) - 1;
                rowsleft &= rowsleft - 1;
                bool a = false;
                int32_t w = 0;
                if (ST == S_CSR) a = masked_csr && ((s_mask[c - c0] >> r) & 1u);
                else w = ix.weight_of(r, vx[q], a);
                if (ST == S_CSR && a) continue;  // the join evaluated the adjacent pairs
                const int32_t x = pair_gain<PROB, int32_t>(sh.rv[r], cv[q], w);
                if (x > D) atomicMax(&sh.best[r], pack_kc(x, c));
              }
            }
          }
      }
      if (ST != S_CSR) {
#pragma unroll
        for (int q = 0; q < 4; q++)
          if (adj[q] && !tb[q]) Q[atomicAdd(&sh.qn, 1)] = cb + q;
      }
      if (ntrk) {
#pragma unroll
        for (int q = 0; q < 4; q++) {
          if (!ok[q] || tb[q]) continue;
          uint32_t mkq = 0u;
          if (ST == S_CSR) mkq = s_mask[cb + q - c0];
          else if (adj[q]) mkq = ix.mask_of(vx[q]);
          const unsigned long long p = pack_kc(cv[q], cb + q);
#pragma unroll
          for (int h = 0; h < kTrack; h++)
            if (h < ntrk && !((mkq >> trk[h]) & 1u)) hb[h] = p > hb[h] ? p : hb[h];
        }
      }
      if (m4 > tcv[1]) {
#pragma unroll
        for (int q = 0; q < 4; q++) {
          if (!ok[q] || tb[q] || !(cv[q] > tcv[1])) continue;
          uint32_t mk = 0u;
          if (ST == S_CSR) mk = masked_csr ? s_mask[cb + q - c0] : 0u;
          else if (adj[q]) mk = ix.mask_of(vx[q]);
          // insert keeping (contribution desc, column asc): this thread's
          // columns come in ascending order, so an equal one stays behind
          if (cv[q] > tcv[0]) {
            tcv[1] = tcv[0]; tc[1] = tc[0]; tmk[1] = tmk[0];
            tcv[0] = cv[q]; tc[0] = cb + q; tmk[0] = mk;
          } else {
            tcv[1] = cv[q]; tc[1] = cb + q; tmk[1] = mk;
          }
        }
      }
#pragma unroll
      for (int q = 0; q < 4; q++) { cv[q] = ncv[q]; ct4[q] = nct[q]; vx[q] = nvx[q]; }
    }
    __syncthreads();

    // ---------------- tabu columns: one warp per column, one lane per row
    {
      const int32_t tqn = min(sh.tqn, kTabuQueue);
      const int r = lane;
      const bool in_grp = (grp >> r) & 1u;
      for (int32_t i = warp; i < tqn; i += (T >> 5)) {
        const int32_t c = sh.tq[i];
        const int32_t v = ld_st<PERSIST>(s.sol_out + c);
        const int32_t cvv = ld_st<PERSIST>(s.vg_out + c);
        if (!in_grp) continue;
        bool a = false;
        int32_t w = 0;
        if (ST == S_CSR) a = masked_csr && ((s_mask[c - c0] >> r) & 1u);
        else w = ix.weight_of(r, v, a);
        if (ST == S_CSR && a) continue;  // the join evaluated the adjacent pairs
        const int32_t x = pair_gain<PROB, int32_t>(sh.rv[r], cvv, w);
        if (x > D) atomicMax(&sh.best[r], pack_kc(x, c));
      }
    }

    // ---------------- tracked rows: their best free column, block-wide
    for (int h = 0; h < ntrk; h++) {
      const unsigned long long m = warp_max_u64(hb[h]);
      if (lane == 0 && m) atomicMax(&sh.trkbest[h], m);
    }

    // ---------------- exact pairs of the adjacent columns
    // (CSR+Bitset: a hit on a row of more than kLongScan entries is queued
    // and scanned by a whole warp afterwards, so one thread's hub-row scans
    // do not hold the CTA at its next barrier; the queue reuses the tabu
    // queue's memory, free once the tabu columns are done)
    if (ST != S_CSR) {
      constexpr int32_t kLongScan = 256;
      if (ST == S_BITSET) __syncthreads();
      const int32_t qn = sh.qn;
      for (int32_t i = tid; i < qn; i += T) {
        const int32_t c = Q[i];
        const int32_t v = ld_st<PERSIST>(s.sol_out + c);
        const int32_t cvv = ld_st<PERSIST>(s.vg_out + c);
        if constexpr (ST == S_BITSET) {
          uint32_t mk = ix.mask_of(v);
          while (mk) {
            const int r = __ffs(mk) - 1;
            mk &= mk - 1;
            if (sh.rdeg[r] > kLongScan) {
              const int32_t at = atomicAdd(&sh.lqn, 1);
              if (at < kTabuQueue) {
                sh.tq[at] = (c << 5) | r;  // c < n: a bitmap that fits in HBM keeps n far below 2^26
                continue;
              }
            }
            atomicMax(&sh.best[r], pack_kc(pair_gain<PROB, int32_t>(sh.rv[r], cvv, ix.staged_weight(r, v)), c));
          }
        } else {
          ix.for_rows(v, [&](int r, int32_t w) {
            atomicMax(&sh.best[r], pack_kc(pair_gain<PROB, int32_t>(sh.rv[r], cvv, w), c));
          });
        }
      }
      if (ST == S_BITSET) {
        __syncthreads();
        const int32_t lqn = min(sh.lqn, kTabuQueue);
        for (int32_t i = warp; i < lqn; i += (T >> 5)) {
          const int32_t it = sh.tq[i];
          const int32_t c = it >> 5;
          const int r = it & 31;
          const int32_t v = ld_st<PERSIST>(s.sol_out + c);
          const int32_t cvv = ld_st<PERSIST>(s.vg_out + c);
          const int32_t w = ix.staged_weight_warp(r, v, lane);
          if (lane == 0) atomicMax(&sh.best[r], pack_kc(pair_gain<PROB, int32_t>(sh.rv[r], cvv, w), c));
        }
      }
    }

    // ---------------- tile top columns: warp top-K, then block top-K
#pragma unroll
    for (int k = 0; k < kTopK; k++) {
      unsigned long long head = tcv[0] == INT32_MIN ? 0ull : pack_kc(tcv[0], tc[0]);
      const unsigned long long wb = warp_max_u64(head);
      const bool mine = wb != 0ull && head == wb;
      const unsigned bal = __ballot_sync(0xffffffffu, mine);
      const uint32_t wm = __shfl_sync(0xffffffffu, tmk[0], bal ? __ffs(bal) - 1 : 0);
      if (lane == 0) { sh.wtop[warp * kTopK + k] = wb; sh.wtopm[warp * kTopK + k] = wb ? wm : 0u; }
      if (mine) {
#pragma unroll
        for (int j = 0; j < kTopK - 1; j++) { tcv[j] = tcv[j + 1]; tc[j] = tc[j + 1]; tmk[j] = tmk[j + 1]; }
        tcv[kTopK - 1] = INT32_MIN; tc[kTopK - 1] = INT32_MAX; tmk[kTopK - 1] = 0u;
      }
    }
    __syncthreads();
    if (warp == 0) {
      const int nw = T >> 5;
      unsigned long long cand = lane < nw * kTopK ? sh.wtop[lane] : 0ull;
      uint32_t cm = lane < nw * kTopK ? sh.wtopm[lane] : 0u;
      int cnt = 0;
#pragma unroll
      for (int k = 0; k < kTopK; k++) {
        const unsigned long long b = warp_max_u64(cand);
        const bool mine = b != 0ull && cand == b;
        const unsigned bal = __ballot_sync(0xffffffffu, mine);
        const uint32_t m = __shfl_sync(0xffffffffu, cm, bal ? __ffs(bal) - 1 : 0);
        if (lane == 0) { sh.top[k] = b; sh.topm[k] = b ? m : 0u; }
        cnt += b != 0ull;
        if (mine) cand = 0ull;
      }
      if (lane == 0) sh.ntop = cnt;
    }
    __syncthreads();
    // each row: its first top column it is not adjacent to (w-free gain);
    // a tracked row has its own best free column
    if (tid < sh.ntrk && sh.trkbest[tid]) {
      const int r = sh.trk[tid];
      const unsigned long long p = sh.trkbest[tid];
      const int32_t x = pair_gain<PROB, int32_t>(sh.rv[r], unpack_key(p), 0);
      atomicMax(&sh.best[r], pack_kc(x, unpack_col(p)));
    }
    if (tid < kFastRows && ((grp >> tid) & 1u) && !((sh.trk_mask >> tid) & 1u)) {
      const int r = tid;
      bool found = false;
      for (int k = 0; k < sh.ntop && !found; k++) {
        if ((sh.topm[k] >> r) & 1u) continue;
        const unsigned long long p = sh.top[k];
        const int32_t x = pair_gain<PROB, int32_t>(sh.rv[r], unpack_key(p), 0);
        atomicMax(&sh.best[r], pack_kc(x, unpack_col(p)));
        found = true;
      }
      if (!found && sh.ntop == kTopK) atomicOr(&sh.rescan, 1u << r);
    }
    __syncthreads();
    // rows adjacent to every top column (typically hubs, adjacent to every
    // other hub): their non-adjacent, non-tabu columns, up to eight rows per
    // extra pass over the chunk, each row's maximum in registers
    uint32_t rs = sh.rescan;
    while (rs) {
      int rr[8];
      int32_t rvv[8];
      uint32_t valid = 0u;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        rr[j] = 0;
        rvv[j] = 0;
        if (rs) {
          rr[j] = __ffs(rs) - 1;
          rs &= rs - 1;
          rvv[j] = sh.rv[rr[j]];
          valid |= 1u << j;
        }
      }
      unsigned long long acc[8];
#pragma unroll
      for (int j = 0; j < 8; j++) acc[j] = 0ull;
      for (int32_t c = c0 + tid; c < c_end; c += T) {
        if (ld_st<PERSIST>(s.tab_out + c) > iter) continue;  // tabu columns were evaluated in the sweep
        uint32_t mk;
        if (ST == S_CSR) mk = masked_csr ? s_mask[c - c0] : 0u;
        else mk = ix.mask_of(ld_st<PERSIST>(s.sol_out + c));
        const int32_t cvv = ld_st<PERSIST>(s.vg_out + c);
#pragma unroll
        for (int j = 0; j < 8; j++) {
          if (((valid >> j) & 1u) && !((mk >> rr[j]) & 1u)) {
            const unsigned long long p = pack_kc(pair_gain<PROB, int32_t>(rvv[j], cvv, 0), c);
            acc[j] = p > acc[j] ? p : acc[j];
          }
        }
      }
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const unsigned long long m = warp_max_u64(acc[j]);
        if (lane == 0 && m && ((valid >> j) & 1u)) atomicMax(&sh.best[rr[j]], m);
      }
    }
    __syncthreads();
  }

  // ---------------- heavy rows (more entries than the index holds): the row's
  // entries of its own structure (Hash: table slots; the others: CSR entries,
  // first of a duplicated pair) placed by the current position of each
  // neighbour, evaluated exactly and marked in a bitmap of the chunk's
  // columns; every unmarked column then gets the w-free gain.
  if (ST != S_CSR) {
    uint32_t hv = all_rows & ~sh.done_rows;
    uint32_t* cbits = reinterpret_cast<uint32_t*>(smem_raw);  // the index is no longer needed
    const int32_t cw = (c_end - c0 + 31) >> 5;
    int32_t unit = sh.ngroups;  // heavy rows follow the groups in the unit order
    while (hv) {
      const int r = __ffs(hv) - 1;
      hv &= hv - 1;
      if (unit++ % nslices != slice) continue;  // another slice's row
      const int32_t u = sh.ru[r], rv = sh.rv[r];
      for (int32_t q = tid; q < cw; q += T) cbits[q] = 0u;
      __syncthreads();
      unsigned long long hmax = 0ull;  // this thread's best exact pair of the row
      auto place = [&](int32_t z, int32_t w) {
        const int32_t c = ld_st<PERSIST>(s.pos + z) - s.m;
        if (c < c0 || c >= c_end) return;
        atomicOr(&cbits[(c - c0) >> 5], 1u << ((c - c0) & 31));
        const int32_t x = pair_gain<PROB, int32_t>(rv, ld_st<PERSIST>(s.vg_out + c), w);
        if (!(ld_st<PERSIST>(s.tab_out + c) > iter) || x > D) {
          const unsigned long long p = pack_kc(x, c);
          hmax = p > hmax ? p : hmax;
        }
      };
      if (ST == S_HASH) {
        const long long hb = g.hoff[u], cap = g.hoff[u + 1] - hb;
        for (long long q = tid; q < cap; q += T) {
          const int32_t z = __ldg(g.hkey + hb + q);
          if (z >= 0) place(z, __ldg(g.hval + hb + q));
        }
      } else {
        const long long a = sh.rrow[r];
        for (long long k = a + tid; k < a + sh.rdeg[r]; k += T) {
          const int2 e = g.adj[k];
          if (k > a && g.adj[k - 1].x == e.x) continue;
          place(e.x, e.y);
        }
      }
      hmax = warp_max_u64(hmax);
      if (lane == 0 && hmax) atomicMax(&sh.best[r], hmax);
      __syncthreads();
      fast_row_sweep<PROB, PERSIST>(s, sh, r, c0, c_end, iter, D, false, [&](int32_t c, int32_t, int32_t& w) {
        w = 0;
        return !((cbits[(c - c0) >> 5] >> ((c - c0) & 31)) & 1u);
      });
      __syncthreads();
    }
  }
  __syncthreads();

  // ---------------- the tile's record: rows in order (lowest flat index on ties)
  if (tid == 0) {
    long long bk = LLONG_MIN, bi = LLONG_MAX;
    for (int r = 0; r < nr; r++) {
      const unsigned long long p = sh.best[r];
      if (!p) continue;
      const int32_t x = unpack_key(p);
      if (sh.rtab[r] && !(x > D)) continue;  // tabu row: only aspirated pairs
      if ((long long)x > bk) { bk = x; bi = (long long)(r0 + r) * s.delta + unpack_col(p); }
    }
    out_key = bk;
    out_idx = bi;
  }
  __syncthreads();
}

}  // namespace tsb
