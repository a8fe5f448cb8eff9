// batch.cu -- the batched form: many independent solves in one persistent launch.
//
// The reference runs one tabu search at a time, and every iteration costs 4-5
// launches plus a blocking copy (src/mdp/GPU-MDP-CSR.cu:644-681); its memetic
// drivers call that loop again and again for restarts and offspring (OBMA
// :754-903,1146-1208; MACUT src/maxbisection/GPU-MAXBS-CSR.cu:523-577,679-732).
//
// Here solves are grouped by (problem, structure, key width, CTAs per solve)
// and each group is ONE persistent launch.  A thread-block cluster of 1-8 CTAs
// owns one slot of solver memory in HBM: it pulls a solve from the group's job
// list (atomic ticket), its leader CTA builds the start state, then every
// iteration the cluster's CTAs evaluate the tiles of the pair space round-robin
// (tile_eval, the plain kernel's code), meet at a cluster barrier, the leader
// merges their records through distributed shared memory and decides/applies
// the move (decide_apply, also the plain kernel's code) and the cluster meets
// again.  No grid-wide wait exists anywhere: clusters never wait on each other,
// and the hardware co-schedules the CTAs of a cluster.  After the last
// iteration the leader rebuilds the best solution from the move log, computes
// its objective from the graph, writes the result and pulls the next solve.
// The group launches are captured once as a CUDA graph (one branch per group
// on its own stream) and replayed.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <memory>
#include <random>
#include <thread>
#include <vector>

#include "packed.cuh"
#include "ts_host.h"

namespace cg = cooperative_groups;

namespace tsb {
namespace {

struct BatchJobDev {
  DevGraph g;
  int32_t n, m;
  long long max_iter;
  int32_t tenure_policy, tenure, maxt, piter, num_pert, c2_fixed;
  int32_t n_row_blocks, n_chunks, chunk_cols, stage_bytes;
  int32_t orig;             // index in the caller's job array
  int32_t adj_mask;         // CSR: adjacent pairs masked out of the w-free sweep
  int32_t tile_rows, fast, fast_ecap;  // tile shape (tile_geometry)
  const int32_t* init;      // MDP: m ids; MaxBS: part[n]
  const long long* draws;   // MaxBS perturbation events x num_pert
  long long draw_events;
  long long sol_off;        // offset of this job's packed best solution
};


// Solver memory of a group: array-major, one slice per slot, each slice sized
// for the largest job of the group (strides in elements of each array).
template <class KeyT>
struct SlotPool {
  int32_t *sol_in, *sol_out, *tab_in, *tab_out, *pos, *cpos, *W;
  KeyT *vg_in, *vg_out;
  DevState* st;
  int2* movelog;
  long long s_m, s_ldc, s_n, s_entries, s_w, s_vgm, s_vgldc, log_cap;
};

template <class KeyT>
__device__ DevSolver<KeyT> slot_solver(const BatchJobDev& J, const SlotPool<KeyT>& P, long long slot,
                                       int problem) {
  DevSolver<KeyT> s;
  s.n = J.n; s.m = J.m; s.delta = J.n - J.m; s.ldc = (s.delta + 3) & ~3;
  s.problem = problem;
  s.tenure_policy = J.tenure_policy; s.tenure = J.tenure; s.maxt = J.maxt; s.piter = J.piter;
  s.num_pert = J.num_pert;
  s.c2_tab[0] = 11; s.c2_tab[1] = 21; s.c2_tab[2] = 42; s.c2_tab[3] = 84;  // round(0.7*C1), C1 = 15..120
  s.c2_fixed = J.c2_fixed;
  s.n_row_blocks = J.n_row_blocks; s.n_chunks = J.n_chunks; s.chunk_cols = J.chunk_cols;
  s.stage_bytes = J.stage_bytes;
  s.adj_mask = J.adj_mask;
  s.tile_rows = J.tile_rows;
  s.fast = J.fast;
  s.fast_ecap = J.fast_ecap;
  s.w16 = 0;  // slot pools hold 32-bit matrices
  s.P = (long long)s.m * s.delta;
  s.sol_in = P.sol_in + slot * P.s_m;
  s.sol_out = P.sol_out + slot * P.s_ldc;
  s.vg_in = P.vg_in + slot * P.s_vgm;
  s.vg_out = P.vg_out + slot * P.s_vgldc;
  s.tab_in = P.tab_in + slot * P.s_m;
  s.tab_out = P.tab_out + slot * P.s_ldc;
  s.pos = P.pos + slot * P.s_n;
  s.cpos = P.cpos ? P.cpos + slot * P.s_entries : nullptr;
  s.W = P.W ? P.W + slot * P.s_w : nullptr;
  s.st = P.st + slot;
  s.recs = nullptr;
  s.movelog = P.movelog + slot * P.log_cap;
  s.log_cap = P.log_cap;
  s.trace = nullptr;
  s.trace_cap = 0;
  s.draws = J.draws;
  s.draw_events = J.draw_events;
  return s;
}

template <int PROB, int ST, class KeyT>
__global__ void __launch_bounds__((TpbOf<ST, true>::v))
batch_kernel(const BatchJobDev* __restrict__ jobs, int njobs, BatchResultDev* __restrict__ out,
             int32_t* __restrict__ best_out, const SlotPool<KeyT> pool, unsigned int* next_job) {
  cg::cluster_group cl = cg::this_cluster();
  const unsigned rank = cl.block_rank(), cs = cl.num_blocks();
  const long long slot = blockIdx.x / cs;
  const int tid = threadIdx.x;
  __shared__ TailShared sh;
  __shared__ int s_job;
  __shared__ CtaRec s_rec;
  __shared__ long long sc[kMaxTPB / 32];
  __shared__ int32_t s_cnt[kMaxTPB];
  for (;;) {
    if (rank == 0 && tid == 0) s_job = (int)atomicAdd(next_job, 1u);
    cl.sync();
    const int j = *cl.map_shared_rank(&s_job, 0);
    cl.sync();  // every CTA has read the leader's ticket before it changes or the leader exits
    if (j >= njobs) return;
    const BatchJobDev J = jobs[j];
    const DevSolver<KeyT> s = slot_solver<KeyT>(J, pool, slot, PROB);
    const DevGraph g = J.g;
    if (rank == 0) {
      slot_init<PROB, ST, KeyT>(g, s, J.init, J.max_iter, sc, s_cnt);
      __threadfence();
    }
    cl.sync();
    cluster_iterate<PROB, ST, KeyT>(g, s, J.max_iter, cl, sh, s_rec);
    if (rank == 0) slot_finish<PROB, KeyT>(g, s, out + J.orig, best_out + J.sol_off, sc);
  }
}

struct HostJob {
  int32_t idx;
  const ts_graph* g;
  ts_params p;
  int32_t n, m, num_pert, cluster;
  bool wide;
  int32_t kind;
  long long events;
  double work;
  std::vector<int32_t> init;
  std::vector<long long> draws;
};

// Start and perturbation stream of one solve, exactly as ts_solver_init draws them.
bool prepare_host_job(HostJob& H, const int32_t* initial) {
  const int32_t n = H.n, m = H.m;
  std::mt19937 rng;
  rng.seed(H.p.seed);
  H.events = 0;
  if (H.p.problem == TS_PROBLEM_MDP) {
    if (initial) {
      std::vector<uint8_t> seen(n, 0);
      H.init.assign(initial, initial + m);
      for (int32_t v : H.init) {
        if (v < 0 || v >= n || seen[v]) return false;
        seen[v] = 1;
      }
    } else {
      mdp_random_set(n, m, H.p.seed, H.init);
    }
    return true;
  }
  H.init.assign(n, 1);
  if (initial) {
    int32_t zeros = 0;
    for (int32_t v = 0; v < n; v++) {
      if (initial[v] != 0 && initial[v] != 1) return false;
      H.init[v] = initial[v];
      zeros += initial[v] == 0;
    }
    if (zeros != m) return false;
  } else {
    std::vector<uint8_t> side0;
    maxbs_random_part(rng, n, side0);
    for (int32_t v = 0; v < n; v++) H.init[v] = side0[v] ? 0 : 1;
  }
  // at most max_iter/piter perturbation events fit in max_iter iterations
  const int64_t P = (int64_t)m * (n - m);
  H.events = H.p.max_iter / H.p.piter + 1;
  H.draws.reserve((size_t)(H.events * H.num_pert));
  for (long long e = 0; e < H.events; e++) draw_event(rng, P, H.num_pert, H.draws);
  return true;
}

using Launcher = std::function<cudaError_t(cudaStream_t, const BatchJobDev*, BatchResultDev*, int32_t*,
                                           unsigned int*)>;

struct Group {
  int32_t problem = 0, kind = 0, cluster = 1;
  bool wide = false;
  std::vector<HostJob*> jobs;
  long long job_off = 0;  // first entry in the device job table
  double work = 0;
  long long slots = 0;
  size_t smem = 0;
  std::unique_ptr<DevBuf> pool;
  Launcher launch;
};

}  // namespace
}  // namespace tsb

using namespace tsb;

struct ts_batch {
  int32_t device = 0;
  int32_t count = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::vector<cudaStream_t> gstreams;
  std::vector<cudaEvent_t> events;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  DevBuf jobs, results, best, init, draws, tickets;
  std::vector<Group> groups;
  std::vector<int32_t> m_of, n_of;
  ts_batch_info info{};
  ~ts_batch() {
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (cudaEvent_t e : events) cudaEventDestroy(e);
    for (cudaStream_t s : gstreams) cudaStreamDestroy(s);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }
};

namespace tsb {
namespace {

// Geometry of every job of the group, slot pool within the budget, launcher.
template <int PROB, int ST, class KeyT>
ts_status plan_group(Group& G, std::vector<BatchJobDev>& table, int64_t budget_bytes,
                     int32_t max_slots, int sms) {
  constexpr int R = Rows<ST>::R;
  constexpr int TPB = TpbOf<ST, true>::v;
  const int cs = G.cluster;
  long long max_m = 1, max_n = 1, max_ldc = 4, max_entries = 1, max_w = 1, log_cap = 1;
  size_t smem = 16;
  for (size_t q = 0; q < G.jobs.size(); q++) {
    const HostJob& H = *G.jobs[q];
    BatchJobDev& J = table[G.job_off + q];
    const int32_t delta = H.n - H.m;
    const long long ldc = (delta + 3) & ~3;
    // tiles as in the plain solver, full row width where it fits; a cluster
    // gets at least one tile per CTA
    const TileGeom tg = tile_geometry(H.g, PROB, H.m, sizeof(KeyT) == 8, cs, H.p.pass, true);
    J.n_row_blocks = tg.n_row_blocks;
    J.tile_rows = tg.rows;
    J.fast = tg.fast;
    J.fast_ecap = tg.fast_ecap;
    J.adj_mask = tg.adj_mask;
    J.chunk_cols = tg.chunk_cols;
    J.n_chunks = tg.n_chunks;
    J.stage_bytes = tg.stage_bytes;
    const size_t need = tg.smem;
    smem = std::max(smem, need);
    max_m = std::max<long long>(max_m, H.m);
    max_n = std::max<long long>(max_n, H.n);
    max_ldc = std::max<long long>(max_ldc, ldc);
    if (ST == S_CSR) max_entries = std::max<long long>(max_entries, H.g->entries);
    if (ST == S_WSWAP) max_w = std::max<long long>(max_w, (long long)J.n_row_blocks * R * ldc);
    long long lc = H.p.max_iter + 1;
    if (PROB == P_MAXBS) lc += (H.p.max_iter / H.p.piter + 1) * (long long)H.num_pert;
    log_cap = std::max(log_cap, lc);
  }
  G.smem = smem;
  auto kern = batch_kernel<PROB, ST, KeyT>;
  TS_CUDA(allow_dyn_smem(reinterpret_cast<const void*>(kern), smem));
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(cs * sms));
  cfg.blockDim = dim3(TPB);
  cfg.dynamicSmemBytes = smem;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int resident = 0;
  TS_CUDA(cudaOccupancyMaxActiveClusters(&resident, kern, &cfg));
  if (resident < 1) {
    cudaFuncAttributes fa;
    std::string why;
    if (cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(kern)) == cudaSuccess)
      why = " (" + std::to_string(TPB) + " threads x " + std::to_string(fa.numRegs) + " registers, " +
            std::to_string(fa.sharedSizeBytes) + " B static + " + std::to_string(smem) +
            " B dynamic shared memory per CTA)";
    else
      cudaGetLastError();
    set_error("ts_batch_create: a cluster of " + std::to_string(cs) + " CTAs does not fit on the device" + why);
    return TS_ERR_UNSUPPORTED;
  }
  // slices padded to 256 B; strides in elements of each array
  const size_t kb = sizeof(KeyT);
  auto pad = [](size_t b) { return (b + 255) & ~(size_t)255; };
  SlotPool<KeyT> pool;
  pool.s_m = (long long)(pad(4 * max_m) / 4);
  pool.s_ldc = (long long)(pad(4 * max_ldc) / 4);
  pool.s_n = (long long)(pad(4 * max_n) / 4);
  pool.s_entries = ST == S_CSR ? (long long)(pad(4 * max_entries) / 4) : 0;
  pool.s_w = ST == S_WSWAP ? (long long)(pad(4 * max_w) / 4) : 0;
  pool.s_vgm = (long long)(pad(kb * max_m) / kb);
  pool.s_vgldc = (long long)(pad(kb * max_ldc) / kb);
  pool.log_cap = (long long)(pad(8 * log_cap) / 8);
  const size_t slices[] = {4 * (size_t)pool.s_m,  4 * (size_t)pool.s_ldc, 4 * (size_t)pool.s_m,
                           4 * (size_t)pool.s_ldc, 4 * (size_t)pool.s_n,   4 * (size_t)pool.s_entries,
                           4 * (size_t)pool.s_w,   kb * (size_t)pool.s_vgm, kb * (size_t)pool.s_vgldc,
                           sizeof(DevState),       8 * (size_t)pool.log_cap};
  size_t per_slot = 0;
  for (size_t x : slices) per_slot += x;
  long long slots = std::min<long long>(resident, (long long)G.jobs.size());
  if (max_slots > 0) slots = std::min<long long>(slots, max_slots);
  slots = std::min<long long>(slots, std::max<long long>(1, budget_bytes / (long long)per_slot));
  G.slots = slots;
  size_t total = 0;
  for (size_t x : slices) total += pad(x * (size_t)slots);
  G.pool.reset(new DevBuf);
  ts_status rc = G.pool->alloc(total, "alloc batch slots");
  if (rc != TS_OK) return rc;
  unsigned char* b = G.pool->as<unsigned char>();
  auto carve = [&](size_t slice) -> unsigned char* {  // one array: `slots` slices, 256 B aligned
    if (slice == 0) return nullptr;
    unsigned char* p = b;
    b += pad(slice * (size_t)slots);
    return p;
  };
  pool.sol_in = reinterpret_cast<int32_t*>(carve(slices[0]));
  pool.sol_out = reinterpret_cast<int32_t*>(carve(slices[1]));
  pool.tab_in = reinterpret_cast<int32_t*>(carve(slices[2]));
  pool.tab_out = reinterpret_cast<int32_t*>(carve(slices[3]));
  pool.pos = reinterpret_cast<int32_t*>(carve(slices[4]));
  pool.cpos = reinterpret_cast<int32_t*>(carve(slices[5]));
  pool.W = reinterpret_cast<int32_t*>(carve(slices[6]));
  pool.vg_in = reinterpret_cast<KeyT*>(carve(slices[7]));
  pool.vg_out = reinterpret_cast<KeyT*>(carve(slices[8]));
  pool.st = reinterpret_cast<DevState*>(carve(slices[9]));
  pool.movelog = reinterpret_cast<int2*>(carve(slices[10]));
  const long long ngrid = slots * cs;
  const int njobs = (int)G.jobs.size();
  const long long off = G.job_off;
  G.launch = [=](cudaStream_t s, const BatchJobDev* djobs, BatchResultDev* dres, int32_t* dbest,
                 unsigned int* ticket) -> cudaError_t {
    cudaLaunchAttribute a[1];
    a[0].id = cudaLaunchAttributeClusterDimension;
    a[0].val.clusterDim.x = cs;
    a[0].val.clusterDim.y = 1;
    a[0].val.clusterDim.z = 1;
    cudaLaunchConfig_t c = {};
    c.gridDim = dim3((unsigned)ngrid);
    c.blockDim = dim3(TPB);
    c.dynamicSmemBytes = smem;
    c.stream = s;
    c.attrs = a;
    c.numAttrs = 1;
    return cudaLaunchKernelEx(&c, kern, djobs + off, njobs, dres, dbest, pool, ticket);
  };
  return TS_OK;
}

template <int PROB, class KeyT>
ts_status plan_group_st(Group& G, std::vector<BatchJobDev>& table, int64_t budget, int32_t max_slots,
                        int sms) {
  switch (G.kind) {
    case S_CSR: return plan_group<PROB, S_CSR, KeyT>(G, table, budget, max_slots, sms);
    case S_HASH: return plan_group<PROB, S_HASH, KeyT>(G, table, budget, max_slots, sms);
    case S_WSWAP: return plan_group<PROB, S_WSWAP, KeyT>(G, table, budget, max_slots, sms);
    case S_BITSET: return plan_group<PROB, S_BITSET, KeyT>(G, table, budget, max_slots, sms);
    case S_BB: return plan_group<PROB, S_BB, KeyT>(G, table, budget, max_slots, sms);
    default: return plan_group<PROB, S_BITSET_BB, KeyT>(G, table, budget, max_slots, sms);
  }
}

// CTAs per solve when the job asks for "auto": a solve whose share of the
// batch's work would outlast the rest on one CTA is spread over a cluster, so
// the batch does not end on one long solve.
int32_t auto_cluster(double work, double total, int sms) {
  const double share = work * (2.0 * sms) / std::max(1.0, total);
  if (share < 0.5) return 1;
  if (share < 1.0) return 2;
  if (share < 2.0) return 4;
  return 8;
}

}  // namespace
}  // namespace tsb

extern "C" {

ts_status ts_batch_create(const ts_batch_job* jobs, int32_t count, const ts_batch_opts* opts,
                          void* stream, ts_batch** out) {
  tsb::TraceRange tr_("ts_batch_create");
  if (!out) { set_error("ts_batch_create: out is NULL"); return TS_ERR_INVALID_ARG; }
  *out = nullptr;
  if (count < 1 || !jobs) { set_error("ts_batch_create: need count >= 1 jobs"); return TS_ERR_INVALID_ARG; }
  ts_batch_opts o{};
  if (opts) o = *opts;
  std::vector<HostJob> hj(count);
  for (int32_t q = 0; q < count; q++) {
    const ts_batch_job& J = jobs[q];
    HostJob& H = hj[q];
    const ts_params& p = J.params;
    if (!J.graph) {
      set_error("ts_batch_create: job " + std::to_string(q) + " has no graph");
      return TS_ERR_INVALID_ARG;
    }
    if (J.graph->device != jobs[0].graph->device) {
      set_error("ts_batch_create: all graphs of a batch must live on one device");
      return TS_ERR_INVALID_ARG;
    }
    H.idx = q;
    H.g = J.graph;
    H.p = p;
    H.n = J.graph->n;
    H.m = p.problem == TS_PROBLEM_MDP ? p.m : H.n / 2;
    if ((p.problem != TS_PROBLEM_MDP && p.problem != TS_PROBLEM_MAXBS) || H.m < 1 || H.m >= H.n ||
        p.max_iter < 0 || p.piter < 1 || p.gamma < 0 || p.maxt < 1 || p.tenure < 0 ||
        (p.tenure_policy != TS_TENURE_REF && p.tenure_policy != TS_TENURE_FIXED) ||
        !(J.cluster == 0 || J.cluster == 1 || J.cluster == 2 || J.cluster == 4 || J.cluster == 8)) {
      set_error("ts_batch_create: bad parameters in job " + std::to_string(q));
      return TS_ERR_INVALID_ARG;
    }
    H.wide = 4 * J.graph->max_wdeg >= (1LL << 30);
    H.kind = J.graph->kind;
    H.num_pert = std::max(1, std::min(p.gamma, H.n) / 2);  // GPU-MAXBS-CSR.cu:433-434
    H.cluster = J.cluster;
    H.work = (double)H.m * (H.n - H.m) * (double)std::max<int64_t>(1, p.max_iter);
  }
  const int32_t device = jobs[0].graph->device;
  TS_CUDA(cudaSetDevice(device));
  int sms = 0;
  TS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));

  // starts and perturbation streams on the host cores
  {
    const int nt = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<int32_t> bad(nt, -1);
    std::vector<std::thread> th;
    for (int t = 0; t < nt; t++)
      th.emplace_back([&, t]() {
        for (int32_t q = t; q < count; q += nt)
          if (!prepare_host_job(hj[q], jobs[q].initial) && bad[t] < 0) bad[t] = q;
      });
    for (auto& x : th) x.join();
    for (int t = 0; t < nt; t++)
      if (bad[t] >= 0) {
        set_error("ts_batch_create: invalid start in job " + std::to_string(bad[t]) +
                  " (MDP: m distinct ids in [0,n); MaxBS: part[] of 0/1 with floor(n/2) zeros)");
        return TS_ERR_INVALID_ARG;
      }
  }

  std::unique_ptr<ts_batch> b(new ts_batch);
  b->device = device;
  b->count = count;
  if (stream) {
    b->stream = static_cast<cudaStream_t>(stream);
  } else {
    TS_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    b->own_stream = true;
  }
  // groups by (problem, structure, key width, CTAs per solve); largest solves first
  double total = 0;
  for (auto& H : hj) total += H.work;
  for (auto& H : hj) {
    const int32_t cs = H.cluster ? H.cluster : auto_cluster(H.work, total, sms);
    Group* G = nullptr;
    for (auto& x : b->groups)
      if (x.problem == H.p.problem && x.kind == H.kind && x.wide == H.wide && x.cluster == cs) G = &x;
    if (!G) {
      b->groups.emplace_back();
      G = &b->groups.back();
      G->problem = H.p.problem;
      G->kind = H.kind;
      G->wide = H.wide;
      G->cluster = cs;
    }
    G->jobs.push_back(&H);
    G->work += H.work;
  }
  long long off = 0;
  for (auto& G : b->groups) {
    std::stable_sort(G.jobs.begin(), G.jobs.end(),
                     [](const HostJob* a, const HostJob* c) { return a->work > c->work; });
    G.job_off = off;
    off += (long long)G.jobs.size();
  }
  long long sol_words = 0, init_words = 0, draw_words = 0;
  std::vector<long long> sol_off(count), init_at(count), draw_at(count);
  for (int32_t q = 0; q < count; q++) {
    sol_off[q] = sol_words;
    init_at[q] = init_words;
    draw_at[q] = draw_words;
    sol_words += hj[q].p.problem == TS_PROBLEM_MDP ? hj[q].m : hj[q].n;
    init_words += (long long)hj[q].init.size();
    draw_words += (long long)hj[q].draws.size();
  }
  ts_status rc;
  if ((rc = b->init.alloc(4 * (size_t)std::max<long long>(1, init_words), "alloc batch starts")) != TS_OK) return rc;
  if ((rc = b->draws.alloc(8 * (size_t)std::max<long long>(1, draw_words), "alloc batch draws")) != TS_OK) return rc;
  if ((rc = b->best.alloc(4 * (size_t)std::max<long long>(1, sol_words), "alloc batch best solutions")) != TS_OK)
    return rc;
  if ((rc = b->results.alloc(sizeof(BatchResultDev) * (size_t)count, "alloc batch results")) != TS_OK) return rc;
  if ((rc = b->jobs.alloc(sizeof(BatchJobDev) * (size_t)count, "alloc batch jobs")) != TS_OK) return rc;
  if ((rc = b->tickets.alloc(sizeof(unsigned int) * b->groups.size(), "alloc batch tickets")) != TS_OK) return rc;
  std::vector<int32_t> hi(std::max<long long>(1, init_words));
  std::vector<long long> hd(std::max<long long>(1, draw_words));
  for (int32_t q = 0; q < count; q++) {
    std::copy(hj[q].init.begin(), hj[q].init.end(), hi.begin() + init_at[q]);
    std::copy(hj[q].draws.begin(), hj[q].draws.end(), hd.begin() + draw_at[q]);
  }
  std::vector<BatchJobDev> table(count);
  for (auto& G : b->groups)
    for (size_t q = 0; q < G.jobs.size(); q++) {
      const HostJob& H = *G.jobs[q];
      BatchJobDev& J = table[G.job_off + q];
      std::memset(&J, 0, sizeof(J));
      J.g = H.g->dev();
      J.n = H.n;
      J.m = H.m;
      J.max_iter = H.p.max_iter;
      J.tenure_policy = H.p.tenure_policy;
      J.tenure = H.p.tenure;
      J.maxt = H.p.maxt;
      J.piter = H.p.piter;
      J.num_pert = H.num_pert;
      J.c2_fixed = (int32_t)round(0.7 * H.p.tenure);
      J.orig = H.idx;
      J.init = b->init.as<int32_t>() + init_at[H.idx];
      J.draws = b->draws.as<long long>() + draw_at[H.idx];
      J.draw_events = H.events;
      J.sol_off = sol_off[H.idx];
    }
  TS_CUDA(cudaMemcpyAsync(b->init.p, hi.data(), 4 * hi.size(), cudaMemcpyHostToDevice, b->stream));
  TS_CUDA(cudaMemcpyAsync(b->draws.p, hd.data(), 8 * hd.size(), cudaMemcpyHostToDevice, b->stream));
  // slot budget, shared out by work
  int64_t budget = o.max_bytes;
  if (budget <= 0) {
    size_t fr = 0, tot = 0;
    TS_CUDA(cudaMemGetInfo(&fr, &tot));
    budget = (int64_t)(0.6 * (double)fr);
  }
  for (auto& G : b->groups) {
    const int64_t gb = (int64_t)((double)budget * G.work / std::max(1.0, total));
    if (G.problem == P_MDP)
      rc = G.wide ? plan_group_st<P_MDP, long long>(G, table, gb, o.max_slots, sms)
                  : plan_group_st<P_MDP, int32_t>(G, table, gb, o.max_slots, sms);
    else
      rc = G.wide ? plan_group_st<P_MAXBS, long long>(G, table, gb, o.max_slots, sms)
                  : plan_group_st<P_MAXBS, int32_t>(G, table, gb, o.max_slots, sms);
    if (rc != TS_OK) return rc;
    b->info.slots += G.slots;
    b->info.slot_bytes += (int64_t)G.pool->bytes;
  }
  TS_CUDA(cudaMemcpyAsync(b->jobs.p, table.data(), sizeof(BatchJobDev) * table.size(), cudaMemcpyHostToDevice,
                          b->stream));
  TS_CUDA(cudaStreamSynchronize(b->stream));

  // capture: fork one branch per group, join on the batch stream
  cudaEvent_t fork;
  TS_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  b->events.push_back(fork);
  for (size_t gi = 0; gi < b->groups.size(); gi++) {
    cudaStream_t s;
    cudaEvent_t e;
    TS_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    b->gstreams.push_back(s);
    TS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->events.push_back(e);
  }
  TS_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t ce = cudaEventRecord(fork, b->stream);
  for (size_t gi = 0; gi < b->groups.size() && ce == cudaSuccess; gi++) {
    cudaStream_t s = b->gstreams[gi];
    unsigned int* ticket = b->tickets.as<unsigned int>() + gi;
    ce = cudaStreamWaitEvent(s, fork, 0);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(ticket, 0, sizeof(unsigned int), s);
    if (ce == cudaSuccess)
      ce = b->groups[gi].launch(s, b->jobs.as<BatchJobDev>(), b->results.as<BatchResultDev>(),
                                b->best.as<int32_t>(), ticket);
    if (ce == cudaSuccess) ce = cudaEventRecord(b->events[gi + 1], s);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(b->stream, b->events[gi + 1], 0);
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(b->stream, &graph);
  if (ce != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return cuda_fail(ce, "ts_batch_create: capture of the batch launches");
  }
  if (ee != cudaSuccess) return cuda_fail(ee, "cudaStreamEndCapture");
  b->graph = graph;
  TS_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
  b->m_of.resize(count);
  b->n_of.resize(count);
  for (int32_t q = 0; q < count; q++) {
    b->m_of[q] = hj[q].m;
    b->n_of[q] = hj[q].n;
  }
  b->info.jobs = count;
  b->info.groups = (int32_t)b->groups.size();
  b->info.input_bytes = (int64_t)(b->init.bytes + b->draws.bytes + b->best.bytes + b->results.bytes +
                                  b->jobs.bytes + b->tickets.bytes);
  b->info.best_sol_words = sol_words;
  *out = b.release();
  return TS_OK;
}

ts_status ts_batch_launch(ts_batch* b) {
  tsb::TraceRange tr_("ts_batch_launch");
  if (!b) { set_error("ts_batch_launch: NULL batch"); return TS_ERR_INVALID_ARG; }
  TS_CUDA(cudaSetDevice(b->device));
  TS_CUDA(cudaGraphLaunch(b->exec, b->stream));
  return TS_OK;
}

ts_status ts_batch_sync(ts_batch* b) {
  tsb::TraceRange tr_("ts_batch_sync");
  if (!b) { set_error("ts_batch_sync: NULL batch"); return TS_ERR_INVALID_ARG; }
  TS_CUDA(cudaSetDevice(b->device));
  TS_CUDA(cudaStreamSynchronize(b->stream));
  return TS_OK;
}

ts_status ts_batch_results(ts_batch* b, ts_result* out, int32_t* best_sols) {
  tsb::TraceRange tr_("ts_batch_results");
  if (!b) { set_error("ts_batch_results: NULL batch"); return TS_ERR_INVALID_ARG; }
  TS_CUDA(cudaSetDevice(b->device));
  std::vector<BatchResultDev> r(b->count);
  TS_CUDA(cudaMemcpyAsync(r.data(), b->results.p, sizeof(BatchResultDev) * r.size(), cudaMemcpyDeviceToHost,
                          b->stream));
  if (best_sols)
    TS_CUDA(cudaMemcpyAsync(best_sols, b->best.p, 4 * (size_t)b->info.best_sol_words, cudaMemcpyDeviceToHost,
                            b->stream));
  TS_CUDA(cudaStreamSynchronize(b->stream));
  int32_t errs = 0;
  for (int32_t q = 0; q < b->count; q++) {
    errs |= r[q].err;
    if (!out) continue;
    ts_result& o = out[q];
    std::memset(&o, 0, sizeof(o));
    o.iterations = r[q].iterations;
    o.evaluations = r[q].evaluations;
    o.cur = r[q].cur;
    o.best = r[q].best;
    o.best_true = r[q].best_true;
    o.perturbations = r[q].perturbations;
    o.stopped = r[q].stopped;
    o.m = b->m_of[q];
    o.n = b->n_of[q];
    o.device_error = r[q].err;
  }
  if (errs) {
    set_error("ts_batch_results: device error word set in at least one job (" + std::to_string(errs) + ")");
    return TS_ERR_DEVICE;
  }
  return TS_OK;
}

ts_status ts_batch_info_get(const ts_batch* b, ts_batch_info* out) {
  if (!b || !out) { set_error("ts_batch_info_get: NULL argument"); return TS_ERR_INVALID_ARG; }
  *out = b->info;
  return TS_OK;
}

ts_status ts_batch_destroy(ts_batch* b) {
  delete b;
  return TS_OK;
}

ts_status ts_batch_run(const ts_batch_job* jobs, int32_t count, const ts_batch_opts* opts, ts_result* out,
                       int32_t* best_sols) {
  ts_batch* b = nullptr;
  ts_status rc = ts_batch_create(jobs, count, opts, nullptr, &b);
  if (rc != TS_OK) return rc;
  rc = ts_batch_launch(b);
  if (rc == TS_OK) rc = ts_batch_sync(b);
  if (rc == TS_OK) rc = ts_batch_results(b, out, best_sols);
  ts_batch_destroy(b);
  return rc;
}

}  // extern "C"
