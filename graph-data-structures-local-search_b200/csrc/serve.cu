// serve.cu -- the served form: a request loop with continuous batching.
//
// One scheduler thread owns the device work.  Each round it
//   1. admits queued requests (FIFO) while their HBM footprint fits the
//      budget: builds the graph on the device and the solve's state;
//   2. advances every admitted solve by a bounded number of iterations sized
//      to the round's target duration:
//        - small solves ("packed"): one launch per (problem, structure, key
//          width, cluster size) group, one thread-block cluster per solve,
//          running its iterations with the batched form's device code
//          (packed.cuh) on state that stays resident between rounds;
//        - large solves ("plain"): the one-launch-per-iteration kernel of
//          ts_solver_* on the solve's own stream, using the whole GPU;
//      all groups and plain solves run concurrently on separate streams;
//   3. collects completed solves (result, best solution), frees their memory.
// A request that arrives during a round joins at the next one, so short
// requests do not wait for long ones.  Every solve computes exactly what the
// plain solver computes for its graph and parameters.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <random>
#include <thread>
#include <tuple>
#include <vector>

#include "packed.cuh"
#include "ts_host.h"

namespace cg = cooperative_groups;

namespace tsb {
namespace {

template <class KeyT>
struct ServeJobDev {
  DevGraph g;
  DevSolver<KeyT> s;
  const int32_t* init;
  long long max_iter;
  long long stop_at;       // this launch runs the solve up to this iteration
  int32_t need_init;
  int32_t pad;
  BatchResultDev* out;     // written when the solve ends
  int32_t* best_out;
};

// One cluster per job; the job runs until stop_at, its end or max_iter.
template <int PROB, int ST, class KeyT>
__global__ void __launch_bounds__((TpbOf<ST, true>::v))
serve_kernel(const ServeJobDev<KeyT>* __restrict__ jobs) {
  cg::cluster_group cl = cg::this_cluster();
  const unsigned rank = cl.block_rank(), cs = cl.num_blocks();
  __shared__ TailShared sh;
  __shared__ CtaRec s_rec;
  __shared__ long long sc[kMaxTPB / 32];
  __shared__ int32_t s_cnt[kMaxTPB];
  const ServeJobDev<KeyT> J = jobs[blockIdx.x / cs];
  if (rank == 0 && J.need_init) {
    slot_init<PROB, ST, KeyT>(J.g, J.s, J.init, J.max_iter, sc, s_cnt);
    __threadfence();
  }
  cl.sync();
  cluster_iterate<PROB, ST, KeyT>(J.g, J.s, J.stop_at < J.max_iter ? J.stop_at : J.max_iter, cl, sh, s_rec);
  if (rank == 0) {
    const DevState* st = J.s.st;
    if (__ldcg(&st->done) || __ldcg(&st->iter) >= J.max_iter)
      slot_finish<PROB, KeyT>(J.g, J.s, J.out, J.best_out, sc);
  }
}

template <int PROB, int ST, class KeyT>
cudaError_t launch_serve(cudaStream_t st, const void* jobs, int njobs, int cs, size_t smem) {
  auto kern = serve_kernel<PROB, ST, KeyT>;
  cudaError_t e = allow_dyn_smem(reinterpret_cast<const void*>(kern), smem);
  if (e != cudaSuccess) return e;
  cudaLaunchAttribute a[1];
  a[0].id = cudaLaunchAttributeClusterDimension;
  a[0].val.clusterDim.x = cs;
  a[0].val.clusterDim.y = 1;
  a[0].val.clusterDim.z = 1;
  cudaLaunchConfig_t c = {};
  c.gridDim = dim3((unsigned)(njobs * cs));
  c.blockDim = dim3(TpbOf<ST, true>::v);
  c.dynamicSmemBytes = smem;
  c.stream = st;
  c.attrs = a;
  c.numAttrs = 1;
  return cudaLaunchKernelEx(&c, kern, static_cast<const ServeJobDev<KeyT>*>(jobs));
}

using ServeLauncher = cudaError_t (*)(cudaStream_t, const void*, int, int, size_t);

template <int PROB, class KeyT>
ServeLauncher serve_launcher_st(int kind) {
  switch (kind) {
    case S_CSR: return launch_serve<PROB, S_CSR, KeyT>;
    case S_HASH: return launch_serve<PROB, S_HASH, KeyT>;
    case S_WSWAP: return launch_serve<PROB, S_WSWAP, KeyT>;
    case S_BITSET: return launch_serve<PROB, S_BITSET, KeyT>;
    case S_BB: return launch_serve<PROB, S_BB, KeyT>;
    default: return launch_serve<PROB, S_BITSET_BB, KeyT>;
  }
}

ServeLauncher serve_launcher(int problem, int kind, bool wide) {
  if (problem == P_MDP) return wide ? serve_launcher_st<P_MDP, long long>(kind) : serve_launcher_st<P_MDP, int32_t>(kind);
  return wide ? serve_launcher_st<P_MAXBS, long long>(kind) : serve_launcher_st<P_MAXBS, int32_t>(kind);
}

double now_s(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

struct Req {
  int64_t ticket = 0;
  int32_t n = 0, m = 0, kind = 0, drop = 0;
  ts_params p{};
  std::vector<int32_t> u, v, w, initial;
  int32_t* best_sol = nullptr;
  double t_submit = 0, t_admit = 0;
  int64_t footprint = 0;
  int64_t P = 0;
  int32_t num_pert = 1;
  bool plain = false, wide = false;
  int32_t cs = 1;
  size_t smem = 16;  // packed: dynamic shared memory of one tile (tile_geometry)
  // device resources
  ts_graph* g = nullptr;
  cudaStream_t stream = nullptr;   // plain: the graph's and solver's stream
  ts_solver* solver = nullptr;     // plain
  std::unique_ptr<DevBuf> mem;     // packed: solver state, start, draws, result, best
  std::vector<unsigned char> dev_solver;  // packed: DevSolver<KeyT> bytes
  DevGraph dg{};
  int32_t* d_init = nullptr;
  BatchResultDev* d_res = nullptr;
  int32_t* d_best = nullptr;
  long long granted = 0;           // packed: iterations granted so far
  bool started = false;
  // plain: streams per priority level (created on first use), the current
  // level and the event that orders a move between them
  cudaStream_t pstream[8] = {};
  int level = -1;
  cudaEvent_t moved = nullptr;
  double spi = 0;      // plain: measured seconds per iteration inside rounds (0: not yet)
  int64_t last_k = 0;  // plain: iterations enqueued in the last round
  cudaEvent_t ev_a = nullptr, ev_b = nullptr;  // plain: bracket the last round's launches
};

int64_t estimate_footprint(const Req& r) {
  const int64_t n = r.n, E = (int64_t)r.u.size(), ent = 2 * E;
  int64_t gb = 8 * (n + 1) + 8 * ent + 8 * ent;  // rowptr, adj, reverse index
  gb += 32 * E;                                  // build temporaries
  if (r.kind == S_BITSET || r.kind == S_BITSET_BB) gb += n * (((n + 127) / 128) * 2) * 8;
  if (r.kind == S_HASH) gb += 8 * (n + 1) + 8 * (8 * ent + 8 * n);
  const int64_t m = r.m, ldc = ((n - m) + 3) & ~3LL;
  int64_t sb = 8 * (m + ldc) * 3 + 4 * n + 4 * ent;
  if (r.kind == S_WSWAP) sb += 4 * (m + 32) * ldc;
  const int64_t events = r.p.problem == P_MAXBS ? r.p.max_iter / std::max(1, r.p.piter) + 1 : 0;
  sb += 8 * (r.p.max_iter + 1 + (events + 1) * r.num_pert) + 8 * events * r.num_pert;
  sb += 16 * 8 * 148;  // per-CTA records of the plain kernel
  return gb + sb + (1 << 20);
}

}  // namespace
}  // namespace tsb

using namespace tsb;

struct ts_server {
  int32_t device = 0;
  int sms = 148;
  int prio_least = 0, prio_greatest = 0;  // stream priority range (greatest = numerically lowest)
  double last_round_s = 0;                // wall time of the previous round
  ts_server_opts opts{};
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::unique_ptr<Req>> queue;
  std::deque<ts_served> done;
  std::vector<std::unique_ptr<Req>> active;
  int64_t next_ticket = 1;
  bool stopping = false;
  std::thread worker;
  ts_server_stats stats{};
  double busy_since = -1;
  // packed groups: per key a stream, a device job table and its pinned copy
  struct Group {
    cudaStream_t stream = nullptr;
    DevBuf table;
    void* host = nullptr;
    size_t cap = 0;
  };
  std::map<std::tuple<int, int, int, int>, Group> groups;
  void run();
  void admit();
  ts_status start(Req& r);
  void finish(Req& r, ts_status st, const ts_result* res);
  void round();
  ~ts_server() {
    for (auto& kv : groups) {
      if (kv.second.stream) cudaStreamDestroy(kv.second.stream);
      if (kv.second.host) cudaFreeHost(kv.second.host);
    }
  }
};

namespace {

template <class KeyT>
ts_status build_packed(Req& r, int32_t kind) {
  const int32_t n = r.n, m = r.m, delta = n - m;
  const int R = rows_of(kind);  // WSwap matrix rows come in whole blocks of R
  const int64_t ldc = (delta + 3) & ~3;
  DevSolver<KeyT> s;
  std::memset(&s, 0, sizeof(s));
  s.n = n; s.m = m; s.delta = delta; s.ldc = (int32_t)ldc;
  s.problem = r.p.problem;
  s.tenure_policy = r.p.tenure_policy; s.tenure = r.p.tenure; s.maxt = r.p.maxt; s.piter = r.p.piter;
  s.num_pert = r.num_pert;
  const int c1s[4] = {15, 30, 60, 120};
  for (int i = 0; i < 4; i++) s.c2_tab[i] = (int32_t)round(0.7 * c1s[i]);
  s.c2_fixed = (int32_t)round(0.7 * r.p.tenure);
  const TileGeom tg = tile_geometry(r.g, r.p.problem, m, sizeof(KeyT) == 8, r.cs, r.p.pass, true);
  s.n_row_blocks = tg.n_row_blocks;
  s.tile_rows = tg.rows;
  s.fast = tg.fast;
  s.fast_ecap = tg.fast_ecap;
  s.adj_mask = tg.adj_mask;
  s.chunk_cols = tg.chunk_cols;
  s.n_chunks = tg.n_chunks;
  s.stage_bytes = tg.stage_bytes;
  r.smem = tg.smem;
  s.P = (int64_t)m * delta;
  const int64_t entries = r.g->entries;
  const int64_t events = r.p.problem == P_MAXBS ? r.p.max_iter / r.p.piter + 1 : 0;
  s.log_cap = r.p.max_iter + 1 + (r.p.problem == P_MAXBS ? (events + 1) * (int64_t)r.num_pert : 0);
  auto pad = [](int64_t b) { return (b + 255) & ~255LL; };
  const int64_t sizes[] = {4 * m, 4 * ldc, 4 * m, 4 * ldc, 4 * (int64_t)n,
                           kind == S_CSR ? 4 * std::max<int64_t>(1, entries) : 0,
                           kind == S_WSWAP ? 4 * (int64_t)s.n_row_blocks * R * ldc : 0,
                           (int64_t)sizeof(KeyT) * m, (int64_t)sizeof(KeyT) * ldc, (int64_t)sizeof(DevState),
                           8 * s.log_cap, 8 * std::max<int64_t>(1, events * r.num_pert),
                           4 * (int64_t)(r.p.problem == P_MDP ? m : n), (int64_t)sizeof(BatchResultDev),
                           4 * (int64_t)(r.p.problem == P_MDP ? m : n)};
  int64_t total = 0;
  for (int64_t x : sizes) total += pad(x);
  r.mem.reset(new DevBuf);
  ts_status rc = r.mem->alloc((size_t)total, "alloc served solve");
  if (rc != TS_OK) return rc;
  unsigned char* b = r.mem->as<unsigned char>();
  unsigned char* ptrs[15];
  for (int i = 0; i < 15; i++) {
    ptrs[i] = sizes[i] ? b : nullptr;
    b += pad(sizes[i]);
  }
  s.sol_in = reinterpret_cast<int32_t*>(ptrs[0]);
  s.sol_out = reinterpret_cast<int32_t*>(ptrs[1]);
  s.tab_in = reinterpret_cast<int32_t*>(ptrs[2]);
  s.tab_out = reinterpret_cast<int32_t*>(ptrs[3]);
  s.pos = reinterpret_cast<int32_t*>(ptrs[4]);
  s.cpos = reinterpret_cast<int32_t*>(ptrs[5]);
  s.W = reinterpret_cast<int32_t*>(ptrs[6]);
  s.vg_in = reinterpret_cast<KeyT*>(ptrs[7]);
  s.vg_out = reinterpret_cast<KeyT*>(ptrs[8]);
  s.st = reinterpret_cast<DevState*>(ptrs[9]);
  s.movelog = reinterpret_cast<int2*>(ptrs[10]);
  s.draws = reinterpret_cast<const long long*>(ptrs[11]);
  s.draw_events = events;
  r.d_init = reinterpret_cast<int32_t*>(ptrs[12]);
  r.d_res = reinterpret_cast<BatchResultDev*>(ptrs[13]);
  r.d_best = reinterpret_cast<int32_t*>(ptrs[14]);
  // starts and draws, as ts_solver_init draws them
  std::vector<long long> draws;
  std::vector<int32_t> init;
  std::mt19937 rng;
  rng.seed(r.p.seed);
  if (r.p.problem == P_MDP) {
    if (r.initial.empty()) mdp_random_set(n, m, r.p.seed, init);
    else init = r.initial;
  } else {
    if (r.initial.empty()) {
      std::vector<uint8_t> side0;
      maxbs_random_part(rng, n, side0);
      init.assign(n, 1);
      for (int32_t v = 0; v < n; v++) init[v] = side0[v] ? 0 : 1;
    } else {
      init = r.initial;
    }
    for (int64_t e = 0; e < events; e++) draw_event(rng, s.P, r.num_pert, draws);
  }
  cudaStream_t st = r.stream;
  if ((int64_t)init.size() * 4 != sizes[12] || (int64_t)draws.size() * 8 > sizes[11]) {
    set_error("ts_server: start or draw sizes do not match the solve");
    return TS_ERR_INVALID_ARG;
  }
  TS_CUDA(cudaMemcpyAsync(r.d_init, init.data(), 4 * init.size(), cudaMemcpyHostToDevice, st));
  if (!draws.empty())
    TS_CUDA(cudaMemcpyAsync(ptrs[11], draws.data(), 8 * draws.size(), cudaMemcpyHostToDevice, st));
  TS_CUDA(cudaMemsetAsync(r.d_res, 0, sizeof(BatchResultDev), st));
  TS_CUDA(cudaStreamSynchronize(st));
  r.dev_solver.resize(sizeof(s));
  std::memcpy(r.dev_solver.data(), &s, sizeof(s));
  r.dg = r.g->dev();
  return TS_OK;
}

}  // namespace

// Creates the request's graph and solve state.
ts_status ts_server::start(Req& r) {
  TS_CUDA(cudaStreamCreateWithFlags(&r.stream, cudaStreamNonBlocking));
  ts_status rc = ts_graph_create(r.n, (int64_t)r.u.size(), r.u.data(), r.v.data(), r.w.data(), r.kind, r.drop,
                                 r.stream, &r.g);
  if (rc != TS_OK) return rc;
  std::vector<int32_t>().swap(r.u);
  std::vector<int32_t>().swap(r.v);
  std::vector<int32_t>().swap(r.w);
  r.wide = 4 * r.g->max_wdeg >= (1LL << 30);
  if (r.plain) {
    if ((rc = ts_solver_create(r.g, &r.p, &r.solver)) != TS_OK) return rc;
    return ts_solver_init(r.solver, r.initial.empty() ? nullptr : r.initial.data());
  }
  if (r.p.problem == P_MDP) {
    std::vector<uint8_t> seen(r.n, 0);
    for (int32_t x : r.initial) {
      if (x < 0 || x >= r.n || seen[x]) { set_error("ts_server: bad MDP start"); return TS_ERR_INVALID_ARG; }
      seen[x] = 1;
    }
  } else if (!r.initial.empty()) {
    int32_t zeros = 0;
    for (int32_t x : r.initial) {
      if (x != 0 && x != 1) { set_error("ts_server: bad MaxBS start"); return TS_ERR_INVALID_ARG; }
      zeros += x == 0;
    }
    if (zeros != r.m) { set_error("ts_server: unbalanced MaxBS start"); return TS_ERR_INVALID_ARG; }
  }
  return r.wide ? build_packed<long long>(r, r.kind) : build_packed<int32_t>(r, r.kind);
}

void ts_server::finish(Req& r, ts_status status, const ts_result* res) {
  ts_served d;
  std::memset(&d, 0, sizeof(d));
  d.ticket = r.ticket;
  d.status = status;
  d.executor = r.plain ? 1 : 0;
  d.kind = r.kind;
  if (res) d.result = *res;
  d.submit_s = r.t_submit;
  d.admit_s = r.t_admit;
  d.done_s = now_s(t0);
  d.footprint_bytes = r.footprint;
  if (r.solver) ts_solver_destroy(r.solver);
  r.solver = nullptr;
  if (r.g) ts_graph_destroy(r.g);
  r.g = nullptr;
  r.mem.reset();
  if (r.stream) cudaStreamDestroy(r.stream);
  r.stream = nullptr;
  for (cudaStream_t& ps : r.pstream) {
    if (ps) cudaStreamDestroy(ps);
    ps = nullptr;
  }
  if (r.moved) cudaEventDestroy(r.moved);
  r.moved = nullptr;
  if (r.ev_a) cudaEventDestroy(r.ev_a);
  if (r.ev_b) cudaEventDestroy(r.ev_b);
  r.ev_a = r.ev_b = nullptr;
  std::lock_guard<std::mutex> lk(mu);
  stats.completed++;
  stats.active--;
  stats.bytes_in_use -= r.footprint;
  done.push_back(d);
  cv_done.notify_all();
}

void ts_server::admit() {
  for (;;) {
    std::unique_ptr<Req> r;
    {
      std::lock_guard<std::mutex> lk(mu);
      if (queue.empty()) return;
      Req& h = *queue.front();
      // FIFO; a request larger than the whole budget is admitted alone
      if (stats.bytes_in_use + h.footprint > stats.bytes_budget && stats.bytes_in_use > 0) return;
      r = std::move(queue.front());
      queue.pop_front();
      stats.queued--;
      stats.admitted++;
      stats.active++;
      stats.bytes_in_use += r->footprint;
    }
    r->t_admit = now_s(t0);
    ts_status rc = start(*r);
    if (rc != TS_OK) {
      finish(*r, rc, nullptr);
      continue;
    }
    active.push_back(std::move(r));
  }
}

void ts_server::round() {
  TraceRange tr_("ts_server round");
  const double round_s = opts.round_ms * 1e-3;
  const double t_round = now_s(t0);
  // Plain solves get the iterations that fill the round at their measured
  // speed (the last round's length, at least round_ms, at most 50 ms), so a
  // large solve never idles while the round waits for the others.
  const double target_s = std::max(round_s, std::min(last_round_s, 0.05));
  // plain solves: admit the next iterations and enqueue their launches.
  // Every solve progresses, on a stream whose priority follows its age (the
  // oldest highest): the block scheduler starts the older solves' CTAs first
  // and the younger ones fill the SMs left idle, so a large early arrival is
  // not slowed to 1/N speed by everything admitted after it.  A solve that
  // changes rank moves to the stream of its new level, ordered after its
  // previous stream by an event.
  std::vector<Req*> plain_done;
  const int levels = std::max(1, prio_least - prio_greatest + 1);
  int rank = 0;
  for (auto& rp : active) {
    Req& r = *rp;
    if (!r.plain) continue;
    const int level = std::min(rank++, levels - 1);
    if (level != r.level && r.g) {
      if (!r.pstream[level])
        cudaStreamCreateWithPriority(&r.pstream[level], cudaStreamNonBlocking, prio_greatest + level);
      if (!r.moved) cudaEventCreateWithFlags(&r.moved, cudaEventDisableTiming);
      if (r.pstream[level] && r.moved && cudaEventRecord(r.moved, r.g->stream) == cudaSuccess &&
          cudaStreamWaitEvent(r.pstream[level], r.moved, 0) == cudaSuccess) {
        r.g->stream = r.pstream[level];
        r.level = level;
      }
      cudaGetLastError();
    }
    const double est = r.spi > 0 ? r.spi : 12e-6 + (double)r.P / 1.5e12;
    const int64_t k = std::max<int64_t>(4, std::min<int64_t>(1 << 16, (int64_t)(target_s / est)));
    int64_t adm = 0;
    ts_status rc = ts_solver_prepare(r.solver, k, &adm);
    r.last_k = 0;
    if (rc == TS_OK && adm > 0) {
      if (!r.ev_a) cudaEventCreate(&r.ev_a);
      if (!r.ev_b) cudaEventCreate(&r.ev_b);
      const bool timed = r.ev_a && r.ev_b && cudaEventRecord(r.ev_a, r.g->stream) == cudaSuccess;
      rc = ts_solver_enqueue(r.solver, adm);
      if (rc == TS_OK && timed && cudaEventRecord(r.ev_b, r.g->stream) == cudaSuccess) r.last_k = adm;
      cudaGetLastError();
    }
    if (rc != TS_OK) {
      r.started = false;
      finish(r, rc, nullptr);
      r.ticket = -1;
      continue;
    }
    if (adm == 0) plain_done.push_back(&r);
  }
  // packed solves: one launch per group
  std::map<std::tuple<int, int, int, int>, std::vector<Req*>> by_group;
  for (auto& rp : active) {
    Req& r = *rp;
    if (r.plain || r.ticket < 0) continue;
    by_group[std::make_tuple(r.p.problem, r.kind, r.wide ? 1 : 0, r.cs)].push_back(&r);
  }
  std::vector<cudaStream_t> used;
  for (auto& kv : by_group) {
    Group& G = groups[kv.first];
    std::vector<Req*>& js = kv.second;
    const bool wide = std::get<2>(kv.first) != 0;
    const size_t rec = wide ? sizeof(ServeJobDev<long long>) : sizeof(ServeJobDev<int32_t>);
    // packed groups hold the small requests: top priority
    if (!G.stream) cudaStreamCreateWithPriority(&G.stream, cudaStreamNonBlocking, prio_greatest);
    if (!G.stream) {
      for (Req* r : js) {
        finish(*r, cuda_fail(cudaGetLastError(), "serve group stream"), nullptr);
        r->ticket = -1;
      }
      continue;
    }
    if (G.cap < js.size()) {
      const size_t cap = std::max<size_t>(64, js.size() * 2);
      if (G.host) cudaFreeHost(G.host);
      G.host = nullptr;
      G.cap = 0;
      ts_status rc = TS_OK;
      if (cudaMallocHost(&G.host, rec * cap) != cudaSuccess) {
        G.host = nullptr;
        rc = cuda_fail(cudaErrorMemoryAllocation, "serve job table (host)");
      } else {
        rc = G.table.alloc(rec * cap, "alloc serve table");
      }
      if (rc != TS_OK) {
        for (Req* r : js) {
          finish(*r, rc, nullptr);
          r->ticket = -1;
        }
        continue;
      }
      G.cap = cap;
    }
    size_t smem = 16;
    for (size_t q = 0; q < js.size(); q++) {
      Req& r = *js[q];
      const double per_cta = 5e9;
      const double est = 6e-6 + (double)r.P / (per_cta * r.cs);
      const int64_t k = std::max<int64_t>(4, std::min<int64_t>(1 << 16, (int64_t)(round_s / est)));
      r.granted += k;
      unsigned char* dst = static_cast<unsigned char*>(G.host) + rec * q;
      auto fill = [&](auto* J) {
        using JT = std::remove_pointer_t<decltype(J)>;
        std::memset(J, 0, sizeof(JT));
        J->g = r.dg;
        std::memcpy(&J->s, r.dev_solver.data(), sizeof(J->s));
        J->init = r.d_init;
        J->max_iter = r.p.max_iter;
        J->stop_at = r.granted;
        J->need_init = r.started ? 0 : 1;
        J->out = r.d_res;
        J->best_out = r.d_best;
        smem = std::max(smem, r.smem);
      };
      if (wide) fill(reinterpret_cast<ServeJobDev<long long>*>(dst));
      else fill(reinterpret_cast<ServeJobDev<int32_t>*>(dst));
      r.started = true;
    }
    cudaMemcpyAsync(G.table.p, G.host, rec * js.size(), cudaMemcpyHostToDevice, G.stream);
    ServeLauncher L = serve_launcher(std::get<0>(kv.first), std::get<1>(kv.first), wide);
    cudaError_t e = L(G.stream, G.table.p, (int)js.size(), std::get<3>(kv.first), smem);
    if (e != cudaSuccess) {
      ts_status rc = cuda_fail(e, "serve kernel launch");
      for (Req* r : js) {
        finish(*r, rc, nullptr);
        r->ticket = -1;
      }
      continue;
    }
    used.push_back(G.stream);
  }
  // wait for the round
  for (Req* r : plain_done) {
    ts_result res;
    ts_status rc = ts_solver_result(r->solver, &res, r->best_sol);
    finish(*r, rc, rc == TS_OK ? &res : nullptr);
    r->ticket = -1;
  }
  for (auto& rp : active) {
    Req& r = *rp;
    if (!r.plain || r.ticket < 0) continue;
    int64_t it = 0;
    ts_status rc = ts_solver_sync(r.solver, &it);
    if (rc != TS_OK) {
      finish(r, rc, nullptr);
      r.ticket = -1;
    }
  }
  for (cudaStream_t s : used) cudaStreamSynchronize(s);
  last_round_s = now_s(t0) - t_round;
  for (auto& rp : active) {  // speed of each plain solve in this round (shared GPU included)
    Req& r = *rp;
    if (!r.plain || r.ticket < 0 || r.last_k <= 0) continue;
    float ms = 0;
    if (cudaEventElapsedTime(&ms, r.ev_a, r.ev_b) != cudaSuccess || ms <= 0) {
      cudaGetLastError();
      continue;
    }
    const double x = 1e-3 * ms / (double)r.last_k;
    r.spi = r.spi > 0 ? 0.5 * (r.spi + x) : x;
  }
  // packed completions
  for (auto& kv : by_group) {
    for (Req* rp : kv.second) {
      Req& r = *rp;
      if (r.ticket < 0) continue;
      BatchResultDev d;
      if (cudaMemcpy(&d, r.d_res, sizeof(d), cudaMemcpyDeviceToHost) != cudaSuccess) {
        finish(r, cuda_fail(cudaGetLastError(), "serve result"), nullptr);
        r.ticket = -1;
        continue;
      }
      if (!d.complete) continue;
      ts_result res;
      std::memset(&res, 0, sizeof(res));
      res.iterations = d.iterations;
      res.evaluations = d.evaluations;
      res.cur = d.cur;
      res.best = d.best;
      res.best_true = d.best_true;
      res.perturbations = d.perturbations;
      res.stopped = d.stopped;
      res.m = r.m;
      res.n = r.n;
      res.device_error = d.err;
      ts_status rc = d.err ? TS_ERR_DEVICE : TS_OK;
      if (r.best_sol)
        cudaMemcpy(r.best_sol, r.d_best, 4 * (size_t)(r.p.problem == P_MDP ? r.m : r.n), cudaMemcpyDeviceToHost);
      finish(r, rc, &res);
      r.ticket = -1;
    }
  }
  active.erase(std::remove_if(active.begin(), active.end(), [](const std::unique_ptr<Req>& r) { return r->ticket < 0; }),
               active.end());
  std::lock_guard<std::mutex> lk(mu);
  stats.rounds++;
}

void ts_server::run() {
  cudaSetDevice(device);
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(mu);
      if (active.empty() && queue.empty()) {
        if (busy_since >= 0) {
          stats.busy_s += now_s(t0) - busy_since;
          busy_since = -1;
        }
        if (stopping) return;
        cv_work.wait_for(lk, std::chrono::milliseconds(2));
        continue;
      }
      if (busy_since < 0) busy_since = now_s(t0);
    }
    admit();
    if (!active.empty()) round();
  }
}

extern "C" {

ts_status ts_server_create(const ts_server_opts* opts, ts_server** out) {
  if (!out) { set_error("ts_server_create: out is NULL"); return TS_ERR_INVALID_ARG; }
  *out = nullptr;
  int dev = 0;
  TS_CUDA(cudaGetDevice(&dev));
  std::unique_ptr<ts_server> s(new ts_server);
  s->device = dev;
  if (opts) s->opts = *opts;
  if (s->opts.round_ms <= 0) s->opts.round_ms = 5.0;
  if (s->opts.plain_min_pairs <= 0) s->opts.plain_min_pairs = 1LL << 20;
  TS_CUDA(cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, dev));
  TS_CUDA(cudaDeviceGetStreamPriorityRange(&s->prio_least, &s->prio_greatest));
  if (s->prio_least - s->prio_greatest + 1 > 8) s->prio_least = s->prio_greatest + 7;  // levels kept per request
  int64_t budget = s->opts.max_bytes;
  if (budget <= 0) {
    size_t fr = 0, tot = 0;
    TS_CUDA(cudaMemGetInfo(&fr, &tot));
    budget = (int64_t)(0.6 * (double)fr);
  }
  s->stats.bytes_budget = budget;
  ts_server* raw = s.release();
  raw->worker = std::thread([raw]() { raw->run(); });
  *out = raw;
  return TS_OK;
}

ts_status ts_server_submit(ts_server* s, const ts_request* q, int64_t* ticket) {
  tsb::TraceRange tr_("ts_server_submit");
  if (!s || !q || (q->num_edges > 0 && (!q->u || !q->v || !q->w)) || q->num_edges < 0) {
    set_error("ts_server_submit: bad arguments");
    return TS_ERR_INVALID_ARG;
  }
  const ts_params& p = q->params;
  const int32_t m = p.problem == TS_PROBLEM_MDP ? p.m : q->n / 2;
  if ((p.problem != TS_PROBLEM_MDP && p.problem != TS_PROBLEM_MAXBS) || q->n < 2 || m < 1 || m >= q->n ||
      p.max_iter < 0 || p.piter < 1 || p.gamma < 0 || p.maxt < 1 || p.tenure < 0 ||
      (p.tenure_policy != TS_TENURE_REF && p.tenure_policy != TS_TENURE_FIXED) || q->kind < -1 ||
      q->kind >= TS_STRUCT_COUNT) {
    set_error("ts_server_submit: bad parameters");
    return TS_ERR_INVALID_ARG;
  }
  std::unique_ptr<Req> r(new Req);
  r->n = q->n;
  r->m = m;
  r->kind = q->kind < 0 ? TS_STRUCT_CSR : q->kind;
  r->drop = q->drop_self_loops;
  r->p = p;
  r->p.trace = 0;
  r->u.assign(q->u, q->u + q->num_edges);
  r->v.assign(q->v, q->v + q->num_edges);
  r->w.assign(q->w, q->w + q->num_edges);
  if (q->initial) r->initial.assign(q->initial, q->initial + (p.problem == TS_PROBLEM_MDP ? m : q->n));
  r->best_sol = q->best_sol;
  r->P = (int64_t)m * (q->n - m);
  r->num_pert = std::max(1, std::min(p.gamma, q->n) / 2);
  r->plain = r->P >= s->opts.plain_min_pairs;
  r->cs = r->P < (1LL << 18) ? 1 : (r->P < (1LL << 19) ? 2 : 4);
  r->footprint = estimate_footprint(*r);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    r->ticket = s->next_ticket++;
    r->t_submit = now_s(s->t0);
    if (ticket) *ticket = r->ticket;
    s->queue.push_back(std::move(r));
    s->stats.submitted++;
    s->stats.queued++;
  }
  s->cv_work.notify_one();
  return TS_OK;
}

ts_status ts_server_poll(ts_server* s, ts_served* out, int32_t cap, int32_t* n_out, int32_t wait_ms) {
  tsb::TraceRange tr_("ts_server_poll");
  if (!s || (cap > 0 && !out)) { set_error("ts_server_poll: bad arguments"); return TS_ERR_INVALID_ARG; }
  std::unique_lock<std::mutex> lk(s->mu);
  if (s->done.empty() && wait_ms > 0)
    s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [s]() { return !s->done.empty(); });
  int32_t k = 0;
  while (k < cap && !s->done.empty()) {
    out[k++] = s->done.front();
    s->done.pop_front();
  }
  if (n_out) *n_out = k;
  return TS_OK;
}

ts_status ts_server_stats_get(ts_server* s, ts_server_stats* out) {
  if (!s || !out) { set_error("ts_server_stats_get: bad arguments"); return TS_ERR_INVALID_ARG; }
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  if (s->busy_since >= 0) out->busy_s += now_s(s->t0) - s->busy_since;
  return TS_OK;
}

double ts_server_now(const ts_server* s) { return s ? now_s(s->t0) : 0.0; }

ts_status ts_server_destroy(ts_server* s) {
  if (!s) return TS_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  delete s;
  return TS_OK;
}

}  // extern "C"
