/*
 * ts_b200.h -- C-ABI of the B200 tabu-search engine (MDP and Max Bisection).
 *
 * Plain C types only: pointers, sizes, status codes.  Every function returns a
 * ts_status; nothing throws or exits across this boundary (the reference's
 * gpuAssert exits the process instead, src/mdp/GPU-MDP-CSR.cu:65-73).
 * A handle is not thread-safe; use one per host thread.  All device work of a
 * handle runs on the CUDA stream it was created with.
 *
 * Reference interfaces replaced (paths relative to the reference project):
 *   graph loaders + structure builders
 *       read_instance/createCSR  src/mdp/GPU-MDP-CSR.cu:210-367
 *       load/createCSR           src/maxbisection/GPU-MAXBS-CSR.cu:112-173
 *       bitmap build             src/mdp/GPU-MDP-CSR-Bitset-BuscaBinaria.cu:321-378,
 *                                src/maxbisection/GPU-MAXBS-CSR-Bitset.cu:160-183
 *       hash build               src/mdp/GPU-MDP-Hash.cu:189-217,413-440,
 *                                src/maxbisection/GPU-MAXBS-Hash.cu:137-227
 *   edge lookup                  gpu_edge  src/mdp/GPU-MDP-CSR.cu:555-564,
 *                                src/mdp/GPU-MDP-CSR-BuscaBinaria.cu:554-566,
 *                                gpu_hashtable_edge src/mdp/GPU-MDP-Hash.cu:168-187,
 *                                hasEdge src/mdp/GPU-MDP-CSR-Bitset-BuscaBinaria.cu:584-586
 *   tabu engine                  tabu_search(int*)  src/mdp/GPU-MDP-CSR.cu:611-693
 *                                perturbationBasedTabuSearch
 *                                    src/maxbisection/GPU-MAXBS-CSR.cu:401-512
 */
#ifndef TS_B200_H
#define TS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TS_ABI_VERSION 1

typedef enum ts_status {
  TS_OK = 0,
  TS_ERR_INVALID_ARG = 1,   /* bad size, id out of range, unbalanced partition ... */
  TS_ERR_CUDA = 2,          /* a CUDA runtime call failed; see ts_last_error() */
  TS_ERR_OUT_OF_MEMORY = 3, /* device allocation failed */
  TS_ERR_UNSUPPORTED = 4,   /* combination not provided (e.g. value range) */
  TS_ERR_DEVICE = 5,        /* a kernel reported an error word (bounded wait expired, index check) */
  TS_ERR_STATE = 6,         /* call order violated (step before init, ...) */
  TS_ERR_NO_DEVICE = 7      /* no CUDA device visible */
} ts_status;

/* Weight-lookup structures; numbering follows the reference runner's table
 * src/run_experimentos.py:10-17 (csr, hash, wswap, csr-bitset, csr-bb, csr-bitset-bb). */
typedef enum ts_struct {
  TS_STRUCT_CSR = 0,
  TS_STRUCT_HASH = 1,
  TS_STRUCT_WSWAP = 2,
  TS_STRUCT_CSR_BITSET = 3,
  TS_STRUCT_CSR_BB = 4,
  TS_STRUCT_CSR_BITSET_BB = 5,
  TS_STRUCT_COUNT = 6
} ts_struct;

typedef enum ts_problem { TS_PROBLEM_MDP = 0, TS_PROBLEM_MAXBS = 1 } ts_problem;

/* TS_TENURE_REF: the reference schedules, determine_tabu_tenure
 * (src/mdp/GPU-MDP-CSR.cu:461-476, C2=round(0.7*C1) :663-664) and tabuTenure
 * (src/maxbisection/GPU-MAXBS-CSR.cu:248-263).  TS_TENURE_FIXED: MDP C1=tenure,
 * C2=round(0.7*tenure); MaxBS tt=tenure. */
typedef enum ts_tenure { TS_TENURE_REF = 0, TS_TENURE_FIXED = 1 } ts_tenure;

/* How an iteration sweeps the swap pairs; every choice gives the same moves.
 * TS_PASS_TILE: a tile of 32 inside positions builds a shared-memory index of
 *   its rows' adjacency from the structure and queries each outside position
 *   once for all 32 rows (32-bit keys only; 64-bit keys use TS_PASS_ROWS).
 * TS_PASS_ROWS: a few rows per tile, each pair looked up in its row's staged
 *   structure (fewer, cheaper tiles: small instances).
 * TS_PASS_AUTO: TILE from 2^22 swap pairs per iteration up (CSR with
 *   MDP or a negative weight: ROWS), else ROWS. */
typedef enum ts_pass { TS_PASS_AUTO = 0, TS_PASS_TILE = 1, TS_PASS_ROWS = 2 } ts_pass;

typedef struct ts_graph ts_graph;
typedef struct ts_solver ts_solver;

typedef struct ts_graph_info {
  int32_t n;
  int32_t kind;              /* ts_struct */
  int64_t num_edges;         /* undirected edges kept */
  int64_t num_entries;       /* CSR entries (2 per edge) */
  int64_t max_weighted_degree; /* max_z sum |w(z,.)| over CSR entries */
  int64_t device_bytes;      /* HBM held by the graph and its structure */
  int64_t hash_slots;        /* Hash: total slots of the per-vertex tables */
  int64_t bitset_words_per_row;
} ts_graph_info;

/* Launch geometry of a solver's iteration kernel (no counterpart in the
 * reference, whose kernels use one thread per pair): ts_solver_info. */
typedef struct ts_solver_info {
  int32_t grid;           /* CTAs per iteration launch (one tile each) */
  int32_t tile_rows;      /* inside positions per tile */
  int32_t chunk_cols;     /* outside positions per tile */
  int32_t n_chunks;       /* tiles per row block */
  int32_t threads;        /* threads per CTA */
  int32_t dyn_smem_bytes; /* dynamic shared memory per CTA */
  int32_t key_bytes;      /* 4: 32-bit pair keys and contributions, 8: 64-bit */
  int32_t w_bytes;        /* WSwap: bytes per matrix element (2 or 4); 0 otherwise */
  int32_t slices;         /* CTAs per tile (grid = row blocks x n_chunks x slices) */
  int32_t reserved[7];
} ts_solver_info;

typedef struct ts_params {
  int32_t problem;        /* ts_problem */
  int32_t m;              /* MDP: selected-set size; MaxBS: ignored (floor(n/2), GPU-MAXBS-CSR.cu:151) */
  int64_t max_iter;       /* iteration budget of the tabu loop (MDP reference: 50000, :55) */
  int32_t tenure_policy;  /* ts_tenure */
  int32_t tenure;         /* fixed tenure value */
  int32_t maxt;           /* MaxBS reference schedule parameter (default 200) */
  int32_t piter;          /* MaxBS non-improving iterations before perturbation (default 500) */
  int32_t gamma;          /* MaxBS perturbation strength (default 150) */
  uint32_t seed;          /* random start + perturbation stream */
  int32_t trace;          /* 1: keep a per-iteration trace on the device */
  int32_t pass;           /* pair sweep (ts_pass; no counterpart in the reference): 0 = by size */
  int32_t reserved[6];    /* zero */
} ts_params;

typedef struct ts_result {
  int64_t iterations;     /* tabu iterations applied */
  int64_t evaluations;    /* swap pairs evaluated, counted like the reference counters
                             (total_evaluations GPU-MDP-CSR.cu:648, avaliations_count GPU-MAXBS-CSR.cu:443) */
  int64_t cur;            /* current objective, reference bookkeeping (incl. MaxBS penalty recovery) */
  int64_t best;           /* best objective, same bookkeeping */
  int64_t best_true;      /* objective of the best solution recomputed from the graph */
  int64_t perturbations;  /* MaxBS perturbation moves applied */
  int32_t stopped;        /* MDP: the reference's all-tabu break (value == -INF, :657) happened */
  int32_t m;
  int32_t n;
  int32_t device_error;   /* device error word (0 = none) */
} ts_result;

typedef struct ts_trace_rec {
  int64_t iter;   /* iteration counter of the record */
  int64_t idx;    /* flat move index i*(n-m)+(j-m) */
  int64_t key;    /* reduced key: gain, MDP sentinel -99999, or MaxBS penalty key; PERTURB: applied gain */
  int64_t cur;    /* objective after the record */
  int64_t best;   /* best objective after the record */
  int32_t kind;   /* 0 move, 1 break, 2 perturbation move */
  int32_t tenure; /* MDP C1 / MaxBS tt */
  int32_t tenure2;/* MDP C2 */
  int32_t pad;
} ts_trace_rec;

/* ---------------------------------------------------------------- library */
int32_t ts_abi_version(void);
const char* ts_status_string(ts_status s);
/* Message of the last failing call on this host thread (never NULL). */
const char* ts_last_error(void);
/* CSV names "csr,hash,wswap,csr-bitset,csr-bb,csr-bitset-bb" -> ts_struct, -1 if unknown. */
int32_t ts_struct_from_name(const char* name);
const char* ts_struct_name(int32_t kind);

/* ---------------------------------------------------------------- graphs */
/* Builds the graph and its lookup structure on the current device from a HOST
 * edge list (0-based endpoints).  drop_self_loops=1 is the MDP loader rule
 * (GPU-MDP-CSR.cu:340), 0 the MaxBS one (GPU-MAXBS-CSR.cu:160-166).  Rows are
 * kept sorted by neighbour id (stable for duplicate edges); contributions sum
 * every entry and lookups return the first entry of a duplicated pair.
 * `stream` is a cudaStream_t (NULL: the legacy default stream). */
ts_status ts_graph_create(int32_t n, int64_t num_edges, const int32_t* u, const int32_t* v,
                          const int32_t* w, int32_t kind, int32_t drop_self_loops,
                          void* stream, ts_graph** out);
/* Same, from DEVICE arrays already resident in HBM. */
ts_status ts_graph_create_device(int32_t n, int64_t num_edges, const int32_t* d_u,
                                 const int32_t* d_v, const int32_t* d_w, int32_t kind,
                                 int32_t drop_self_loops, void* stream, ts_graph** out);
ts_status ts_graph_info_get(const ts_graph* g, ts_graph_info* out);
ts_status ts_graph_destroy(ts_graph* g);

/* The one lookup interface over all structures: w_out[k] = w(u[k], v[k]),
 * 0 when not adjacent.  Device arrays; runs on the graph's stream. */
ts_status ts_lookup(const ts_graph* g, int64_t count, const int32_t* d_u, const int32_t* d_v,
                    int32_t* d_w_out);
/* Same with host arrays (copies in/out, synchronous). */
ts_status ts_lookup_host(const ts_graph* g, int64_t count, const int32_t* u, const int32_t* v,
                         int32_t* w_out);

/* ---------------------------------------------------------------- solver */
ts_status ts_params_default(int32_t problem, ts_params* out);
/* One tabu-search state bound to a graph.  The structure used for w(u,v) is
 * the graph's kind. */
ts_status ts_solver_create(ts_graph* g, const ts_params* p, ts_solver** out);
/* Starting point of tabu_search / perturbationBasedTabuSearch.
 *   initial == NULL: the reference's seeded random start -- MDP: srand(seed),
 *     rand()%n rejection (GPU-MDP-CSR.cu:773-784, :1248); MaxBS: mt19937(seed),
 *     shuffle (GPU-MAXBS-CSR.cu:187-195, :682) -- and the perturbation stream
 *     continues that generator.
 *   MDP:   initial = m distinct vertex ids (host).
 *   MaxBS: initial = part[n] in {0,1}, exactly floor(n/2) zeros (host); the
 *     perturbation stream is mt19937(seed) from its start. */
ts_status ts_solver_init(ts_solver* s, const int32_t* initial);
/* MaxBS: after ts_solver_init and before the first step, replaces the
 * perturbation stream with the caller's n_events events of
 * k = max(1, min(gamma, n)/2) flat move indices each (host, copied).  For
 * drivers that keep one generator across many searches, as MACUT does: its
 * perturbationBasedTabuSearch draws from the program-wide mt19937
 * (src/maxbisection/GPU-MAXBS-CSR.cu:481-492, seeded once at :682).  A search
 * that needs more events than given stops with TS_ERR_DEVICE; the events it
 * used are ts_result.perturbations / k. */
ts_status ts_solver_set_perturbations(ts_solver* s, const int64_t* draws, int64_t n_events);
/* Runs up to k more iterations on the device (no host round trip per
 * iteration).  Stops early at max_iter or at the MDP all-tabu break.
 * Blocks until they are done; *done_iters (may be NULL) = iterations applied
 * by this call. */
ts_status ts_solver_step(ts_solver* s, int64_t k, int64_t* done_iters);
/* Asynchronous stepping, for callers that overlap work or bracket iterations
 * with their own CUDA events:
 *   ts_solver_prepare(s, k, &adm)  synchronises, admits adm <= k iterations
 *       (bounded by max_iter; MaxBS also by its staged perturbation draws,
 *       about 62*piter per call) and stages what they need;
 *   ts_solver_enqueue(s, j)        puts j iteration launches on the solver's
 *       stream and returns at once; launches past the admitted target do nothing;
 *   ts_solver_sync(s, &iter)       waits, completes the admitted iterations if
 *       exact re-evaluation passes consumed launches, checks the device error
 *       word; iter = iteration counter. */
ts_status ts_solver_prepare(ts_solver* s, int64_t k, int64_t* prepared);
ts_status ts_solver_enqueue(ts_solver* s, int64_t k);
ts_status ts_solver_sync(ts_solver* s, int64_t* iter);
/* best_sol (host, may be NULL): MDP m vertex ids of the best set in position
 * order; MaxBS part[n] of the best bisection. */
ts_status ts_solver_result(ts_solver* s, ts_result* out, int32_t* best_sol);
/* Current state (host arrays, each may be NULL): sol[n] in position order,
 * pos[n], tab[n] tabu expiry per vertex, vg[n] contribution per vertex. */
ts_status ts_solver_state(ts_solver* s, int32_t* sol, int32_t* pos, int32_t* tab, int64_t* vg);
/* Copies up to cap trace records (params.trace=1). */
ts_status ts_solver_trace(ts_solver* s, ts_trace_rec* out, int64_t cap, int64_t* n_out);
/* Launch geometry and element widths the solver picked (ts_solver_info). */
ts_status ts_solver_info_get(const ts_solver* s, ts_solver_info* out);
ts_status ts_solver_destroy(ts_solver* s);

/* ---------------------------------------------------------------- host helpers
 * No GPU needed.  The reference-compatible random starts and the MaxBS
 * perturbation stream, exactly as ts_solver_init(s, NULL) draws them. */
/* MDP: out[m] = the ids drawn by srand(seed); rand()%n rejection
 * (GPU-MDP-CSR.cu:773-784).  MaxBS: out[n] = part[] of mt19937(seed) +
 * shuffle(iota) (GPU-MAXBS-CSR.cu:187-195); m is ignored. */
ts_status ts_random_start(int32_t problem, int32_t n, int32_t m, uint32_t seed, int32_t* out);
/* MaxBS perturbation draws (GPU-MAXBS-CSR.cu:481-492): n_events events of
 * k = max(1, min(gamma, n)/2) distinct flat move indices each, from
 * mt19937(seed) after the shuffle when init_random != 0. out[n_events*k]. */
ts_status ts_perturb_draws(int32_t n, uint32_t seed, int32_t gamma, int32_t init_random,
                           int32_t n_events, int64_t* out);

/* ---------------------------------------------------------------- batched form
 * Many independent solves (instances, restarts) in one persistent launch per
 * (problem, structure, key width, CTAs per solve) group, recorded once as a
 * CUDA graph and replayed.  Stands in for the reference's one-at-a-time
 * restart loops around tabu_search / perturbationBasedTabuSearch (OBMA
 * src/mdp/GPU-MDP-CSR.cu:754-903,1146-1208; MACUT
 * src/maxbisection/GPU-MAXBS-CSR.cu:523-577,679-732).  Every solve gives the
 * same result as ts_solver_create + ts_solver_init(initial) +
 * ts_solver_step(max_iter) on its graph and parameters. */
typedef struct ts_batch ts_batch;

typedef struct ts_batch_job {
  const ts_graph* graph;    /* all graphs of one batch on one device */
  ts_params params;         /* params.trace is ignored (no trace in batches) */
  const int32_t* initial;   /* host, as ts_solver_init; NULL: seeded random start */
  int32_t cluster;          /* CTAs per solve (a thread-block cluster): 0 auto, or 1, 2, 4, 8 */
  int32_t reserved[3];      /* zero */
} ts_batch_job;

typedef struct ts_batch_opts {
  int64_t max_bytes;        /* HBM budget for solver slots; 0: 60% of free memory */
  int32_t max_slots;        /* cap on concurrent solves per group; 0: as many as are resident */
  int32_t reserved[5];      /* zero */
} ts_batch_opts;

typedef struct ts_batch_info {
  int32_t jobs;
  int32_t groups;           /* launches in the captured graph */
  int64_t slots;            /* concurrent solves, all groups */
  int64_t slot_bytes;       /* HBM held for solver slots */
  int64_t input_bytes;      /* HBM held for starts, draws, job table, results */
  int64_t best_sol_words;   /* int32 words of the packed best solutions */
} ts_batch_info;

/* Prepares a batch: draws the seeded starts and MaxBS perturbation streams on
 * host threads, copies them and the job table to the device, sizes solver
 * slots within the budget and captures the launches as a CUDA graph on
 * `stream` (a cudaStream_t; NULL: a stream of the library's own).  The graphs
 * must outlive the batch. */
ts_status ts_batch_create(const ts_batch_job* jobs, int32_t count, const ts_batch_opts* opts,
                          void* stream, ts_batch** out);
/* Replays the captured graph on the batch's stream (asynchronous); every
 * replay recomputes all solves from their starts. */
ts_status ts_batch_launch(ts_batch* b);
ts_status ts_batch_sync(ts_batch* b);
/* out[count] (may be NULL); best_sols (host, may be NULL) receives the best
 * solutions packed in job order: MDP m ids in position order, MaxBS part[n]. */
ts_status ts_batch_results(ts_batch* b, ts_result* out, int32_t* best_sols);
ts_status ts_batch_info_get(const ts_batch* b, ts_batch_info* out);
ts_status ts_batch_destroy(ts_batch* b);
/* create + launch + sync + results + destroy. */
ts_status ts_batch_run(const ts_batch_job* jobs, int32_t count, const ts_batch_opts* opts,
                       ts_result* out, int32_t* best_sols);

/* ---------------------------------------------------------------- served form
 * A request loop with continuous batching.  Requests (a host edge list plus
 * solve parameters) are admitted while their estimated HBM footprint fits the
 * budget; the server builds each graph on the device, keeps graph and tabu
 * state resident, and advances every admitted solve a bounded number of
 * iterations per round: small solves as clusters of one persistent launch
 * (the batched form's kernel), large ones with the plain one-launch-per-
 * iteration kernel on their own stream, all overlapping on the GPU.  Requests
 * that arrive meanwhile join at the next round.  A solve's result does not
 * depend on what else runs: it equals ts_solver_* on the same graph and
 * parameters.  No counterpart in the reference, which runs one search per
 * process (src/run_experimentos.py:101-117). */
typedef struct ts_server ts_server;

typedef struct ts_request {
  int32_t n;
  int64_t num_edges;
  const int32_t* u;          /* host, copied by ts_server_submit */
  const int32_t* v;
  const int32_t* w;
  int32_t kind;              /* ts_struct, or -1: the server's choice by size */
  int32_t drop_self_loops;
  ts_params params;
  const int32_t* initial;    /* host, copied; NULL: seeded random start */
  int32_t* best_sol;         /* host, may be NULL; written before completion is reported;
                                MDP m ids, MaxBS part[n]; must stay valid until then */
} ts_request;

typedef struct ts_server_opts {
  int64_t max_bytes;         /* HBM budget for admitted requests; 0: 60% of free memory */
  double round_ms;           /* shortest round (rounds stretch to the last one's length, up to 50 ms); 0: 5 ms */
  int64_t plain_min_pairs;   /* pairs per iteration from which a solve runs plain; 0: 2^20 */
  int32_t reserved[8];
} ts_server_opts;

typedef struct ts_served {
  int64_t ticket;
  int32_t status;            /* ts_status of the request */
  int32_t executor;          /* 0 packed (cluster of a persistent launch), 1 plain */
  int32_t kind;              /* structure used */
  int32_t pad;
  ts_result result;
  double submit_s, admit_s, done_s;   /* server clock, seconds */
  int64_t footprint_bytes;
} ts_served;

typedef struct ts_server_stats {
  int64_t submitted, admitted, completed, queued, active;
  int64_t rounds;
  int64_t bytes_in_use, bytes_budget;
  double busy_s;             /* time with at least one admitted request */
} ts_server_stats;

/* Starts the scheduler thread on the current device. */
ts_status ts_server_create(const ts_server_opts* opts, ts_server** out);
/* Queues a request (copies its arrays); *ticket identifies it. */
ts_status ts_server_submit(ts_server* s, const ts_request* req, int64_t* ticket);
/* Copies up to cap completed requests to out (oldest first), waiting up to
 * wait_ms for the first one; *n_out = records copied. */
ts_status ts_server_poll(ts_server* s, ts_served* out, int32_t cap, int32_t* n_out, int32_t wait_ms);
ts_status ts_server_stats_get(ts_server* s, ts_server_stats* out);
/* Seconds on the server clock (the clock of submit_s / admit_s / done_s). */
double ts_server_now(const ts_server* s);
/* Stops the scheduler after the admitted and queued requests complete. */
ts_status ts_server_destroy(ts_server* s);

/* ---------------------------------------------------------------- no allocation
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory -- plugins whose host application owns all of HBM through its own
 * pool, services held to a fixed device-memory budget.  From a tabu state the
 * caller keeps in its own device buffers, evaluates every swap of one
 * iteration with the reference's key rule and ArgMax tie rule and writes the
 * decision; it allocates nothing, using a fixed scratch array compiled into
 * the library (about 3 MiB, held on every GPU that loads the library until
 * exit).
 *   d_rowptr int64[n+1], d_col / d_w int32[entries]: CSR rows sorted by
 *     neighbour id (the first entry of a duplicated pair is the one used);
 *   d_sol int32[n]: vertex at each position, the inside set at [0, m);
 *   d_vg int64[n], d_tab int32[n]: contribution and tabu expiry per vertex;
 *   iter, cur, best: iteration counter and objective bookkeeping;
 *   d_out int64[2]: {key, flat index i*(n-m)+(j-m)} of the chosen swap.
 * n above TS_NOALLOC_MAX_N is rejected (TS_ERR_INVALID_ARG).  Work runs on
 * `stream` without synchronising, in the CUDA context current on the calling
 * thread (the device's primary context if none is).  The first call in each
 * context looks the scratch address up.  All calls share the scratch, so calls that overlap on the GPU
 * (other streams or host threads) race on it.  Cost: one binary search of a
 * global CSR row per pair, roughly P / 1e10 s for P = m*(n-m) pairs. */
#define TS_NOALLOC_MAX_N 262144
ts_status ts_best_swap_noalloc(int32_t problem, int32_t n, int32_t m, int64_t iter, int64_t cur,
                               int64_t best, const int64_t* d_rowptr, const int32_t* d_col,
                               const int32_t* d_w, const int32_t* d_sol, const int64_t* d_vg,
                               const int32_t* d_tab, int64_t* d_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* TS_B200_H */
