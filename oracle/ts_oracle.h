/*
 * ts_oracle.h -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * CPU restatement of the reference's tabu-search hot path, used only by
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference leg
 * as the checker and the timed CPU baseline.  The product library never links,
 * loads or calls anything here.
 *
 * It restates, in exact int64 arithmetic, the control flow of
 *   MDP  : src/mdp/GPU-MDP-CSR.cu            tabu_search            :611-693
 *          (kernels :523-584, tenure :461-476, init :479-519)
 *   MaxBS: src/maxbisection/GPU-MAXBS-CSR.cu perturbationBasedTabuSearch :401-512
 *          (kernels :337-399, tenure :248-263, init :197-219,:307-324)
 * including the CUB ArgMax tie rule (lowest flat index wins,
 * cub/thread/thread_operators.cuh:103-121), the MDP -99999 sentinel/break and
 * the MaxBS float-quantised penalty key fl32(double(-9999999999)+g) with its
 * "value < INF/4" recovery.  The reference keeps every sum in float, which is
 * exact while all magnitudes stay below 2^24; the oracle's integers agree with
 * it there and define the semantics beyond it.
 */
#ifndef TS_ORACLE_H
#define TS_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_graph or_graph;

/* Undirected edge list (0-based).  drop_self_loops=1 follows the MDP loader
 * (GPU-MDP-CSR.cu:340), 0 the MaxBS loader (GPU-MAXBS-CSR.cu:156-166).
 * Rows are sorted by neighbour id, stable in input order; a lookup returns the
 * first entry of a duplicated pair, contributions sum every entry. */
or_graph* or_graph_create(int32_t n, int64_t num_edges, const int32_t* u,
                          const int32_t* v, const int32_t* w, int drop_self_loops);
void or_graph_destroy(or_graph* g);
int64_t or_graph_num_entries(const or_graph* g);
int32_t or_lookup(const or_graph* g, int32_t u, int32_t v);

/* glibc srand(seed); rand()%n rejection draw of m distinct ids, the first
 * solution of build_pool_with_OBL (GPU-MDP-CSR.cu:773-784, seed :1248). */
void or_mdp_random_initial(int32_t n, int32_t m, uint32_t seed, int32_t* sol_out);
/* mt19937(seed); shuffle(iota); part[first n/2]=0 (GPU-MAXBS-CSR.cu:187-195). */
void or_maxbs_random_partition(int32_t n, uint32_t seed, int32_t* part_out);

enum { OR_MDP = 0, OR_MAXBS = 1 };
enum { OR_TENURE_REF = 0, OR_TENURE_FIXED = 1 };
enum { OR_INIT_EXPLICIT = 0, OR_INIT_RANDOM = 1 };

typedef struct {
  int32_t problem;        /* OR_MDP / OR_MAXBS */
  int32_t m;              /* MDP: selected-set size; MaxBS: ignored (n/2) */
  int64_t max_iter;
  int32_t tenure_policy;  /* OR_TENURE_REF / OR_TENURE_FIXED */
  int32_t tenure_fixed;   /* MDP: C1 (C2=round(0.7*C1)); MaxBS: tt */
  int32_t maxt;           /* MaxBS reference schedule parameter */
  int32_t piter;          /* MaxBS perturbation trigger */
  int32_t gamma;          /* MaxBS perturbation strength */
  uint32_t seed;
  int32_t init_mode;      /* OR_INIT_EXPLICIT / OR_INIT_RANDOM */
  int32_t threads;        /* OpenMP threads for the pair sweep (<=0: all) */
} or_params;

enum { OR_REC_MOVE = 0, OR_REC_BREAK = 1, OR_REC_PERTURB = 2 };

typedef struct {
  int64_t iter;     /* iteration counter when the record was produced */
  int64_t idx;      /* flat move index i*(n-m)+(j-m) */
  int64_t key;      /* reduced key (gain, MDP sentinel or MaxBS penalty key); PERTURB: applied gain */
  int64_t cur;      /* objective after the record */
  int64_t best;     /* best objective after the record */
  int32_t kind;     /* OR_REC_* */
  int32_t tenure;   /* MDP: C1; MaxBS: tt; PERTURB: 0 */
  int32_t tenure2;  /* MDP: C2; else 0 */
  int32_t pad;
} or_trace_rec;

typedef struct {
  int64_t iterations;      /* tabu iterations applied */
  int64_t evaluations;     /* pairs evaluated, counted like the reference */
  int64_t cur;
  int64_t best;
  int64_t best_true;       /* objective of the best solution recomputed from scratch */
  int64_t n_trace;
  int32_t stopped;         /* MDP sentinel break */
  int32_t pad;
} or_result;

/* initial: MDP -> m vertex ids (explicit mode); MaxBS -> part[n] in {0,1}.
 * out_* buffers may be NULL.  out_sol/out_pos/out_tab/out_vg are the final
 * current state (position order / vertex order); out_best_sol is the best
 * solution in position order (MDP: first m entries; MaxBS: n entries). */
int or_run(const or_graph* g, const or_params* p, const int32_t* initial,
           or_result* res, or_trace_rec* trace, int64_t trace_cap,
           int32_t* out_sol, int32_t* out_pos, int32_t* out_tab, int64_t* out_vg,
           int32_t* out_best_sol);

/* Bounded CPU-baseline sample: from the start state of `p` (initial or the
 * seeded random start), runs `sweeps` argmax sweeps restricted to the first
 * `rows` inside positions (rows <= m) with `threads` OpenMP threads and
 * returns the wall seconds spent in the sweeps; *pairs = pairs evaluated.
 * The per-pair work is the full loop's. */
double or_sweep_sample(const or_graph* g, const or_params* p, const int32_t* initial,
                       int32_t rows, int32_t sweeps, int64_t* pairs, int64_t* last_key,
                       int64_t* last_idx);

/* Reference tenure schedules, exported for known-answer tests. */
int32_t or_mdp_tenure(int64_t iter);                  /* GPU-MDP-CSR.cu:461-476 */
int32_t or_mdp_c2(int32_t c1);                        /* round(0.7*C1) :664 */
int32_t or_maxbs_tenure(int64_t iter, int32_t maxt);  /* GPU-MAXBS-CSR.cu:248-263 */
int64_t or_round_f32(int64_t x);                      /* nearest-even to 24 bits */
int64_t or_maxbs_penalty(int64_t g);                  /* fl32(-9999999999+g) */

/* Perturbation draw stream (MaxBS): the flat move indices the reference's
 * randInt/unordered_set dedupe (GPU-MAXBS-CSR.cu:480-492) produces after the
 * optional shuffle, for n_events events of k distinct draws each. */
void or_maxbs_perturb_draws(int32_t n, uint32_t seed, int32_t init_random,
                            int32_t n_events, int32_t k, int64_t* out);

#ifdef __cplusplus
}
#endif
#endif
