/*
 * maxflow_b200.h — C ABI of the B200 exact max-flow engine.
 *
 * Drop-in boundary for the per-query solve of the Region-Aware push-relabel
 * program (reference project file Region_Aware_PR_with_Pruning_BoundaryCore.cu,
 * "RA" below).  The reference has no library API: its in-process seam is
 *   init_global_graph_on_device(CSRGraph&, R, region_start, region_end, region_id)  RA:1293
 *   init_state_for_st(DynamicState&, V, E, R)                                      RA:1336
 *   flow_t run_gpu_static_with_state(int s, int t, DynamicState&)                  RA:2119
 *   free_state_for_st(DynamicState&)                                               RA:86
 * and its outer boundary is the CLI  prog <input_dir> <output_dir> [static|dynamic]
 * (RA:2561-2570) reading graph.txt / test.txt and writing res_mt.txt.
 * The entry points below replace that seam; the CLI maxflow_b200 is built on
 * them.
 *
 * Conventions: every function returns an int status (MF_OK = 0, else an
 * MF_ERR_* code; mf_last_error_string() describes the last failure on the
 * calling thread).  No exceptions cross the ABI.  The caller owns every host
 * buffer; the engine owns device memory.  Vertex ids at this ABI are 0-based
 * ids of the caller's graph (the engine's internal region order is hidden).
 * Flows and capacities are int64 and exact.  A graph handle may be used by
 * one thread at a time.
 */
#ifndef MAXFLOW_B200_H
#define MAXFLOW_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MF_OK 0
#define MF_ERR_ARG 1          /* invalid argument */
#define MF_ERR_CUDA 2         /* CUDA runtime error (no device, launch failure, ...) */
#define MF_ERR_NOMEM 3        /* device or host allocation failed / admission refused */
#define MF_ERR_IO 4           /* file missing or malformed header */
#define MF_ERR_ITER_LIMIT 5   /* a solve exceeded opts.iter_max rounds */
#define MF_ERR_TIMEOUT 6      /* a device wait exceeded its time limit */
#define MF_ERR_INEXACT 7      /* internal consistency check failed */
#define MF_ERR_CERTIFY 8      /* certificate check failed */

typedef struct mf_graph mf_graph;

/* Solver options.  mf_opts_default() fills the defaults; fields mirror the
 * reference's knobs (RA:1459-1484, RA:1936, RA:2644-2648). */
typedef struct mf_opts {
    int kernel_cycles;     /* K: discharge cycles per active vertex per round (RA:1467 uses max(4, avg
                              degree) with one push per cycle; each cycle here pushes to every
                              downhill arc); 0 = 8 */
    int gr_freq;           /* rounds between global relabels at most (default 16; RA:1466 uses 128) */
    double gr_work_alpha;  /* also relabel once scanned arcs exceed alpha x mask arcs (0 = off) */
    int prune_mode;        /* 0: RA:1391-1445 mask (fwd(s) & undirected comp(t)); 1: fwd(s) & bwd(t) (default);
                              2: no prune, every vertex kept (graphs whose terminals touch most vertices) */
    int path_push_switch;  /* active count at or below which path-push starts (RA:1480) */
    int max_path_len;      /* path-push hop limit (RA:1481) */
    int use_path_push;     /* 1 = enable sparse-phase path push (RA:1765-1831) */
    int use_hot_sweep;     /* 1 = enable hot-region extra sweep (RA:1899-1984) */
    int hot_regions;       /* top-K regions for the hot sweep (RA:1936) */
    int use_rm;            /* 1 = enable region-aware invalid-arc repair (RA:1991-2097) */
    int rm_freq;           /* initial RM frequency (RM_FREQ0, RA:1468) */
    int h_cut;             /* height threshold for "high" active vertices (RA:1470) */
    int stagnate_rounds;   /* stagnation window (RA:1472) */
    int force_rm;          /* tests: run RM every rm_freq rounds regardless of frac_high */
    int force_path_push;   /* tests: use path push whenever active <= path_push_switch */
    long long iter_max;    /* round cap per solve (RA:1476) */
    int group_ctas;        /* CTAs per query group in batched solves (0 = 8) */
    int threads;           /* threads per CTA: a multiple of 32 in [64, 512] (0 = 512) */
    int certify;           /* 1 = return excess to the source and check the certificate */
    int verbose;           /* 1 = per-query log lines on stderr */
    int use_kept_cache;    /* 1 = queries with s and t in the graph's cached strongly connected
                              component take it as their kept set (prune_mode 1 only) */
    int schedule;          /* batched solves: 1 = start the queries expected to cost most first
                              (s and t in the cached component, then larger min(deg s, deg t));
                              0 = input order.  Results are in input order either way. */
    int relabel_early_stop; /* 1 = a global relabel's search ends once every active vertex has its
                               exact height (vertices it did not reach stay at height n until the
                               next relabel; a search that cannot reach every active vertex runs to
                               the end, so the relabel that ends a solve is exact) */
    int local_relabel;     /* k > 0: after every k-th discharge round between global relabels, when
                              the round's active heights span at most 128 levels, relabel the regions
                              holding active vertices by a depth-bounded search (RA:1583-1720;
                              heights only rise; RM is off while it is on); 0 = off (default) */
} mf_opts;

/* Per-query statistics (all counts exact device counters). */
typedef struct mf_stats {
    long long flow;
    int status;               /* MF_OK or MF_ERR_* for this query */
    int mask_vertices;        /* vertices kept by the prune */
    long long mask_arcs;      /* arcs out of kept vertices */
    long long rounds;         /* discharge rounds */
    long long global_relabels;
    long long arcs_examined;  /* residual-arc examinations (16 B each, algorithmic) */
    long long vertices_examined; /* vertex examinations (16 B each, algorithmic) */
    long long pushes;
    long long rm_fixed;       /* arcs repaired by RM */
    long long path_push_rounds;
    long long hot_sweeps;
    long long deficit_phases; /* times the solver drained deficits back to the sink */
    long long cut_capacity;   /* certify only: capacity of the residual s-t cut */
    double time_ms;           /* device time of the launch (single-query calls) */
    double service_ms;        /* device time from the query's start to its answer */
    double finish_ms;         /* batched calls: device time from the launch's first
                                 query start to this query's answer */
    double prune_ms;          /* device time in prune + init + preflow */
    double relabel_ms;        /* device time in global relabels */
    double rounds_ms;         /* device time in discharge rounds */
    long long relabel_arcs;   /* arc examinations inside global relabels */
    long long hub_arcs;       /* arc examinations by the chunked discharge of hubs */
    long long hub_passes;     /* hub discharge passes */
    long long hub_relabels;   /* hub passes that ended in a relabel (excess left) */
    long long levels;         /* search levels (prune, global relabels, certificate) */
    long long levels_bottom_up; /* of which bottom-up */
    long long levels_solo;    /* of which run by a single CTA */
    long long local_relabels; /* local relabels (mf_opts.local_relabel) */
} mf_stats;

void mf_opts_default(mf_opts *o);
const char *mf_last_error_string(void);
const char *mf_version(void);

/* ---- graphs ---------------------------------------------------------- */

/* Build a graph from 0-based edge arrays with the reference's reader rules
 * (RA:1068-1089): edges with an endpoint outside [0,n), u == v or cap <= 0
 * are dropped; each kept edge gives a forward arc and a zero-capacity
 * reverse arc.  The CSR is partitioned into R regions by capacity-degree
 * score and renumbered region-contiguously on the device (RA:1130-1276);
 * R = 0 means 128 (RA:2583), and R is clamped to [1, n]. */
int mf_graph_create_from_edges(int n, long long m, const int32_t *u, const int32_t *v,
                               const int64_t *cap, int R, mf_graph **out);
/* Same from edge arrays already in device memory (d_u, d_v, d_cap: device
 * pointers of m entries each; read only, the caller keeps them). */
int mf_graph_create_from_device_edges(int n, long long m, const int32_t *d_u, const int32_t *d_v,
                                      const int64_t *d_cap, int R, mf_graph **out);
/* Same, reading <path> in graph.txt format (1-based ids; replaces
 * build_graph, RA:1044-1126).  The file's bytes are copied to the device and
 * tokenised there with fscanf's rules (an "n m" header, then up to m
 * "u v cap" triples, stopping at the first triple that does not scan,
 * RA:1068-1075); the CSR is built on the device in the host build's arc
 * order.  MF_ERR_IO if the file cannot be read or has no "n m" header with
 * n > 0, m >= 0. */
int mf_graph_load_file(const char *path, int R, mf_graph **out);
/* Binary CSR cache: mf_graph_save writes the region-ordered graph and its
 * maps; mf_graph_load_binary restores it without parsing, building or
 * partitioning (checked for consistency on the device; MF_ERR_IO for a file
 * that is not a cache of this library, truncated or inconsistent).  The
 * loaded graph equals the saved one array for array. */
int mf_graph_save(const mf_graph *g, const char *path);
int mf_graph_load_binary(const char *path, mf_graph **out);
int mf_graph_destroy(mf_graph *g);
/* n, kept arcs (2 x kept edges), R. */
int mf_graph_info(const mf_graph *g, int *n, long long *arcs, int *R);
/* Copy the region-ordered CSR and the maps back to the host (any pointer may
 * be NULL).  new_id[old] = region-ordered id; region_start has R+1 entries. */
int mf_graph_export(const mf_graph *g, int32_t *row, int32_t *col, int64_t *cap, int32_t *rev,
                    int32_t *new_id, int32_t *region_start, double *score, int32_t *part);
/* Repartition the graph into R regions (rebuilds the region-ordered CSR). */
int mf_graph_repartition(mf_graph *g, int R);
/* Strongly connected components of the graph's edges with capacity > 0 (as
 * they stand after any capacity updates), computed on the device by
 * trimming, a forward-backward search from the highest-degree vertex and
 * colour propagation.  Replaces the offline Kosaraju tool
 * SCC_CONTRACT/scc_contract.cpp:43-96: the same partition, but components
 * are numbered 0 .. ncomp-1 in the order of their smallest vertex id (the
 * tool numbers them in its depth-first discovery order).  comp (n entries,
 * caller ids; may be NULL): component of each vertex.  m_contracted: arcs
 * of the contracted graph, read with mf_graph_scc_contracted.  Not while a
 * server changes this graph's capacities. */
int mf_graph_scc(mf_graph *g, int32_t *comp, int32_t *ncomp, long long *m_contracted);
/* The contracted graph of the last mf_graph_scc on g (scc_contract.cpp:
 * 98-128): one arc per ordered pair of distinct components joined by an
 * edge, its capacity the sum of theirs, in increasing (cu, cv).  max: room
 * in each array; MF_ERR_ARG when it is too small or mf_graph_scc has not
 * run. */
int mf_graph_scc_contracted(const mf_graph *g, int32_t *cu, int32_t *cv, int64_t *cap, long long max);

/* ---- solves ----------------------------------------------------------- */

/* One (s,t) solve on the whole GPU (replaces run_gpu_static_with_state,
 * RA:2119, plus the per-query prune of RA:2666-2698).  Invalid ids or s == t
 * give flow 0 and MF_OK (RA:2659-2663).  opts/stats may be NULL. */
int mf_solve(mf_graph *g, int32_t s, int32_t t, const mf_opts *opts, int64_t *flow,
             mf_stats *stats);
/* nq independent solves in one persistent launch: query groups of CTAs pull
 * queries from a device queue, each with its own residual slot.  flows[i]
 * (and stats[i], if stats != NULL) for query i. */
int mf_solve_batch(mf_graph *g, int nq, const int32_t *s, const int32_t *t, const mf_opts *opts,
                   int64_t *flows, mf_stats *stats);
/* nq solves in one launch, each on the graph with its own capacities for a
 * fixed set of narcs forward arcs u[j] -> v[j] (caller ids): query i runs
 * with capacity caps[i * narcs + j] on arc j, every other arc keeps the
 * graph's capacity.  Every (u[j], v[j]) must name an arc of the graph and
 * 0 <= caps[i * narcs + j] <= its capacity (MF_ERR_ARG otherwise): the graph
 * is built with the largest capacity each overridden arc takes, so each
 * query's prune stays a superset of its own.  A query batch of terminal
 * sets on one segmentation grid (terminal arcs to both super terminals at
 * the largest weight, each query zeroing or lowering them) replaces one run
 * of the reference per input directory (RA:2561-2570) when only those
 * capacities differ.  opts->certify is rejected (the cut check reads the
 * graph's capacities).  narcs == 0 is mf_solve_batch. */
int mf_solve_batch_override(mf_graph *g, int nq, const int32_t *s, const int32_t *t, long long narcs,
                            const int32_t *u, const int32_t *v, const int64_t *caps,
                            const mf_opts *opts, int64_t *flows, mf_stats *stats);
/* Device time (ms) of the last mf_solve_batch / mf_solve call on g. */
double mf_last_device_ms(const mf_graph *g);

/* Debug/parity views of single phases (0-based caller ids):
 * prune mask for (s,t) under opts->prune_mode (mask: n bytes, caller order);
 * exact residual heights after the initial preflow (heights: n ints, caller
 * order; unreachable = n). */
int mf_debug_prune_mask(mf_graph *g, int32_t s, int32_t t, const mf_opts *opts, uint8_t *mask,
                        int *kept);
int mf_debug_initial_heights(mf_graph *g, int32_t s, int32_t t, const mf_opts *opts,
                             int32_t *heights);
/* Allocation accounting and failure injection, for tests of the failure
 * paths (no counterpart in the reference, whose allocations are unchecked,
 * RA:1336-1372).  Every device and pinned-host allocation the engine makes
 * goes through one wrapper.  mf_debug_alloc_fail_after(k): the k-th next
 * allocation (0 = the next one) reports out-of-memory without allocating;
 * k < 0 disarms it.  mf_debug_alloc_live: allocations and bytes the engine
 * holds now, and the armed countdown (-1 = none); any pointer may be NULL. */
int mf_debug_alloc_fail_after(long long k);
int mf_debug_alloc_live(long long *count, long long *bytes, long long *fail_after);

/* Solve and copy the final residual capacities back (arcs in region order,
 * matching mf_graph_export's CSR). */
int mf_solve_residual(mf_graph *g, int32_t s, int32_t t, const mf_opts *opts, int64_t *flow,
                      int64_t *res, mf_stats *stats);

/* Solve (s,t), return the excess to the source (phase 2), and check on the
 * device: residuals non-negative and pairwise conserved, zero excess at every
 * vertex other than s and t, and a residual s-t cut whose capacity equals
 * the flow.  MF_OK only when every check passes; stats->cut_capacity. */
int mf_certify(mf_graph *g, int32_t s, int32_t t, const mf_opts *opts, int64_t *flow,
               mf_stats *stats);

/* Allocation-free solve.  No counterpart in the reference (its every solve
 * allocates per-query state, RA:1336-1372).  For callers that may not
 * allocate device memory where they need a flow — a framework that owns the
 * device memory pool, a service that reserves everything at start-up and
 * must not let cudaMalloc synchronize the device on the request path, a
 * plugin handed only device pointers.  The caller passes a paired-arc CSR
 * already in device memory (d_row: n+1 offsets from 0 to arcs; d_col/d_rev/
 * d_cap: arcs entries, any vertex order; every head in [0, n); rev[e] is an
 * arc of e's head back to e's tail with rev[rev[e]] == e; capacities >= 0)
 * and gets the exact max flow from s to t in *flow (host).  A check kernel
 * validates those rules first and a CSR that breaks one is rejected with
 * MF_ERR_ARG.  Scratch is a fixed file-scope device array of about 11 MB
 * sized for n <= 65536 vertices and arcs <= 1048576; larger graphs are
 * rejected with MF_ERR_ARG.  The call makes no cudaMalloc / cudaFree or
 * other allocating call.  Its first call on a device resolves the array's
 * device address and zeroes it (once per device, also when several host
 * threads make their first call together).  The address is kept for the
 * process's life, so a
 * cudaDeviceReset of that device is not supported afterwards.  Options are
 * resolved and device statuses reported exactly as mf_solve does.  Every
 * call waits for its stream to finish its work before returning.  Every call
 * shares the array and it keeps the last call's contents, so calls that
 * overlap on the GPU race: serialize them.  stream: a cudaStream_t (NULL =
 * default stream); stats may be NULL. */
int mf_solve_csr_noalloc(int n, long long arcs, const int32_t *d_row, const int32_t *d_col,
                         const int32_t *d_rev, const int64_t *d_cap, int32_t s, int32_t t,
                         const mf_opts *opts, void *stream, int64_t *flow, mf_stats *stats);

/* ---- dynamic capacities ----------------------------------------------- */

/* Apply nb capacity changes: arc u->v (first matching forward arc, caller
 * ids) gets cap += delta[i], clamped at 0 (extends OnAdd_kernel, RA:959-1000,
 * which handled increases only).  Pairs with no such arc are skipped and
 * counted in *skipped (may be NULL). */
int mf_update_caps(mf_graph *g, int nb, const int32_t *u, const int32_t *v, const int64_t *delta,
                   int *skipped);

/* Resident queries: a session keeps the residual state of nq queries on the
 * device across capacity updates (what the reference's dynamic mode,
 * RA:2844-2916, sets up but never updates).  mf_session_solve solves all of
 * them from scratch; mf_session_update applies a capacity batch to the graph
 * and repairs every resident query incrementally from its kept residual
 * state (flow cancelled on arcs whose capacity fell below their flow, new
 * capacity saturated from the source, then push-relabel resumes).  A batch
 * that changes more than 1/2000 of the graph's arcs re-solves the resident
 * queries from scratch instead (faster at that size; environment variable
 * MF_REPAIR_MAX_UPDATES sets another limit). */
typedef struct mf_session mf_session;
int mf_session_create(mf_graph *g, int nq, const int32_t *s, const int32_t *t, const mf_opts *opts,
                      mf_session **out);
int mf_session_solve(mf_session *ss, int64_t *flows, mf_stats *stats);
int mf_session_update(mf_session *ss, int nb, const int32_t *u, const int32_t *v,
                      const int64_t *delta, int64_t *flows, mf_stats *stats);
int mf_session_destroy(mf_session *ss);

/* ---- serving ------------------------------------------------------------ */

/* Continuous-batching server over several device-resident graphs (the
 * reference's dynamic mode, RA:2844-2916, grown into a request loop; its
 * capacity updates replace the unwired incremental_update_max_flow_with_state,
 * RA:2273-2335).  One persistent kernel takes requests from a host-written
 * ring in ticket order: (s,t) queries and capacity-update batches.  Requests
 * that arrive while others run are admitted as soon as a query group with a
 * residual slot frees up.  Slots are sized for the largest graph and
 * admitted by free HBM as requests open up: the server starts with up to 4
 * and, whenever more requests are open than slots exist, allocates another
 * if cudaMemGetInfo shows room (85 % of free HBM), up to max_slots (0 = one
 * per query group of the GPU).  The ring holds 65536 requests (environment
 * variable MF_SERVER_RING sets another size): a ticket's entry is reused
 * once the ticket `ring size` later is submitted, so poll each result before
 * that; a submit while that many requests are still unfinished returns
 * MF_ERR_NOMEM.  The graphs must not be used through other entry points
 * while the server exists; after mf_server_destroy they are usable again
 * with the capacities the served updates left. */
typedef struct mf_server mf_server;
int mf_server_create(mf_graph **graphs, int ngraphs, const mf_opts *opts, int max_slots,
                     mf_server **out);
/* Slots admitted so far. */
int mf_server_slots(const mf_server *sv, int *slots);
/* Enqueue one query; returns its ticket (0,1,2,...) in *ticket.  It is
 * answered on the graph as left by every update batch submitted before it
 * on that graph, and by none submitted after it. */
int mf_server_submit(mf_server *sv, int graph, int32_t s, int32_t t, long long *ticket);
/* Enqueue a capacity-update batch on one graph: arc u[i] -> v[i] (first
 * matching forward arc, caller ids) gets cap += delta[i], clamped at 0 after
 * each change, in order (mf_update_caps semantics; pairs with no such arc
 * are skipped).  It is applied on the device after every query submitted
 * before it on that graph has finished and before any query submitted after
 * it starts; queries on other graphs run on meanwhile.  Its ticket polls
 * done (flow 0) once applied.  The batch's distinct (u, v) pairs must fit
 * the update arena (1048576 entries; MF_SERVER_UPDATE_ARENA sets another). */
int mf_server_update(mf_server *sv, int graph, int nb, const int32_t *u, const int32_t *v,
                     const int64_t *delta, long long *ticket);
/* Non-blocking: 1 in *done when the ticket finished (flow, device latency in
 * ms from admission to completion, status). */
int mf_server_poll(mf_server *sv, long long ticket, int *done, int64_t *flow, double *latency_ms,
                   int *status);
/* Block until every submitted request has finished. */
int mf_server_drain(mf_server *sv);
/* Stops the kernel (requests not yet started are dropped: drain first). */
int mf_server_destroy(mf_server *sv);

/* ---- autotuning ---------------------------------------------------------- */

/* Time mf_solve_batch on the given sample of queries over a grid of
 * (R, kernel_cycles, gr_freq, group_ctas) and write the fastest into *best
 * (R into *best_R).  Repartitions g to the best R before returning. */
int mf_autotune(mf_graph *g, int nq, const int32_t *s, const int32_t *t, const mf_opts *base,
                mf_opts *best, int *best_R);

/* ---- synthetic workloads (seeded; used by the bench and the tests) -------- */

/* Uniform directed graph: u != v uniform in [0,n), cap uniform in [lo,hi]. */
int mf_gen_uniform(int n, long long m, long long lo, long long hi, unsigned long long seed,
                   int32_t *u, int32_t *v, int64_t *cap);
/* R-MAT with n = 2^scale and m draws of probabilities (a,b,c,1-a-b-c); self
 * loops dropped; returns the kept count in *kept (arrays hold m entries). */
int mf_gen_rmat(int scale, long long m, double a, double b, double c, long long lo, long long hi,
                unsigned long long seed, int32_t *u, int32_t *v, int64_t *cap, long long *kept);
/* W x H 4-connected grid plus source (id W*H) and sink (id W*H+1):
 * neighbour arcs cap 1+floor(255*exp(-d^2/50)), d ~ N(0,40); each pixel gets
 * one terminal arc (source->p or p->sink by a seeded coin) with cap uniform
 * in [0,255].  Arrays hold 4*W*H + W*H entries; *m receives the count. */
int mf_gen_grid(int W, int H, unsigned long long seed, int32_t *u, int32_t *v, int64_t *cap,
                long long *m);
/* Queries for a power-law graph: nhub pairs with s in the top 1% by
 * out-degree and t in the top 1% by in-degree, then nuni uniform pairs;
 * s != t. */
int mf_gen_queries_hub(int n, long long m, const int32_t *u, const int32_t *v, int nhub, int nuni,
                       unsigned long long seed, int32_t *s, int32_t *t);
/* Write graph.txt / test.txt (1-based ids). */
int mf_write_graph_txt(const char *path, int n, long long m, const int32_t *u, const int32_t *v,
                       const int64_t *cap);
int mf_write_test_txt(const char *path, int nq, const int32_t *s, const int32_t *t);
/* Parse graph.txt with the reference's rules (RA:1051-1075) into 0-based
 * arrays holding cap_len entries; *n, *m_read. */
int mf_read_graph_txt(const char *path, int *n, long long *m_read, int32_t *u, int32_t *v,
                      int64_t *cap, long long cap_len);
/* Count of edge lines in a graph.txt header (to size the arrays). */
int mf_graph_txt_header(const char *path, int *n, long long *m);

#ifdef __cplusplus
}
#endif

#endif /* MAXFLOW_B200_H */
