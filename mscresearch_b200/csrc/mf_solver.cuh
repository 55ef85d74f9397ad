// Solver-side device structures shared by mf_solver.cu and the host API.
#pragma once
#include "mf_common.cuh"

// Region-ordered CSR of one graph (device pointers).
struct DGraph {
    int n;
    int R;
    i64 arcs;
    const int *row;        // n+1
    const int *col;        // arcs
    const int *rev;        // arcs
    const i64 *cap;        // arcs (current capacities)
    const int *region_of;  // n
    // Vertices with more than HUB_T arcs (NULL: not available; the prune
    // then runs its searches top-down only).
    const int *hubs;
    int nhub;
    // Kept-set cache: the strongly connected component of a pivot vertex.
    // For s and t both in it, fwd(s) & bwd(t) is exactly that component, so
    // a query can take its kept list (vlist layout: front kc_f entries, back
    // kc_b entries) and initial residuals (kc_res: cap, arcs to heads outside
    // the component 0) instead of pruning.  kc_in == NULL: no cache.
    const unsigned char *kc_in;  // n: 1 = in the component
    const int *kc_img;           // n: kept list image
    const i64 *kc_res;           // arcs: initial residuals
    // Closures of the pivot (KC_F / KC_B bits, NULL: none).  s in B implies
    // fwd(s) covers F, t in F implies bwd(t) covers B, so a query with
    // s in B and t in F keeps the component plus a few extra vertices, and
    // for t outside F (s outside B) the search from t (s) stays outside F (B).
    const unsigned char *kc_fb;
    int kc_f, kc_b;
    i64 kc_arcs;                 // arcs out of the component's vertices
    // Vertices with more than GIANT_T arcs (NULL: none listed; warp-per-vertex
    // loops then take every vertex themselves).
    const int *giants;
    int ngiant;
    const unsigned char *fwd;  // arcs: 1 = forward arc of an input edge (capacity updates)
};

// Vertices with more arcs than this are "giants": loops that give each
// vertex one warp (state init, certificate, residual export) skip them and
// spread their arcs over every thread of the group instead -- one warp
// walking a 4-million-arc super terminal took ~150 ms.
#define GIANT_T 4096

// Vertices with more arcs than this are "hubs": worklists keep them at the
// back and their arcs are processed in 32-arc chunks by all warps of a group.
#define HUB_T 512

// Per-hub state of one chunked discharge pass.
struct HubWork {
    i64 budget;  // excess not yet handed out to chunks
    int minh;    // lowest head height over arcs left with residual
    int done;    // chunks finished
    int hv;      // hub height at set-up
    int nch;     // chunks (0 = nothing to do)
    int cstart;  // chunks of the hubs before this one (exclusive prefix of nch)
};

// Working state of one residual slot.  All arrays are full-size for the
// graph the slot serves; stamps make resets unnecessary between queries.
// Control words per slot (list tails, query hand-off, search state).
#define CNT_WORDS 64

struct DSlot {
    i64 *res;          // arcs: residual capacity
    i64 *ex;           // n: excess
    int *h;            // n: height
    unsigned *mark;    // n: prune / mask / relabel stamps
    unsigned *qmark;   // n: worklist de-dup stamps (also undirected-prune stamps)
    unsigned *claim;   // n: path-push ownership stamps / old-mask stamps
    int *vlist;        // n: the query's kept (mask) vertices
    int *qa;           // n: BFS queue / worklist
    int *qb;           // n: worklist
    int *hot;          // 1024: region counts / hot flags
    int *ract;         // 1024: active-region flags
    int *cnt;          // CNT_WORDS ints: rotating list tails (front, back) + control words
    i64 *acc;          // 64 i64: rotating round accumulators + query totals
    GroupBar *bar;     // group barrier
    unsigned *clock;   // persistent stamp clock
    int *meta;         // per-slot query meta (mask stamp, nv, s, t, front count) for warm starts
    HubWork *hubw;     // nhub entries
    int nhub;          // capacity of hubw (hub vertices of the largest graph served)
    unsigned *bits;    // 5 bitmaps of (n + 31) / 32 words: kept, visited, 3 frontier maps
};

// Words of one per-vertex bitmap.
__host__ __device__ inline int bitmap_words(int n) { return (n + 31) >> 5; }

// Options as seen by the kernel (resolved on the host).
struct KOpts {
    int K;
    int gr_freq;
    double gr_alpha;
    int prune_mode;
    int pp_switch;
    int max_path;
    int use_pp;
    int use_hot;
    int hot_k;
    int use_rm;
    int rm_freq;
    int h_cut;
    int stagnate;
    int force_rm;
    int force_pp;
    int use_cache;
    int bu_factor;  // bottom-up when frontier x bu_factor > unvisited (and >= 1/64 of all)
    i64 iter_max;
    int gr_stop;    // global relabels end once every active vertex is labelled
    int bu_arcs;    // relabel searches also go bottom-up when the frontier has more than
                    // bu_arcs arcs per unvisited vertex (0: vertex counts only)
    int local_rl;   // local relabel after every local_rl-th round between global ones (0: off)
};

// Per-query outputs.
struct QOut {
    i64 flow;
    i64 rounds;
    i64 relabels;
    i64 arcs_ex;
    i64 verts_ex;
    i64 pushes;
    i64 rm_fixed;
    i64 pp_rounds;
    i64 hot_sweeps;
    i64 deficit_phases;
    i64 cut;
    i64 mask_arcs;
    u64 t_begin;   // globaltimer ns when the group took the query
    u64 t_done;    // globaltimer ns when its answer was written
    u64 t_prune;   // ns in prune + init + preflow
    u64 t_relabel; // ns in global relabels
    u64 t_rounds;  // ns in discharge rounds (incl. hot sweep, path push, RM)
    i64 arcs_relabel; // arc examinations inside global relabels
    i64 arcs_hubs;    // arc examinations by the chunked hub discharge
    i64 hub_passes;   // hub discharge passes (a hub with excess, all its chunks)
    i64 hub_relabels; // passes that ended with excess left (the hub was relabeled)
    i64 levels;           // search levels (prune, relabels, certificate)
    i64 levels_bottom_up; // of which bottom-up
    i64 levels_solo;      // of which run by one CTA
    int mask_n;
    int status;
    int kept_front;  // kept vertices in vlist's front part
    int local_relabels;  // local relabels between global ones
};

// One capacity change, resolved to an arc (region-ordered index).
struct ArcUpdate {
    int arc;
    int pad;
    i64 old_cap;
    i64 new_cap;
};

enum KMode {
    KM_SOLVE = 0,       // prune + solve
    KM_PRUNE = 1,       // prune only; writes the 0/1 mask into dbg (n bytes, internal order)
    KM_HEIGHTS = 2,     // prune + init + preflow + one global relabel; heights into dbg (ints)
    KM_CERTIFY = 3,     // solve + return excess to source + certificate checks
    KM_RESIDUAL = 4,    // solve, then write full-graph residuals into dbg (i64 per arc)
    KM_REPAIR = 5,      // warm start from the slot's kept state after capacity updates
    KM_KEPTSET = 6,     // prune from a pivot (s == t): the pivot's SCC; kept list image and
                        // membership written to the KcOut in dbg
};

// Output of KM_KEPTSET.
struct KcOut {
    int *img;             // n: kept list image (vlist layout)
    unsigned char *in;    // n: membership (caller zeroes it)
    unsigned char *fb;    // n: KC_F | KC_B bits
};

// kc_fb bits: the vertex is reachable from the pivot (F) / reaches it (B).
// F is closed under forward arcs, B under backward arcs, F & B = component.
#define KC_F 1
#define KC_B 2

// ---- continuous-batching server ---------------------------------------------
// One request in the server's ring (host-written, mapped).  kind 0: an (s,t)
// query on `graph` that must see the graph after `epoch` capacity-update
// batches on it; kind 1: the update batch number `epoch` of `graph`, whose
// upd_n entries start at upd_off in the update arena, applied once the
// graph's first `need_done` queries (all queries submitted before it) are
// done.
struct RingReq {
    int kind;
    int graph;
    int s, t;
    int epoch;
    int upd_n;
    long long upd_off;
    unsigned long long need_done;
    long long pad;
};
#define RQ_QUERY 0
#define RQ_UPDATE 1

// One capacity change in an update batch: the first forward arc u -> v
// (internal ids) gets capacity max(a, cap + b).  The host folds every change
// of one (u, v) pair in a batch into one entry: a sequence of "cap += d,
// clamped at 0" steps composes to exactly this form.
struct UpdEntry {
    int u, v;
    i64 a, b;
};

// Per-graph server state (device): update batches applied, queries done,
// kept-set cache invalid (set by the first update).
struct GState {
    int epoch;
    int no_cache;
    unsigned long long done_q;
};

// Per-group server control block (device): the group's barrier (a group
// may run before it has a slot), broadcast words and its slot.
struct GroupCtl {
    GroupBar bar;
    unsigned long long q;
    int w[8];
    DSlot slot;
};

// Server-wide control (device): the next request to claim, and the count of
// groups serving (parked groups leave when it reaches 0).
struct SrvCtl {
    unsigned long long next;
    int live;
    int pad;
};

struct KParams {
    const DGraph *graphs;
    DSlot *slots;
    int G;            // CTAs per query group
    int nq;
    const int *q_s;   // internal ids
    const int *q_t;
    const int *q_g;   // graph index per query (NULL = 0)
    const int *q_slot;// slot per query (NULL = group id)
    int *q_next;      // work queue head
    QOut *out;
    int *err;
    u64 bar_limit_ns;
    u64 time_limit_ns;  // per launch; 0 = none.  Past it the solve stops with MFD_TIMEOUT.
    KOpts o;
    int mode;
    void *dbg;
    const ArcUpdate *upd;
    int nupd;
    // per-query capacity overrides (NULL: none): query q sees capacity
    // ov_cap[q * ov_n + j] on forward arc ov_arc[j] (never above its cap)
    const int *ov_arc;
    const i64 *ov_cap;
    long long ov_n;
    // serving ring (mode KM_SOLVE with ring_tail != NULL): request k (a
    // 64-bit ticket) lives in entry k % ring_cap and may be claimed once the
    // host-written ring_tail exceeds k.  All host-side arrays are mapped.
    volatile unsigned long long *ring_tail;
    const RingReq *ring_req;
    int ring_cap;
    volatile int *ring_done;     // per entry: 2 while running, 1 when finished
    u64 *ring_t0;                // per entry: admission / completion timestamps (ns)
    volatile int *ring_stop;     // host sets 1 to end the persistent kernel
    u64 idle_limit_ns;           // a group idle this long leaves
    SrvCtl *srv;
    GState *gstate;              // per graph
    GroupCtl *gctl;              // per group
    const volatile DSlot *slot_tab;   // per group: its slot (mapped)
    volatile int *slot_ready;    // per group: 0 none yet, 1 new (clear it first), 2 ready
    int slot_n;                  // vertices the server's slots are sized for
    const UpdEntry *srv_upd;     // update arena (mapped)
};

void mf_launch_kernel(const KParams &p, int grid, int threads, cudaStream_t st, bool cooperative,
                      cudaError_t *err);
int mf_kernel_max_blocks_per_sm(int threads);
// mf_serve_kernel.cu: the serving kernel (the solver compiled with coherent
// capacity loads).
cudaError_t mf_launch_serve_kernel(const KParams &p, int grid, int threads, cudaStream_t st, bool cooperative);
int mf_serve_kernel_max_blocks_per_sm(int threads);
