// Host side of the C ABI (include/maxflow_b200.h): graph residency, residual
// slots, launch configuration, batched / session / serving drivers.
//
// Reference seam replaced (Region_Aware_PR_with_Pruning_BoundaryCore.cu):
//   build_graph RA:1044-1126 ............ host CSR build below (same reader rules)
//   init_global_graph_on_device RA:1293 .. mf_graph_create_from_edges (device-resident,
//                                          region-ordered CSR built on the device)
//   init_state_for_st / free_state RA:1336, RA:86 .. residual slots (allocated once,
//                                          stamp-reset, reused across queries)
//   run_gpu_static_with_state RA:2119 .... mf_solve / mf_solve_batch
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <condition_variable>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/maxflow_b200.h"
#include "mf_alloc.h"
#include "mf_build.cuh"
#include "mf_scc.cuh"
#include "mf_solver.cuh"

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(e_ == cudaErrorMemoryAllocation ? MF_ERR_NOMEM : MF_ERR_CUDA,     \
                        "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                        __LINE__);                                                        \
    } while (0)

struct DevInfo {
    int sms = 0;
    int bps = 0;  // co-resident mf_kernel CTAs per SM at the default block size
    int threads = 512;
    bool ok = false;
};

int dev_info(DevInfo &d, int threads) {
    if (threads < 64 || threads > 512 || threads % 32)
        return fail(MF_ERR_ARG, "threads per CTA must be a multiple of 32 in [64, 512] (got %d)", threads);
    int dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev));
    // L2 fetch granularity hint for this process's context (bytes fetched
    // from DRAM per L2 miss: 0..128); it lasts as long as the context
    if (const char *e = getenv("MF_L2_FETCH_BYTES")) CK(cudaDeviceSetLimit(cudaLimitMaxL2FetchGranularity, (size_t)atoi(e)));
    d.threads = threads;
    d.bps = mf_kernel_max_blocks_per_sm(threads);
    if (d.bps <= 0) return fail(MF_ERR_CUDA, "mf_kernel cannot be resident with %d threads", threads);
    d.ok = true;
    return MF_OK;
}

size_t slot_bytes(int n, i64 arcs, int nhub) {
    size_t b = 0;
    auto add = [&](size_t x) { b += (x + 255) & ~(size_t)255; };
    add(sizeof(i64) * (size_t)std::max<i64>(arcs, 1));  // res
    add(sizeof(i64) * (size_t)n);                        // ex
    for (int i = 0; i < 7; ++i) add(sizeof(int) * (size_t)n);  // h mark qmark claim vlist qa qb
    add(sizeof(int) * 1024);                             // hot
    add(sizeof(int) * 1024);                             // ract
    add(sizeof(int) * CNT_WORDS);                        // cnt
    add(sizeof(i64) * 128);                              // acc
    add(sizeof(GroupBar));
    add(sizeof(unsigned));                               // clock
    add(sizeof(int) * 8);                                // meta
    add(sizeof(HubWork) * (size_t)std::max(nhub, 1));    // hubw
    add(sizeof(unsigned) * 5 * (size_t)bitmap_words(n));  // bits
    return b;
}

// The arrays of one residual slot inside one allocation of slot_bytes(),
// each 256-byte aligned, in this order (the residuals first: everything
// after them is what a new slot must have zeroed).
DSlot carve_slot(char *p, int n, i64 arcs, int nhub) {
    auto take = [&](size_t x) {
        char *r = p;
        p += (x + 255) & ~(size_t)255;
        return (void *)r;
    };
    DSlot s;
    s.res = (i64 *)take(sizeof(i64) * (size_t)std::max<i64>(arcs, 1));
    s.ex = (i64 *)take(sizeof(i64) * (size_t)n);
    s.h = (int *)take(sizeof(int) * (size_t)n);
    s.mark = (unsigned *)take(sizeof(int) * (size_t)n);
    s.qmark = (unsigned *)take(sizeof(int) * (size_t)n);
    s.claim = (unsigned *)take(sizeof(int) * (size_t)n);
    s.vlist = (int *)take(sizeof(int) * (size_t)n);
    s.qa = (int *)take(sizeof(int) * (size_t)n);
    s.qb = (int *)take(sizeof(int) * (size_t)n);
    s.hot = (int *)take(sizeof(int) * 1024);
    s.ract = (int *)take(sizeof(int) * 1024);
    s.cnt = (int *)take(sizeof(int) * CNT_WORDS);
    s.acc = (i64 *)take(sizeof(i64) * 128);
    s.bar = (GroupBar *)take(sizeof(GroupBar));
    s.clock = (unsigned *)take(sizeof(unsigned));
    s.meta = (int *)take(sizeof(int) * 8);
    s.hubw = (HubWork *)take(sizeof(HubWork) * (size_t)std::max(nhub, 1));
    s.nhub = std::max(nhub, 1);
    s.bits = (unsigned *)take(sizeof(unsigned) * 5 * (size_t)bitmap_words(n));
    return s;
}

struct SlotPool {
    int n = 0;
    i64 arcs = 0;
    int nhub = 0;
    std::vector<void *> bases;
    std::vector<DSlot> host;
    DSlot *dev = nullptr;
    int dev_cap = 0;

    int grow(int want) {
        while ((int)host.size() < want) {
            size_t bytes = slot_bytes(n, arcs, nhub);
            void *base = nullptr;
            cudaError_t e = mf_dmalloc(&base, bytes);
            if (e != cudaSuccess) {
                cudaGetLastError();
                return fail(MF_ERR_NOMEM, "residual slot allocation (%zu bytes) failed: %s", bytes,
                            cudaGetErrorString(e));
            }
            // the legacy-stream clear and table upload below are waited for:
            // the solves run on non-blocking streams that do not wait on them
            e = cudaMemset(base, 0, bytes);
            if (e == cudaSuccess) e = cudaStreamSynchronize(0);
            if (e != cudaSuccess) {
                mf_dfree(base);
                return fail(MF_ERR_CUDA, "residual slot clear failed: %s", cudaGetErrorString(e));
            }
            DSlot s = carve_slot((char *)base, n, arcs, nhub);
            bases.push_back(base);
            host.push_back(s);
        }
        if (dev_cap < (int)host.size()) {
            if (dev) mf_dfree(dev);
            dev = nullptr;
            dev_cap = 0;
            CK(mf_dmalloc(&dev, sizeof(DSlot) * host.size()));
            dev_cap = (int)host.size();
        }
        CK(cudaMemcpy(dev, host.data(), sizeof(DSlot) * host.size(), cudaMemcpyHostToDevice));
        CK(cudaStreamSynchronize(0));
        return MF_OK;
    }
    void release() {
        for (void *b : bases) mf_dfree(b);
        bases.clear();
        host.clear();
        if (dev) mf_dfree(dev);
        dev = nullptr;
        dev_cap = 0;
    }
};

// Zero the group barriers of the first nslots slots and read their clocks.
__global__ void k_prepare_slots(DSlot *slots, int nslots, unsigned *clocks) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nslots) {
        slots[i].bar->arrive = 0;
        slots[i].bar->gen = 0;
        clocks[i] = *slots[i].clock;
    }
}

// Stamp arrays are only compared against the slot's own monotonic clock;
// before the 32-bit clock can wrap, the slot is reset to zero.
__global__ void k_reset_slot(DSlot s, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        s.mark[i] = 0;
        s.qmark[i] = 0;
        s.claim[i] = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *s.clock = 0;
}

// Capacity updates: resolve (u,v) to the first forward arc u->v (lowest
// index in u's list).  The shorter of the two lists is scanned: in v's list
// every reverse arc v->u (fwd = 0) is paired with a forward arc u->v, found
// through rev, so a hub tail (a super source, an R-MAT hub) does not cost
// its whole list per update.  A warp per update scans 32 arcs per step and
// stops at the first step holding a match: arc lists keep the edges' input
// order (the CSR build and the region reorder are stable), so the first
// matching reverse arc in v's list pairs with the lowest forward arc; the
// minimum over that step's matches is taken all the same.
__global__ void k_find_arcs(int nb, const int *u, const int *v, const int *row, const int *col,
                            const int *rev, const unsigned char *fwd, const i64 *cap, int *arc,
                            i64 *capv) {
    const int i = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (i >= nb) return;  // whole warps leave together (i is uniform in a warp)
    int a = INT_MAX;
    const int x = u[i], y = v[i];
    if (x >= 0 && y >= 0) {
        const bool by_head = row[y + 1] - row[y] < row[x + 1] - row[x];
        const int w = by_head ? y : x, other = by_head ? x : y;
        const int b = row[w], e1 = row[w + 1];
        for (int eb = b; eb < e1; eb += 32) {
            const int e = eb + lane;
            int cand = INT_MAX;
            if (e < e1 && col[e] == other && (fwd[e] != 0) != by_head) cand = by_head ? rev[e] : e;
            const int m = __reduce_min_sync(0xffffffffu, cand);
            if (m != INT_MAX) {
                a = m;
                break;
            }
        }
    }
    if (lane == 0) {
        arc[i] = a == INT_MAX ? -1 : a;
        capv[i] = a == INT_MAX ? 0 : cap[a];
    }
}

// Override checks: every arc resolved, every query's capacity in
// [0, the graph's capacity of the arc]; counts the violations.
__global__ void k_check_overrides(long long nov, int nq, const int *arc, const i64 *gcap, const i64 *ov,
                                  int *bad) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nov * (long long)nq) return;
    long long j = i % nov;
    i64 c = ov[i];
    if (arc[j] < 0 || c < 0 || c > gcap[j]) atomicAdd(bad, 1);
}

__global__ void k_apply_caps(int nu, const ArcUpdate *upd, i64 *cap) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nu) cap[upd[i].arc] = upd[i].new_cap;
}

}  // namespace

struct mf_graph {
    int n = 0;
    i64 arcs = 0;
    int R = 0;
    int avg_deg = 0;
    int nhub = 0;  // vertices with more than HUB_T arcs
    int pivot = 0;  // internal id of the highest-degree vertex (kept-set cache pivot)
    int *hubs = nullptr;  // device: internal ids of the hubs
    int ngiant = 0;       // vertices with more than GIANT_T arcs
    int *giants = nullptr;  // device: their internal ids
    std::vector<int> deg_host;                // internal id -> arcs
    std::vector<unsigned char> kc_in_host;    // internal id -> in the cached component
    // grow-only device buffers of capacity-update batches (resolution arrays;
    // resolved records), kept so that a batch allocates nothing
    void *upd_scratch = nullptr;
    size_t upd_scratch_bytes = 0;
    ArcUpdate *upd_recs = nullptr;
    size_t upd_recs_cap = 0;
    // kept-set cache (see DGraph)
    unsigned char *kc_in = nullptr;
    unsigned char *kc_fb = nullptr;
    int *kc_img = nullptr;
    i64 *kc_res = nullptr;
    int kc_f = 0, kc_b = 0;
    i64 kc_arcs = 0;
    bool kc_valid = false;
    bool kc_tried = false;
    std::vector<int> new_id;  // caller id -> internal id
    std::vector<int> old_id;  // internal id -> caller id
    std::vector<double> score_caller;
    std::vector<int> part_caller;
    SccOut scc;  // the last mf_graph_scc result (contracted arcs for mf_graph_scc_contracted)
    bool scc_done = false;
    // region-ordered device CSR
    int *row = nullptr, *col = nullptr, *rev = nullptr, *region_of = nullptr,
        *region_start = nullptr;
    i64 *cap = nullptr;
    unsigned char *fwd = nullptr;
    DGraph *d_graph = nullptr;
    SlotPool pool;
    DevInfo dev;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int *d_err = nullptr, *d_qnext = nullptr;
    unsigned *d_clocks = nullptr;
    int clocks_cap = 0;
    QOut *d_out = nullptr;
    int out_cap = 0;
    int *d_q = nullptr;  // s | t | slot, 3*q_cap
    int q_cap = 0;
    int *h_pin = nullptr;  // pinned staging for queries
    QOut *h_out = nullptr;
    int pin_cap = 0;
    double last_ms = 0.0;
    long launches = 0;
};

namespace {
cudaError_t up(const mf_graph *g, void *dst, const void *src, size_t n) {
    return n ? cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, g->stream) : cudaSuccess;
}
cudaError_t zero(const mf_graph *g, void *dst, size_t n) {
    return n ? cudaMemsetAsync(dst, 0, n, g->stream) : cudaSuccess;
}
cudaError_t down(const mf_graph *g, void *dst, const void *src, size_t n) {
    cudaError_t e = n ? cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, g->stream) : cudaSuccess;
    return e == cudaSuccess ? cudaStreamSynchronize(g->stream) : e;
}
}  // namespace

struct mf_session {
    mf_graph *g = nullptr;
    int nq = 0;
    std::vector<int> s, t;  // internal
    SlotPool pool;
    mf_opts opts;
    bool solved = false;
};

namespace {

// Copies and clears of graph data, ordered on the graph's stream.  The
// stream is non-blocking (it does not wait on the legacy default stream),
// so a plain cudaMemcpy / cudaMemset -- which run on the legacy stream, the
// former even returning before a pageable upload's DMA has landed -- would
// not be ordered before the kernels launched on it afterwards.
cudaError_t up(const mf_graph *g, void *dst, const void *src, size_t n);
cudaError_t zero(const mf_graph *g, void *dst, size_t n);
cudaError_t down(const mf_graph *g, void *dst, const void *src, size_t n);

// Marks the kept-set cache stale (capacities changed) and keeps its buffers
// for the rebuild: freeing and re-allocating ~9 bytes per arc on every
// update batch cost a device-wide synchronization and tens of ms.
void invalidate_kept_cache(mf_graph *g) {
    g->kc_valid = false;
    g->kc_tried = false;
    g->kc_in_host.clear();
}

void free_kept_cache(mf_graph *g) {
    mf_dfree(g->kc_in);
    mf_dfree(g->kc_fb);
    g->kc_fb = nullptr;
    mf_dfree(g->kc_img);
    mf_dfree(g->kc_res);
    g->kc_in = nullptr;
    g->kc_img = nullptr;
    g->kc_res = nullptr;
    g->kc_valid = false;
    g->kc_tried = false;
    g->kc_in_host.clear();
}

void free_graph_arrays(mf_graph *g) {
    free_kept_cache(g);
    mf_dfree(g->upd_scratch);
    g->upd_scratch = nullptr;
    g->upd_scratch_bytes = 0;
    mf_dfree(g->upd_recs);
    g->upd_recs = nullptr;
    g->upd_recs_cap = 0;
    mf_dfree(g->row);
    mf_dfree(g->col);
    mf_dfree(g->rev);
    mf_dfree(g->cap);
    mf_dfree(g->fwd);
    mf_dfree(g->region_of);
    mf_dfree(g->region_start);
    mf_dfree(g->d_graph);
    mf_dfree(g->hubs);
    g->hubs = nullptr;
    mf_dfree(g->giants);
    g->giants = nullptr;
    g->ngiant = 0;
    g->row = g->col = g->rev = g->region_of = g->region_start = nullptr;
    g->cap = nullptr;
    g->fwd = nullptr;
    g->d_graph = nullptr;
}

DGraph make_dgraph(const mf_graph *g) {
    DGraph dg{};
    dg.n = g->n;
    dg.R = g->R;
    dg.arcs = g->arcs;
    dg.row = g->row;
    dg.col = g->col;
    dg.rev = g->rev;
    dg.cap = g->cap;
    dg.region_of = g->region_of;
    dg.hubs = g->hubs;
    dg.nhub = g->hubs ? g->nhub : 0;
    dg.giants = g->giants;
    dg.ngiant = g->giants ? g->ngiant : 0;
    dg.fwd = g->fwd;
    if (g->kc_valid) {
        dg.kc_in = g->kc_in;
        dg.kc_fb = g->kc_fb;
        dg.kc_img = g->kc_img;
        dg.kc_res = g->kc_res;
        dg.kc_f = g->kc_f;
        dg.kc_b = g->kc_b;
        dg.kc_arcs = g->kc_arcs;
    }
    return dg;
}

int upload_dgraph(mf_graph *g) {
    DGraph dg = make_dgraph(g);
    CK(up(g, g->d_graph, &dg, sizeof(DGraph)));
    return MF_OK;
}

int finalize_graph(mf_graph *g);

// Partition + reorder the device CSR given in (row,col,cap,rev,fwd), whose
// vertex i is caller vertex in_ids[i].  Replaces the graph arrays.
int partition_into(mf_graph *g, int R, int *row, int *col, i64 *cap, int *rev, unsigned char *fwd,
                   const std::vector<int> &in_to_caller) {
    const int n = g->n;
    const i64 arcs = g->arcs;
    BuildIn in{n, R, arcs, row, col, cap, rev, fwd};
    BuildOut out{};
    // the new graph arrays (kept on success) and the build's temporaries:
    // both scopes free what they hold if any step fails
    DevScope keep, tmp;
    CK(keep.alloc(&out.row, sizeof(int) * ((size_t)n + 1)));
    CK(keep.alloc(&out.col, sizeof(int) * (size_t)std::max<i64>(arcs, 1)));
    CK(keep.alloc(&out.cap, sizeof(i64) * (size_t)std::max<i64>(arcs, 1)));
    CK(keep.alloc(&out.rev, sizeof(int) * (size_t)std::max<i64>(arcs, 1)));
    CK(keep.alloc(&out.fwd, (size_t)std::max<i64>(arcs, 1)));
    CK(keep.alloc(&out.region_start, sizeof(int) * ((size_t)R + 1)));
    CK(keep.alloc(&out.region_of, sizeof(int) * (size_t)n));
    CK(tmp.alloc(&out.new_id, sizeof(int) * (size_t)n));
    CK(tmp.alloc(&out.old_id, sizeof(int) * (size_t)n));
    CK(tmp.alloc(&out.score, sizeof(double) * (size_t)n));
    CK(tmp.alloc(&out.part, sizeof(int) * (size_t)n));
    void *scratch = nullptr;
    CK(tmp.alloc(&scratch, mf_partition_scratch_bytes(n, arcs, R)));
    CK(mf_partition_reorder(in, out, scratch, g->stream));
    CK(cudaStreamSynchronize(g->stream));
    std::vector<int> nid(n), sc_part(n);
    std::vector<double> sc(n);
    CK(down(g, nid.data(), out.new_id, sizeof(int) * n));
    CK(down(g, sc.data(), out.score, sizeof(double) * n));
    CK(down(g, sc_part.data(), out.part, sizeof(int) * n));
    // compose: caller -> input index -> internal
    std::vector<int> new_id(n), old_id(n);
    g->score_caller.assign(n, 0.0);
    g->part_caller.assign(n, 0);
    for (int i = 0; i < n; ++i) {
        int x = in_to_caller[i];
        new_id[x] = nid[i];
        old_id[nid[i]] = x;
        g->score_caller[x] = sc[i];
        g->part_caller[x] = sc_part[i];
    }
    free_graph_arrays(g);
    keep.release();
    g->row = out.row;
    g->col = out.col;
    g->cap = out.cap;
    g->rev = out.rev;
    g->fwd = out.fwd;
    g->region_start = out.region_start;
    g->region_of = out.region_of;
    g->new_id.swap(new_id);
    g->old_id.swap(old_id);
    g->R = R;
    return finalize_graph(g);
}

// Host copies of the degrees, the hub list, the cache pivot and the device
// graph record, from the region-ordered arrays.
int finalize_graph(mf_graph *g) {
    const int n = g->n;
    int best = 0;
    {
        std::vector<int> rw(n + 1), hl, gl;
        CK(down(g, rw.data(), g->row, sizeof(int) * (n + 1)));
        for (int x = 1; x < n; ++x)
            if (rw[x + 1] - rw[x] > rw[best + 1] - rw[best]) best = x;
        g->deg_host.resize(n);
        for (int x = 0; x < n; ++x) {
            g->deg_host[x] = rw[x + 1] - rw[x];
            if (rw[x + 1] - rw[x] > HUB_T) hl.push_back(x);
            if (rw[x + 1] - rw[x] > GIANT_T) gl.push_back(x);
        }
        g->nhub = (int)hl.size();
        if (!hl.empty()) {
            CK(mf_dmalloc(&g->hubs, sizeof(int) * hl.size()));
            CK(up(g, g->hubs, hl.data(), sizeof(int) * hl.size()));
        }
        g->ngiant = (int)gl.size();
        if (!gl.empty()) {
            CK(mf_dmalloc(&g->giants, sizeof(int) * gl.size()));
            CK(up(g, g->giants, gl.data(), sizeof(int) * gl.size()));
        }
    }
    g->pivot = best;
    CK(mf_dmalloc(&g->d_graph, sizeof(DGraph)));
    return upload_dgraph(g);
}

int ensure_launch_buffers(mf_graph *g, int nq, int nslots) {
    if (!g->d_err) {
        CK(mf_dmalloc(&g->d_err, sizeof(int) * 2));
        g->d_qnext = g->d_err + 1;
    }
    if (g->out_cap < nq) {
        mf_dfree(g->d_out);
        mf_hfree(g->h_out);
        g->d_out = nullptr;
        g->h_out = nullptr;
        g->out_cap = 0;  // a failed allocation below leaves no stale capacity
        CK(mf_dmalloc(&g->d_out, sizeof(QOut) * nq));
        CK(mf_hmalloc(&g->h_out, sizeof(QOut) * nq));
        g->out_cap = nq;
    }
    if (g->q_cap < nq) {
        mf_dfree(g->d_q);
        mf_hfree(g->h_pin);
        g->d_q = nullptr;
        g->h_pin = nullptr;
        g->q_cap = 0;
        CK(mf_dmalloc(&g->d_q, sizeof(int) * 3 * (size_t)nq));
        CK(mf_hmalloc(&g->h_pin, sizeof(int) * 3 * (size_t)nq));
        g->q_cap = nq;
    }
    if (g->clocks_cap < nslots) {
        mf_dfree(g->d_clocks);
        g->d_clocks = nullptr;
        g->clocks_cap = 0;
        CK(mf_dmalloc(&g->d_clocks, sizeof(unsigned) * nslots));
        g->clocks_cap = nslots;
    }
    return MF_OK;
}

KOpts resolve_opts(const mf_opts &o, int avg_deg) {
    KOpts k;
    k.K = o.kernel_cycles > 0 ? o.kernel_cycles : 8;
    (void)avg_deg;
    k.gr_freq = std::max(1, o.gr_freq);
    k.gr_alpha = o.gr_work_alpha;
    k.prune_mode = o.prune_mode;
    k.pp_switch = o.path_push_switch;
    k.max_path = std::max(1, o.max_path_len);
    k.use_pp = o.use_path_push;
    k.use_hot = o.use_hot_sweep;
    k.hot_k = std::max(1, o.hot_regions);
    k.use_rm = o.use_rm;
    k.rm_freq = std::max(1, o.rm_freq);
    k.h_cut = o.h_cut;
    k.stagnate = std::max(1, o.stagnate_rounds);
    k.force_rm = o.force_rm;
    k.force_pp = o.force_path_push;
    k.use_cache = o.use_kept_cache;
    // bottom-up once the frontier exceeds 1/56 of the unvisited vertices
    // (measured on the B200: 1/14, the usual edge-count rule, kept hub-heavy
    // early levels top-down; MF_BU_FACTOR overrides it for tuning)
    k.bu_factor = 56;
    if (const char *e = getenv("MF_BU_FACTOR")) k.bu_factor = std::max(1, atoi(e));
    k.iter_max = o.iter_max > 0 ? o.iter_max : 20000000;
    k.gr_stop = o.relabel_early_stop;
    if (const char *e = getenv("MF_RELABEL_EARLY_STOP")) k.gr_stop = atoi(e);
    // relabel searches go bottom-up when the frontier's arcs exceed bu_arcs
    // per unvisited vertex (MF_BU_ARCS overrides it; 0 = vertex counts only)
    k.bu_arcs = 8;
    if (const char *e = getenv("MF_BU_ARCS")) k.bu_arcs = std::max(0, atoi(e));
    k.local_rl = std::max(0, o.local_relabel);
    if (const char *e = getenv("MF_LOCAL_RELABEL")) k.local_rl = std::max(0, atoi(e));
    return k;
}

// Device time limit per solve launch: MF_TIME_LIMIT_S seconds (default 600).
u64 launch_time_limit_ns() {
    const char *e = getenv("MF_TIME_LIMIT_S");
    double s = e ? atof(e) : 600.0;
    if (s <= 0) return 0;
    return (u64)(s * 1e9);
}

int status_from_err(int e) {
    switch (e) {
    case MFD_OK: return MF_OK;
    case MFD_ITER_LIMIT: return MF_ERR_ITER_LIMIT;
    case MFD_TIMEOUT: return MF_ERR_TIMEOUT;
    case MFD_INEXACT: return MF_ERR_INEXACT;
    case MFD_CERTIFY: return MF_ERR_CERTIFY;
    default: return MF_ERR_CUDA;
    }
}

// Core launcher: nq queries (internal ids; s < 0 = skip) in `pool`'s slots.
// per_query_slot: query i uses slot i (sessions); else a slot per group.
int launch(mf_graph *g, SlotPool &pool, int nq, const int *s_int, const int *t_int,
           bool per_query_slot, const mf_opts &o, int mode, void *dbg, const ArcUpdate *d_upd,
           int nupd, int G_req, QOut *outs, const int *ov_arc = nullptr, const i64 *ov_cap = nullptr,
           long long ov_n = 0) {
    const int want_threads = o.threads > 0 ? o.threads : 512;
    if (!g->dev.ok || g->dev.threads != want_threads) {
        int rc = dev_info(g->dev, want_threads);
        if (rc) return rc;
    }
    const int threads = g->dev.threads;
    const int max_grid = g->dev.sms * g->dev.bps;
    int G, ngroups;
    if (G_req <= 0 || G_req >= max_grid) {
        G = max_grid;
        ngroups = 1;
    } else {
        G = G_req;
        ngroups = std::max(1, max_grid / G);
    }
    ngroups = std::min(ngroups, std::max(1, nq));
    int nslots = per_query_slot ? nq : ngroups;
    if (!per_query_slot) {
        if ((int)pool.host.size() < nslots) {
            size_t fr = 0, tot = 0;
            CK(cudaMemGetInfo(&fr, &tot));
            size_t per = slot_bytes(pool.n, pool.arcs, pool.nhub);
            int fit = (int)pool.host.size() + (int)((fr * 0.85) / (double)per);
            if (fit < 1) return fail(MF_ERR_NOMEM, "admission: no HBM for a residual slot (%zu bytes)", per);
            nslots = std::min(nslots, fit);
            ngroups = nslots;
        }
        int rc = pool.grow(nslots);
        if (rc) return rc;
    } else {
        ngroups = std::min(ngroups, (int)pool.host.size());
    }
    int rc = ensure_launch_buffers(g, nq, (int)pool.host.size());
    if (rc) return rc;
    int *hp = g->h_pin;
    for (int i = 0; i < nq; ++i) {
        hp[i] = s_int[i];
        hp[nq + i] = t_int[i];
        hp[2 * nq + i] = per_query_slot ? i : 0;
    }
    CK(cudaMemcpyAsync(g->d_q, hp, sizeof(int) * 3 * (size_t)nq, cudaMemcpyHostToDevice, g->stream));
    CK(cudaMemsetAsync(g->d_err, 0, sizeof(int) * 2, g->stream));
    int ns = (int)pool.host.size();
    k_prepare_slots<<<(ns + 127) / 128, 128, 0, g->stream>>>(pool.dev, ns, g->d_clocks);
    KParams p{};
    p.graphs = g->d_graph;
    p.slots = pool.dev;
    p.G = G;
    p.nq = nq;
    p.q_s = g->d_q;
    p.q_t = g->d_q + nq;
    p.q_g = nullptr;
    p.q_slot = per_query_slot ? g->d_q + 2 * nq : nullptr;
    p.q_next = g->d_qnext;
    p.out = g->d_out;
    p.err = g->d_err;
    p.bar_limit_ns = 20ull * 1000 * 1000 * 1000;
    p.time_limit_ns = launch_time_limit_ns();
    p.o = resolve_opts(o, g->avg_deg);
    p.mode = mode;
    p.dbg = dbg;
    p.upd = d_upd;
    p.nupd = nupd;
    p.ov_arc = ov_arc;
    p.ov_cap = ov_cap;
    p.ov_n = ov_n;
    int grid = ngroups * G;
    cudaError_t le = cudaSuccess;
    CK(cudaEventRecord(g->ev0, g->stream));
    mf_launch_kernel(p, grid, threads, g->stream, G > 1, &le);
    if (le != cudaSuccess) return fail(MF_ERR_CUDA, "mf_kernel launch (grid %d x %d): %s", grid, threads, cudaGetErrorString(le));
    CK(cudaEventRecord(g->ev1, g->stream));
    CK(cudaMemcpyAsync(g->h_out, g->d_out, sizeof(QOut) * nq, cudaMemcpyDeviceToHost, g->stream));
    int herr[2] = {0, 0};
    CK(cudaMemcpyAsync(herr, g->d_err, sizeof(int) * 2, cudaMemcpyDeviceToHost, g->stream));
    CK(cudaStreamSynchronize(g->stream));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, g->ev0, g->ev1));
    g->last_ms = ms;
    g->launches++;
    if (herr[0] != 0) {
        // bounded wait expired somewhere: reset barriers, report
        return fail(status_from_err(herr[0]), "device solve aborted (status %d)", herr[0]);
    }
    if (outs) memcpy(outs, g->h_out, sizeof(QOut) * nq);
    // clock housekeeping: reset slots whose stamp clock passed 2^30
    if ((g->launches & 15) == 0) {
        std::vector<unsigned> clk(ns);
        CK(down(g, clk.data(), g->d_clocks, sizeof(unsigned) * ns));
        for (int i = 0; i < ns; ++i)
            if (clk[i] > (1u << 30)) k_reset_slot<<<256, 256, 0, g->stream>>>(pool.host[i], pool.n);
        CK(cudaStreamSynchronize(g->stream));
    }
    return MF_OK;
}

void fill_stats(mf_stats *st, const QOut &q, double ms, u64 launch_t0) {
    memset(st, 0, sizeof(*st));
    st->service_ms = (double)(q.t_done - q.t_begin) * 1e-6;
    st->prune_ms = (double)q.t_prune * 1e-6;
    st->relabel_ms = (double)q.t_relabel * 1e-6;
    st->rounds_ms = (double)q.t_rounds * 1e-6;
    st->relabel_arcs = q.arcs_relabel;
    st->hub_arcs = q.arcs_hubs;
    st->hub_passes = q.hub_passes;
    st->hub_relabels = q.hub_relabels;
    st->levels = q.levels;
    st->levels_bottom_up = q.levels_bottom_up;
    st->levels_solo = q.levels_solo;
    st->local_relabels = q.local_relabels;
    st->finish_ms = launch_t0 ? (double)(q.t_done - launch_t0) * 1e-6 : 0.0;
    st->flow = q.flow;
    st->status = status_from_err(q.status);
    st->mask_vertices = q.mask_n;
    st->mask_arcs = q.mask_arcs;
    st->rounds = q.rounds;
    st->global_relabels = q.relabels;
    st->arcs_examined = q.arcs_ex;
    st->vertices_examined = q.verts_ex;
    st->pushes = q.pushes;
    st->rm_fixed = q.rm_fixed;
    st->path_push_rounds = q.pp_rounds;
    st->hot_sweeps = q.hot_sweeps;
    st->deficit_phases = q.deficit_phases;
    st->cut_capacity = q.cut;
    st->time_ms = ms;
}

int to_internal(const mf_graph *g, int s, int t, int &si, int &ti) {
    if (s < 0 || s >= g->n || t < 0 || t >= g->n || s == t) {
        si = ti = -1;
        return 0;
    }
    si = g->new_id[s];
    ti = g->new_id[t];
    return 1;
}

// File -> device copy through two pinned staging buffers: each chunk's copy
// overlaps the next chunk's read.
struct FileStream {
    unsigned char *pin[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
    cudaStream_t st = nullptr;
    size_t chunk = 16u << 20;
    int k = 0;
    bool init(cudaStream_t s) {
        st = s;
        return mf_hmalloc(&pin[0], chunk) == cudaSuccess && mf_hmalloc(&pin[1], chunk) == cudaSuccess &&
               cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming) == cudaSuccess &&
               cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming) == cudaSuccess;
    }
    // reads up to `bytes` from f into dst; returns the bytes copied
    size_t copy(FILE *f, void *dst, size_t bytes) {
        size_t got = 0;
        while (got < bytes) {
            const int b = k & 1;
            if (k >= 2) cudaEventSynchronize(done[b]);
            size_t want = std::min(chunk, bytes - got);
            size_t r = fread(pin[b], 1, want, f);
            if (r == 0) break;
            if (cudaMemcpyAsync((unsigned char *)dst + got, pin[b], r, cudaMemcpyHostToDevice, st) != cudaSuccess)
                break;
            cudaEventRecord(done[b], st);
            ++k;
            got += r;
        }
        return got;
    }
    ~FileStream() {
        if (st) cudaStreamSynchronize(st);
        mf_hfree(pin[0]);
        mf_hfree(pin[1]);
        if (done[0]) cudaEventDestroy(done[0]);
        if (done[1]) cudaEventDestroy(done[1]);
    }
};

// A graph object with its stream and events, no arrays yet.
int new_graph(int n, mf_graph **out) {
    mf_graph *g = new mf_graph();
    g->n = n;
    cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete g;
        return fail(MF_ERR_CUDA, "no CUDA device usable: %s", cudaGetErrorString(e));
    }
    cudaEventCreate(&g->ev0);
    cudaEventCreate(&g->ev1);
    *out = g;
    return MF_OK;
}

// Graph from device edge arrays (caller ids, the reference reader's skip
// rules): device CSR in input order, then partition + reorder.
int graph_from_device_edges(int n, i64 m, const int *du, const int *dv, const i64 *dc, int R,
                            mf_graph **out) {
    *out = nullptr;
    if (R <= 0) R = 128;
    R = std::min(std::min(R, n), 1024);
    mf_graph *g = nullptr;
    int rc = new_graph(n, &g);
    if (rc) return rc;
    DevCsr csr;
    cudaError_t e = mf_device_csr(n, m, du, dv, dc, g->stream, csr);
    if (e != cudaSuccess) {
        mf_graph_destroy(g);
        return fail(e == cudaErrorMemoryAllocation ? MF_ERR_NOMEM : MF_ERR_CUDA, "device CSR build failed: %s",
                    cudaGetErrorString(e));
    }
    g->arcs = csr.arcs;
    g->avg_deg = (int)(g->arcs / n);
    std::vector<int> ident(n);
    for (int i = 0; i < n; ++i) ident[i] = i;
    rc = partition_into(g, R, csr.row, csr.col, csr.cap, csr.rev, csr.fwd, ident);
    mf_free_dev_csr(csr);
    if (rc != MF_OK) {
        mf_graph_destroy(g);
        return rc;
    }
    g->pool.n = n;
    g->pool.arcs = g->arcs;
    g->pool.nhub = g->nhub;
    *out = g;
    return MF_OK;
}

}  // namespace

// Sets the text returned by mf_last_error_string() on the calling thread
// (used by entry points implemented in other translation units).
void mf_set_last_error(const char *msg) { g_err = msg ? msg : ""; }

// ---- allocation wrapper (mf_alloc.h) -------------------------------------
namespace {
std::mutex g_alloc_mu;
std::unordered_map<void *, size_t> g_alloc_live;  // live allocation -> bytes
long long g_alloc_bytes = 0;
long long g_alloc_fail_after = -1;  // allocations left before an injected failure (-1: none)

// true: this allocation is the injected failure
bool alloc_inject() {
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    if (g_alloc_fail_after < 0) return false;
    if (g_alloc_fail_after == 0) {
        g_alloc_fail_after = -1;
        return true;
    }
    --g_alloc_fail_after;
    return false;
}
void alloc_track(void *p, size_t bytes) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    g_alloc_live[p] = bytes;
    g_alloc_bytes += (long long)bytes;
}
void alloc_untrack(void *p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    auto it = g_alloc_live.find(p);
    if (it == g_alloc_live.end()) return;
    g_alloc_bytes -= (long long)it->second;
    g_alloc_live.erase(it);
}
}  // namespace

cudaError_t mf_dmalloc_raw(void **p, size_t bytes) {
    *p = nullptr;
    if (alloc_inject()) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaSuccess) alloc_track(*p, bytes);
    return e;
}
cudaError_t mf_dfree(void *p) {
    alloc_untrack(p);
    return cudaFree(p);
}
cudaError_t mf_dmalloc_async_raw(void **p, size_t bytes, cudaStream_t st) {
    *p = nullptr;
    if (alloc_inject()) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMallocAsync(p, bytes, st);
    if (e == cudaSuccess) alloc_track(*p, bytes);
    return e;
}
cudaError_t mf_dfree_async(void *p, cudaStream_t st) {
    alloc_untrack(p);
    return p ? cudaFreeAsync(p, st) : cudaSuccess;
}
cudaError_t mf_hmalloc_raw(void **p, size_t bytes) {
    *p = nullptr;
    if (alloc_inject()) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMallocHost(p, bytes);
    if (e == cudaSuccess) alloc_track(*p, bytes);
    return e;
}
cudaError_t mf_hostalloc_raw(void **p, size_t bytes, unsigned flags) {
    *p = nullptr;
    if (alloc_inject()) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaHostAlloc(p, bytes, flags);
    if (e == cudaSuccess) alloc_track(*p, bytes);
    return e;
}
cudaError_t mf_hfree(void *p) {
    alloc_untrack(p);
    return cudaFreeHost(p);
}

extern "C" int mf_debug_alloc_fail_after(long long k) {
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    g_alloc_fail_after = k < 0 ? -1 : k;
    return MF_OK;
}

extern "C" int mf_debug_alloc_live(long long *count, long long *bytes, long long *fail_after) {
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    if (count) *count = (long long)g_alloc_live.size();
    if (bytes) *bytes = g_alloc_bytes;
    if (fail_after) *fail_after = g_alloc_fail_after;
    return MF_OK;
}

// Option resolution, the launch time limit and the device-status mapping,
// shared with entry points in other translation units so that every entry
// point resolves options and reports device statuses alike.
KOpts mf_resolve_opts(const mf_opts &o, int avg_deg) { return resolve_opts(o, avg_deg); }
u64 mf_launch_time_limit_ns() { return launch_time_limit_ns(); }
int mf_status_from_err(int e) { return status_from_err(e); }

// ===========================================================================
extern "C" {

void mf_opts_default(mf_opts *o) {
    memset(o, 0, sizeof(*o));
    o->kernel_cycles = 0;
    o->gr_freq = 16;         // RA:1466 starts at 128; exact relabels are cheap here
    o->gr_work_alpha = 0.35; // also relabel after ~a third of a pass over the kept arcs
    o->prune_mode = 1;
    o->path_push_switch = 8;  // PATH_PUSH_SWITCH (RA:1480)
    o->max_path_len = 256;    // MAX_PATH_LENGTH (RA:1481)
    o->use_path_push = 1;
    o->use_hot_sweep = 1;
    o->hot_regions = 32;  // RA:1936
    o->use_rm = 1;
    o->rm_freq = 64;   // RM_FREQ0 (RA:1468)
    o->h_cut = 100;    // H_cut (RA:1470)
    o->stagnate_rounds = 128;  // STAGNATE_ROUNDS (RA:1472)
    o->iter_max = 20000000;    // ITER_MAX (RA:1476)
    o->group_ctas = 0;
    o->threads = 512;
    o->certify = 0;
    o->verbose = 0;
    o->use_kept_cache = 1;
    o->schedule = 1;
    o->relabel_early_stop = 1;
    o->local_relabel = 0;
}

const char *mf_last_error_string(void) { return g_err.c_str(); }
const char *mf_version(void) { return "mscresearch_b200 maxflow 0.1 (sm_100a)"; }

int mf_graph_create_from_edges(int n, long long m, const int32_t *u, const int32_t *v,
                               const int64_t *cap, int R, mf_graph **out) {
    if (!out) return fail(MF_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (n <= 0) return fail(MF_ERR_ARG, "n must be positive (got %d)", n);
    if (m < 0 || (m > 0 && (!u || !v || !cap))) return fail(MF_ERR_ARG, "bad edge arrays");
    if (2 * m > 0x7fffffffLL) return fail(MF_ERR_ARG, "too many edges for int32 arc ids");
    int *du = nullptr, *dv = nullptr;
    i64 *dc = nullptr;
    const size_t M = (size_t)std::max<long long>(m, 1);
    int rc = MF_OK;
    if (mf_dmalloc(&du, sizeof(int) * M) != cudaSuccess || mf_dmalloc(&dv, sizeof(int) * M) != cudaSuccess ||
        mf_dmalloc(&dc, sizeof(i64) * M) != cudaSuccess) {
        cudaGetLastError();
        rc = fail(MF_ERR_NOMEM, "edge upload allocation failed (%lld edges)", m);
    } else if (m > 0 && (cudaMemcpy(du, u, sizeof(int) * m, cudaMemcpyHostToDevice) != cudaSuccess ||
                         cudaMemcpy(dv, v, sizeof(int) * m, cudaMemcpyHostToDevice) != cudaSuccess ||
                         cudaMemcpy(dc, cap, sizeof(i64) * m, cudaMemcpyHostToDevice) != cudaSuccess)) {
        rc = fail(MF_ERR_CUDA, "edge upload failed");
    } else if (cudaStreamSynchronize(0) != cudaSuccess) {  // the uploads' DMA has landed
        rc = fail(MF_ERR_CUDA, "edge upload failed");
    } else {
        rc = graph_from_device_edges(n, m, du, dv, dc, R, out);
    }
    mf_dfree(du);
    mf_dfree(dv);
    mf_dfree(dc);
    return rc;
}

int mf_graph_create_from_device_edges(int n, long long m, const int32_t *d_u, const int32_t *d_v,
                                      const int64_t *d_cap, int R, mf_graph **out) {
    if (!out) return fail(MF_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (n <= 0) return fail(MF_ERR_ARG, "n must be positive (got %d)", n);
    if (m < 0 || (m > 0 && (!d_u || !d_v || !d_cap))) return fail(MF_ERR_ARG, "bad edge arrays");
    if (2 * m > 0x7fffffffLL) return fail(MF_ERR_ARG, "too many edges for int32 arc ids");
    return graph_from_device_edges(n, m, d_u, d_v, reinterpret_cast<const i64 *>(d_cap), R, out);
}

int mf_graph_load_file(const char *path, int R, mf_graph **out) {
    if (!out || !path) return fail(MF_ERR_ARG, "path or out is NULL");
    *out = nullptr;
    FILE *f = fopen(path, "rb");
    if (!f) return fail(MF_ERR_IO, "cannot open %s", path);
    fseek(f, 0, SEEK_END);
    long long S = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (S < 0) S = 0;
    // token indices are 32-bit: a file below 4 GiB holds fewer than 2^31
    // integers (each takes a digit and a separator)
    if (S >= (4LL << 30)) {
        fclose(f);
        return fail(MF_ERR_ARG, "%s is %lld bytes; text graphs of 4 GiB or more are not read (pass edge arrays "
                                "or a binary CSR cache)", path, S);
    }
    unsigned char *dtxt = nullptr;
    cudaStream_t st = nullptr;
    int rc = MF_OK;
    long long got = 0;
    TextEdges te;
    do {
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
            mf_dmalloc(&dtxt, (size_t)std::max<long long>(S, 1)) != cudaSuccess) {
            cudaGetLastError();
            rc = fail(MF_ERR_NOMEM, "text staging for %lld bytes failed", S);
            break;
        }
        {
            FileStream fs;
            if (!fs.init(st)) {
                cudaGetLastError();
                rc = fail(MF_ERR_NOMEM, "pinned staging failed");
                break;
            }
            got = (long long)fs.copy(f, dtxt, (size_t)S);
        }
        if (got != S) {
            rc = fail(MF_ERR_IO, "read of %s stopped at byte %lld of %lld", path, got, S);
            break;
        }
        cudaError_t e = mf_parse_graph_text(dtxt, got, st, te);
        if (e != cudaSuccess) {
            rc = fail(e == cudaErrorMemoryAllocation ? MF_ERR_NOMEM : MF_ERR_CUDA, "graph text parse failed: %s",
                      cudaGetErrorString(e));
            break;
        }
        if (!te.header_ok || te.n <= 0 || te.m_header < 0) {
            rc = fail(MF_ERR_IO, "%s: no valid \"n m\" header", path);
            break;
        }
        mf_dfree(dtxt);
        dtxt = nullptr;
        if (2 * te.m > 0x7fffffffLL) {
            rc = fail(MF_ERR_ARG, "too many edges for int32 arc ids");
            break;
        }
        rc = graph_from_device_edges(te.n, te.m, te.u, te.v, te.c, R, out);
    } while (0);
    fclose(f);
    mf_free_text_edges(te);
    mf_dfree(dtxt);
    if (st) cudaStreamDestroy(st);
    return rc;
}

int mf_graph_repartition(mf_graph *g, int R) {
    if (!g) return fail(MF_ERR_ARG, "graph is NULL");
    if (R <= 0) R = 128;
    R = std::min(std::min(R, g->n), 1024);
    if (R == g->R) return MF_OK;
    // current region-ordered arrays become the input; their vertex i is
    // caller vertex old_id[i]
    int *row = g->row, *col = g->col, *rev = g->rev;
    i64 *cap = g->cap;
    unsigned char *fwd = g->fwd;
    int *ro = g->region_of, *rs = g->region_start;
    DGraph *dg = g->d_graph;
    g->row = g->col = g->rev = g->region_of = g->region_start = nullptr;
    g->cap = nullptr;
    g->fwd = nullptr;
    g->d_graph = nullptr;
    std::vector<int> in_to_caller = g->old_id;
    int rc = partition_into(g, R, row, col, cap, rev, fwd, in_to_caller);
    mf_dfree(row);
    mf_dfree(col);
    mf_dfree(rev);
    mf_dfree(cap);
    mf_dfree(fwd);
    mf_dfree(ro);
    mf_dfree(rs);
    mf_dfree(dg);
    return rc;
}

int mf_graph_destroy(mf_graph *g) {
    if (!g) return MF_OK;
    free_graph_arrays(g);
    g->pool.release();
    mf_dfree(g->d_err);
    mf_dfree(g->d_clocks);
    mf_dfree(g->d_out);
    mf_dfree(g->d_q);
    mf_hfree(g->h_pin);
    mf_hfree(g->h_out);
    if (g->ev0) cudaEventDestroy(g->ev0);
    if (g->ev1) cudaEventDestroy(g->ev1);
    if (g->stream) cudaStreamDestroy(g->stream);
    delete g;
    return MF_OK;
}

int mf_graph_info(const mf_graph *g, int *n, long long *arcs, int *R) {
    if (!g) return fail(MF_ERR_ARG, "graph is NULL");
    if (n) *n = g->n;
    if (arcs) *arcs = g->arcs;
    if (R) *R = g->R;
    return MF_OK;
}

int mf_graph_scc(mf_graph *g, int32_t *comp, int32_t *ncomp, long long *m_contracted) {
    if (!g) return fail(MF_ERR_ARG, "graph is NULL");
    SccIn in{g->n, g->arcs, g->row, g->col, g->rev, g->cap, g->new_id.data(), g->old_id.data()};
    g->scc_done = false;
    CK(mf_scc_run(in, g->stream, g->scc));
    g->scc_done = true;
    if (comp) memcpy(comp, g->scc.comp.data(), sizeof(int) * (size_t)g->n);
    if (ncomp) *ncomp = g->scc.ncomp;
    if (m_contracted) *m_contracted = (long long)g->scc.cu.size();
    return MF_OK;
}

int mf_graph_scc_contracted(const mf_graph *g, int32_t *cu, int32_t *cv, int64_t *cap, long long max) {
    if (!g) return fail(MF_ERR_ARG, "graph is NULL");
    if (!g->scc_done) return fail(MF_ERR_ARG, "mf_graph_scc has not run on this graph");
    const size_t K = g->scc.cu.size();
    if (max < (long long)K) return fail(MF_ERR_ARG, "room for %lld contracted arcs, %zu needed", max, K);
    if (K == 0) return MF_OK;
    if (!cu || !cv || !cap) return fail(MF_ERR_ARG, "NULL output array");
    memcpy(cu, g->scc.cu.data(), sizeof(int) * K);
    memcpy(cv, g->scc.cv.data(), sizeof(int) * K);
    memcpy(cap, g->scc.cap.data(), sizeof(int64_t) * K);
    return MF_OK;
}

int mf_graph_export(const mf_graph *g, int32_t *row, int32_t *col, int64_t *cap, int32_t *rev,
                    int32_t *new_id, int32_t *region_start, double *score, int32_t *part) {
    if (!g) return fail(MF_ERR_ARG, "graph is NULL");
    if (row) CK(down(g, row, g->row, sizeof(int) * ((size_t)g->n + 1)));
    if (col && g->arcs) CK(down(g, col, g->col, sizeof(int) * g->arcs));
    if (cap && g->arcs) CK(down(g, cap, g->cap, sizeof(i64) * g->arcs));
    if (rev && g->arcs) CK(down(g, rev, g->rev, sizeof(int) * g->arcs));
    if (region_start)
        CK(down(g, region_start, g->region_start, sizeof(int) * ((size_t)g->R + 1)));
    if (new_id) memcpy(new_id, g->new_id.data(), sizeof(int) * g->n);
    if (score) memcpy(score, g->score_caller.data(), sizeof(double) * g->n);
    if (part) memcpy(part, g->part_caller.data(), sizeof(int) * g->n);
    return MF_OK;
}

// ---- binary CSR cache ------------------------------------------------------
// File: CacheHead, then row[n+1] i32, col[A] i32, cap[A] i64, rev[A] i32,
// fwd[A] u8, region_start[R+1] i32, region_of[n] i32 (region-ordered CSR),
// new_id[n] i32, score[n] f64, part[n] i32 (caller ids); native byte order.
struct CacheHead {
    char magic[8];
    int32_t version;
    int32_t n;
    int64_t arcs;
    int32_t R;
    int32_t pad;
    int64_t bytes;  // whole file
};
static const char kCacheMagic[8] = {'M', 'F', 'B', '2', '0', '0', 'C', 'S'};

static int64_t cache_bytes(int n, i64 A, int R) {
    return (int64_t)sizeof(CacheHead) + 4 * ((int64_t)n + 1) + 4 * A + 8 * A + 4 * A + A + 4 * ((int64_t)R + 1) +
           4 * (int64_t)n + 4 * (int64_t)n + 8 * (int64_t)n + 4 * (int64_t)n;
}

// Consistency of a loaded region-ordered CSR (row and region starts already
// checked monotone on the host): a warp per vertex over its arcs -- heads in
// range, rev an involution pairing opposite arcs, one forward arc per pair,
// capacities >= 0 and 0 on reverse arcs, region ranges covering each vertex.
// Counts violations.
__global__ void k_check_csr(int n, i64 A, int R, const int *row, const int *col, const i64 *cap, const int *rev,
                            const unsigned char *fwd, const int *region_start, const int *region_of, int *bad) {
    const int lane = threadIdx.x & 31;
    const int w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    int nb = 0;
    if (w0 == 0 && lane == 0) {
        if (row[0] != 0 || (i64)row[n] != A) ++nb;
        if (region_start[0] != 0 || region_start[R] != n) ++nb;
    }
    for (int x = w0; x < n; x += nw) {
        const int b = row[x], e1 = row[x + 1];
        if (lane == 0) {
            int r = region_of[x];
            if (r < 0 || r >= R || region_start[r] > x || region_start[r + 1] <= x) ++nb;
        }
        if (b < 0 || (i64)e1 > A) {
            if (lane == 0) ++nb;
            continue;
        }
        for (int e = b + lane; e < e1; e += 32) {
            int w = col[e], re = rev[e];
            if (w < 0 || w >= n || w == x || re < 0 || (i64)re >= A) {
                ++nb;
                continue;
            }
            if (rev[re] != e || col[re] != x || fwd[e] == fwd[re] || cap[e] < 0 || (!fwd[e] && cap[e] != 0)) ++nb;
        }
    }
    if (nb) atomicAdd(bad, nb);
}

// kc_res[e] = cap[e] if both ends of e are in the component, else 0;
// kc_arcs = arcs out of component vertices.
__global__ void k_kept_res(int n, const int *row, const int *col, const i64 *cap,
                           const unsigned char *in, i64 *res, unsigned long long *arcs) {
    int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    int nw = (gridDim.x * blockDim.x) >> 5;
    unsigned long long mine = 0;
    for (int v = w; v < n; v += nw) {
        bool iv = in[v];
        int b = row[v], e1 = row[v + 1];
        for (int e = b + lane; e < e1; e += 32) res[e] = (iv && in[col[e]]) ? cap[e] : 0;
        if (iv && lane == 0) mine += (unsigned long long)(e1 - b);
    }
    if (lane == 0 && mine) atomicAdd(arcs, mine);
}

// Builds the kept-set cache once per graph state (prune mode 1 only): the
// strongly connected component of the highest-degree vertex, found by the
// solver's own prune with s = t = pivot, and the pivot's forward / backward
// closures (F / B bits per vertex).
static int build_kept_cache(mf_graph *g, const mf_opts &o);

// Builds the kept-set cache on first use.  Any failure frees what the build
// allocated and marks the cache as tried: the error is returned once and
// later solves run without the cache.
static int ensure_kept_cache(mf_graph *g, const mf_opts &o) {
    if (g->kc_valid || g->kc_tried || o.prune_mode != 1 || !o.use_kept_cache) return MF_OK;
    int rc = build_kept_cache(g, o);
    if (rc) {
        free_kept_cache(g);
        g->kc_tried = true;
        upload_dgraph(g);
    }
    return rc;
}

static int build_kept_cache(mf_graph *g, const mf_opts &o) {
    g->kc_tried = true;
    int n = g->n;
    KcOut ko{};
    // buffers kept from an invalidated cache are reused
    if (!g->kc_in) CK(mf_dmalloc(&g->kc_in, n));
    if (!g->kc_img) CK(mf_dmalloc(&g->kc_img, sizeof(int) * (size_t)n));
    if (!g->kc_res) CK(mf_dmalloc(&g->kc_res, sizeof(i64) * (size_t)std::max<i64>(g->arcs, 1)));
    CK(zero(g, g->kc_in, n));
    if (!g->kc_fb) CK(mf_dmalloc(&g->kc_fb, n));
    ko.img = g->kc_img;
    ko.in = g->kc_in;
    ko.fb = g->kc_fb;
    KcOut *dko = nullptr;
    CK(mf_dmalloc(&dko, sizeof(KcOut)));
    if (up(g, dko, &ko, sizeof(KcOut)) != cudaSuccess) {
        mf_dfree(dko);
        return fail(MF_ERR_CUDA, "kept-set cache set-up copy failed");
    }
    int piv = g->pivot;
    QOut out;
    int rc = launch(g, g->pool, 1, &piv, &piv, false, o, KM_KEPTSET, dko, nullptr, 0, 0, &out);
    mf_dfree(dko);
    if (rc) return rc;
    g->kc_f = out.kept_front;
    g->kc_b = out.mask_n - out.kept_front;
    unsigned long long *darcs = nullptr;
    DevScope tmp;
    CK(tmp.alloc(&darcs, sizeof(unsigned long long)));
    CK(zero(g, darcs, sizeof(unsigned long long)));
    k_kept_res<<<g->dev.sms * 8, 256, 0, g->stream>>>(n, g->row, g->col, g->cap, g->kc_in, g->kc_res, darcs);
    unsigned long long ka = 0;
    CK(cudaMemcpyAsync(&ka, darcs, sizeof(ka), cudaMemcpyDeviceToHost, g->stream));
    CK(cudaStreamSynchronize(g->stream));
    g->kc_arcs = (i64)ka;
    g->kc_valid = out.mask_n >= 2;
    if (g->kc_valid) {
        g->kc_in_host.resize(n);
        CK(down(g, g->kc_in_host.data(), g->kc_in, n));
        // The image in vertex order (the search left it in discovery
        // order): the queries that take it sweep their kept list in every
        // relabel and worklist pass, and consecutive ids share the rows,
        // heights and arc ranges those passes read.  Front part: vertices
        // with at most HUB_T arcs; back part (from the end down): the hubs.
        // On the headline batch: 94.3 -> 90 ms per batch.
        {
            std::vector<int> img((size_t)n);
            int f = 0, b = 0;
            for (int v = 0; v < n; ++v) {
                if (!g->kc_in_host[v]) continue;
                if (g->deg_host[v] > HUB_T) img[(size_t)n - 1 - b++] = v;
                else img[f++] = v;
            }
            if (f == g->kc_f && b == g->kc_b) {
                CK(up(g, g->kc_img, img.data(), sizeof(int) * (size_t)f));
                if (b) CK(up(g, g->kc_img + (n - b), img.data() + (n - b), sizeof(int) * (size_t)b));
                CK(cudaStreamSynchronize(g->stream));
            }
        }
    }
    if (!g->kc_valid) {
        bool tried = true;
        free_kept_cache(g);
        g->kc_tried = tried;
        return MF_OK;
    }
    return upload_dgraph(g);
}

// Queue order for a batch: queries whose s and t are both in the cached
// component first (their kept set is the whole component), then the rest;
// within each class, larger min(deg s, deg t) first (the flow, and with it
// the push work, is bounded by the smaller end).  Invalid queries last.
static std::vector<int> cost_order(const mf_graph *g, int nq, const int *si, const int *ti, const mf_opts &o) {
    std::vector<long long> key(nq);
    bool kc = g->kc_valid && o.use_kept_cache && o.prune_mode == 1 && !g->kc_in_host.empty();
    for (int i = 0; i < nq; ++i) {
        int a = si[i], b = ti[i];
        if (a < 0 || b < 0 || a == b || g->deg_host.empty()) {
            key[i] = -1;
            continue;
        }
        long long k = std::min(g->deg_host[a], g->deg_host[b]);
        if (kc && g->kc_in_host[a] && g->kc_in_host[b]) k += 1LL << 40;
        key[i] = k;
    }
    std::vector<int> perm(nq);
    for (int i = 0; i < nq; ++i) perm[i] = i;
    std::stable_sort(perm.begin(), perm.end(), [&](int x, int y) { return key[x] > key[y]; });
    return perm;
}

static int solve_common(mf_graph *g, int nq, const int32_t *s, const int32_t *t, const mf_opts *opts,
                        int64_t *flows, mf_stats *stats, int mode, void *dbg, bool single) {
    if (!g) return fail(MF_ERR_ARG, "graph is NULL");
    if (nq < 0 || (nq > 0 && (!s || !t || !flows))) return fail(MF_ERR_ARG, "bad query arrays");
    if (nq == 0) return MF_OK;
    mf_opts o;
    if (opts) o = *opts;
    else mf_opts_default(&o);
    // opts.certify: every answer also returns its excess to s and is checked
    // on the device (zero-excess flow, equal-capacity s-t cut)
    if (o.certify && mode == KM_SOLVE) mode = KM_CERTIFY;
    std::vector<int> si(nq), ti(nq);
    for (int i = 0; i < nq; ++i) to_internal(g, s[i], t[i], si[i], ti[i]);
    int rc0 = ensure_kept_cache(g, o);
    if (rc0) return rc0;
    std::vector<QOut> outs(nq);
    int G = single ? 0 : (o.group_ctas > 0 ? o.group_ctas : 8);
    // batched: queue order by expected cost (largest first), results unpermuted
    std::vector<int> perm;
    if (!single && o.schedule && nq > 1 && (mode == KM_SOLVE || mode == KM_CERTIFY)) {
        perm = cost_order(g, nq, si.data(), ti.data(), o);
        std::vector<int> s2(nq), t2(nq);
        for (int i = 0; i < nq; ++i) {
            s2[i] = si[perm[i]];
            t2[i] = ti[perm[i]];
        }
        si.swap(s2);
        ti.swap(t2);
    }
    int rc = launch(g, g->pool, nq, si.data(), ti.data(), false, o, mode, dbg, nullptr, 0, G, outs.data());
    if (rc) return rc;
    if (!perm.empty()) {
        std::vector<QOut> o2(nq);
        for (int i = 0; i < nq; ++i) o2[perm[i]] = outs[i];
        outs.swap(o2);
    }
    int worst = MF_OK;
    u64 t0min = ~0ull;
    for (int i = 0; i < nq; ++i) t0min = std::min(t0min, outs[i].t_begin);
    for (int i = 0; i < nq; ++i) {
        flows[i] = outs[i].flow;
        if (stats) fill_stats(&stats[i], outs[i], single ? g->last_ms : 0.0, t0min);
        int st = status_from_err(outs[i].status);
        if (st != MF_OK && worst == MF_OK) worst = st;
        if (o.verbose)
            fprintf(stderr, "[mf] q=%d s=%d t=%d flow=%lld kept=%d rounds=%lld relabels=%lld status=%d\n",
                    i, s[i], t[i], (long long)outs[i].flow, outs[i].mask_n, (long long)outs[i].rounds,
                    (long long)outs[i].relabels, outs[i].status);
    }
    if (worst != MF_OK) return fail(worst, "a query ended with status %d", worst);
    return MF_OK;
}

int mf_solve(mf_graph *g, int32_t s, int32_t t, const mf_opts *opts, int64_t *flow, mf_stats *stats) {
    int64_t f = 0;
    int rc = solve_common(g, 1, &s, &t, opts, &f, stats, KM_SOLVE, nullptr, true);
    if (flow) *flow = f;
    return rc;
}

int mf_solve_batch(mf_graph *g, int nq, const int32_t *s, const int32_t *t, const mf_opts *opts,
                   int64_t *flows, mf_stats *stats) {
    return solve_common(g, nq, s, t, opts, flows, stats, KM_SOLVE, nullptr, false);
}

int mf_solve_batch_override(mf_graph *g, int nq, const int32_t *s, const int32_t *t, long long narcs,
                            const int32_t *u, const int32_t *v, const int64_t *caps, const mf_opts *opts,
                            int64_t *flows, mf_stats *stats) {
    if (!g) return fail(MF_ERR_ARG, "graph is NULL");
    if (nq < 0 || narcs < 0 || narcs > 0x7fffffffLL || (nq > 0 && (!s || !t || !flows)) ||
        (narcs > 0 && nq > 0 && (!u || !v || !caps)))
        return fail(MF_ERR_ARG, "bad query or override arrays");
    if (nq == 0) return MF_OK;
    if (narcs == 0) return mf_solve_batch(g, nq, s, t, opts, flows, stats);
    mf_opts o;
    if (opts) o = *opts;
    else mf_opts_default(&o);
    if (o.certify) return fail(MF_ERR_ARG, "certify is not available with capacity overrides");
    const int nb = (int)narcs;
    std::vector<int> iu(nb), iv(nb);
    for (int j = 0; j < nb; ++j) {
        iu[j] = (u[j] >= 0 && u[j] < g->n) ? g->new_id[u[j]] : -1;
        iv[j] = (v[j] >= 0 && v[j] < g->n) ? g->new_id[v[j]] : -1;
    }
    int *du = nullptr, *dv = nullptr, *darc = nullptr, *dbad = nullptr;
    i64 *dgcap = nullptr, *dov = nullptr;
    const size_t ovn = (size_t)nq * (size_t)nb;
    int rc = MF_OK;
    do {
        if (mf_dmalloc(&du, sizeof(int) * nb) != cudaSuccess || mf_dmalloc(&dv, sizeof(int) * nb) != cudaSuccess ||
            mf_dmalloc(&darc, sizeof(int) * nb) != cudaSuccess || mf_dmalloc(&dgcap, sizeof(i64) * nb) != cudaSuccess ||
            mf_dmalloc(&dov, sizeof(i64) * ovn) != cudaSuccess || mf_dmalloc(&dbad, sizeof(int)) != cudaSuccess) {
            cudaGetLastError();
            rc = fail(MF_ERR_NOMEM, "override buffers (%zu capacities) do not fit", ovn);
            break;
        }
        if (up(g, du, iu.data(), sizeof(int) * nb) != cudaSuccess ||
            up(g, dv, iv.data(), sizeof(int) * nb) != cudaSuccess ||
            up(g, dov, caps, sizeof(i64) * ovn) != cudaSuccess || zero(g, dbad, sizeof(int)) != cudaSuccess) {
            rc = fail(MF_ERR_CUDA, "override upload failed");
            break;
        }
        k_find_arcs<<<(unsigned)((nb + 7) / 8), 256, 0, g->stream>>>(nb, du, dv, g->row, g->col, g->rev, g->fwd, g->cap,
                                                              darc, dgcap);
        k_check_overrides<<<(unsigned)((ovn + 255) / 256), 256, 0, g->stream>>>(nb, nq, darc, dgcap, dov, dbad);
        int hbad = 0;
        if (cudaMemcpyAsync(&hbad, dbad, sizeof(int), cudaMemcpyDeviceToHost, g->stream) != cudaSuccess ||
            cudaStreamSynchronize(g->stream) != cudaSuccess) {
            rc = fail(MF_ERR_CUDA, "override check failed: %s", cudaGetErrorString(cudaGetLastError()));
            break;
        }
        if (hbad) {
            rc = fail(MF_ERR_ARG, "%d override entries name no forward arc or lie outside [0, the arc's capacity]",
                      hbad);
            break;
        }
        std::vector<int> si(nq), ti(nq);
        for (int i = 0; i < nq; ++i) to_internal(g, s[i], t[i], si[i], ti[i]);
        if ((rc = ensure_kept_cache(g, o))) break;
        std::vector<QOut> outs(nq);
        const int G = o.group_ctas > 0 ? o.group_ctas : 8;
        if ((rc = launch(g, g->pool, nq, si.data(), ti.data(), false, o, KM_SOLVE, nullptr, nullptr, 0, G,
                         outs.data(), darc, dov, narcs)))
            break;
        int worst = MF_OK;
        u64 t0min = ~0ull;
        for (int i = 0; i < nq; ++i) t0min = std::min(t0min, outs[i].t_begin);
        for (int i = 0; i < nq; ++i) {
            flows[i] = outs[i].flow;
            if (stats) fill_stats(&stats[i], outs[i], 0.0, t0min);
            int st = status_from_err(outs[i].status);
            if (st != MF_OK && worst == MF_OK) worst = st;
        }
        if (worst != MF_OK) rc = fail(worst, "a query ended with status %d", worst);
    } while (0);
    mf_dfree(du);
    mf_dfree(dv);
    mf_dfree(darc);
    mf_dfree(dgcap);
    mf_dfree(dov);
    mf_dfree(dbad);
    return rc;
}

double mf_last_device_ms(const mf_graph *g) { return g ? g->last_ms : 0.0; }

int mf_graph_save(const mf_graph *g, const char *path) {
    if (!g || !path) return fail(MF_ERR_ARG, "graph or path is NULL");
    const int n = g->n, R = g->R;
    const i64 A = g->arcs;
    std::vector<int> row(n + 1), col(A), rev(A), rs(R + 1), ro(n);
    std::vector<i64> cap(A);
    std::vector<unsigned char> fwd(A);
    CK(down(g, row.data(), g->row, sizeof(int) * (n + 1)));
    if (A) {
        CK(down(g, col.data(), g->col, sizeof(int) * A));
        CK(down(g, cap.data(), g->cap, sizeof(i64) * A));
        CK(down(g, rev.data(), g->rev, sizeof(int) * A));
        CK(down(g, fwd.data(), g->fwd, A));
    }
    CK(down(g, rs.data(), g->region_start, sizeof(int) * (R + 1)));
    CK(down(g, ro.data(), g->region_of, sizeof(int) * n));
    CacheHead h{};
    memcpy(h.magic, kCacheMagic, 8);
    h.version = 1;
    h.n = n;
    h.arcs = A;
    h.R = R;
    h.bytes = cache_bytes(n, A, R);
    FILE *f = fopen(path, "wb");
    if (!f) return fail(MF_ERR_IO, "cannot create %s", path);
    bool ok = fwrite(&h, sizeof(h), 1, f) == 1;
    auto put = [&](const void *p, size_t bytes) {
        if (ok && bytes) ok = fwrite(p, 1, bytes, f) == bytes;
    };
    put(row.data(), 4 * row.size());
    put(col.data(), 4 * (size_t)A);
    put(cap.data(), 8 * (size_t)A);
    put(rev.data(), 4 * (size_t)A);
    put(fwd.data(), (size_t)A);
    put(rs.data(), 4 * rs.size());
    put(ro.data(), 4 * ro.size());
    put(g->new_id.data(), 4 * (size_t)n);
    put(g->score_caller.data(), 8 * (size_t)n);
    put(g->part_caller.data(), 4 * (size_t)n);
    if (fclose(f) != 0) ok = false;
    return ok ? MF_OK : fail(MF_ERR_IO, "write to %s failed", path);
}

int mf_graph_load_binary(const char *path, mf_graph **out) {
    if (!path || !out) return fail(MF_ERR_ARG, "path or out is NULL");
    *out = nullptr;
    FILE *f = fopen(path, "rb");
    if (!f) return fail(MF_ERR_IO, "cannot open %s", path);
    fseek(f, 0, SEEK_END);
    long long S = ftell(f);
    fseek(f, 0, SEEK_SET);
    CacheHead h{};
    if (fread(&h, sizeof(h), 1, f) != 1 || memcmp(h.magic, kCacheMagic, 8) != 0 || h.version != 1 || h.n <= 0 ||
        h.arcs < 0 || h.arcs > 0x7fffffffLL || h.R <= 0 || h.R > std::min(h.n, 1024) ||
        h.bytes != cache_bytes(h.n, h.arcs, h.R) || S != h.bytes) {
        fclose(f);
        return fail(MF_ERR_IO, "%s is not a CSR cache of this library (or is truncated)", path);
    }
    const int n = h.n, R = h.R;
    const i64 A = h.arcs;
    mf_graph *g = nullptr;
    int rc = new_graph(n, &g);
    if (rc) {
        fclose(f);
        return rc;
    }
    std::vector<int> row(n + 1), rs(R + 1), nid(n), part(n), old(n, -1);
    std::vector<double> score(n);
    int *dbad = nullptr;
    do {
        const size_t AA = (size_t)std::max<i64>(A, 1);
        if (mf_dmalloc(&g->row, sizeof(int) * (n + 1)) || mf_dmalloc(&g->col, sizeof(int) * AA) ||
            mf_dmalloc(&g->cap, sizeof(i64) * AA) || mf_dmalloc(&g->rev, sizeof(int) * AA) ||
            mf_dmalloc(&g->fwd, AA) || mf_dmalloc(&g->region_start, sizeof(int) * (R + 1)) ||
            mf_dmalloc(&g->region_of, sizeof(int) * n) || mf_dmalloc(&dbad, sizeof(int))) {
            cudaGetLastError();
            rc = fail(MF_ERR_NOMEM, "graph allocation failed");
            break;
        }
        // arc arrays and region ids stream to the device; the rest via the host
        bool ok = fread(row.data(), 4, (size_t)n + 1, f) == (size_t)n + 1;
        {
            FileStream fs;
            if (!fs.init(g->stream)) {
                cudaGetLastError();
                rc = fail(MF_ERR_NOMEM, "pinned staging failed");
                break;
            }
            ok = ok && fs.copy(f, g->col, 4 * (size_t)A) == 4 * (size_t)A &&
                 fs.copy(f, g->cap, 8 * (size_t)A) == 8 * (size_t)A &&
                 fs.copy(f, g->rev, 4 * (size_t)A) == 4 * (size_t)A && fs.copy(f, g->fwd, (size_t)A) == (size_t)A;
            ok = ok && fread(rs.data(), 4, (size_t)R + 1, f) == (size_t)R + 1;
            ok = ok && fs.copy(f, g->region_of, 4 * (size_t)n) == 4 * (size_t)n;
        }
        ok = ok && fread(nid.data(), 4, n, f) == (size_t)n && fread(score.data(), 8, n, f) == (size_t)n &&
             fread(part.data(), 4, n, f) == (size_t)n;
        if (!ok) {
            rc = fail(MF_ERR_IO, "read of %s failed", path);
            break;
        }
        for (int x = 0; x < n && rc == MF_OK; ++x) {
            int y = nid[x];
            if (y < 0 || y >= n || old[y] != -1) rc = fail(MF_ERR_IO, "%s: new_id is not a permutation", path);
            else old[y] = x;
        }
        // row and region monotonicity on the host (the device check indexes by them)
        for (int x = 0; x < n && rc == MF_OK; ++x)
            if (row[x] > row[x + 1]) rc = fail(MF_ERR_IO, "%s: row offsets decrease at %d", path, x);
        for (int r = 0; r < R && rc == MF_OK; ++r)
            if (rs[r] > rs[r + 1]) rc = fail(MF_ERR_IO, "%s: region starts decrease at %d", path, r);
        if (rc) break;
        if (up(g, g->row, row.data(), sizeof(int) * (n + 1)) != cudaSuccess ||
            up(g, g->region_start, rs.data(), sizeof(int) * (R + 1)) != cudaSuccess ||
            zero(g, dbad, sizeof(int)) != cudaSuccess) {
            rc = fail(MF_ERR_CUDA, "graph upload failed");
            break;
        }
        k_check_csr<<<std::max(1, std::min(g->dev.ok ? g->dev.sms * 8 : 148 * 8, (n + 7) / 8)), 256, 0,
                      g->stream>>>(n, A, R, g->row, g->col, g->cap, g->rev, g->fwd, g->region_start, g->region_of,
                                   dbad);
        int hbad = 0;
        if (cudaMemcpyAsync(&hbad, dbad, sizeof(int), cudaMemcpyDeviceToHost, g->stream) != cudaSuccess ||
            cudaStreamSynchronize(g->stream) != cudaSuccess) {
            rc = fail(MF_ERR_CUDA, "cache check failed: %s", cudaGetErrorString(cudaGetLastError()));
            break;
        }
        if (hbad) {
            rc = fail(MF_ERR_IO, "%s: %d inconsistencies in the stored CSR", path, hbad);
            break;
        }
        g->arcs = A;
        g->avg_deg = (int)(A / n);
        g->R = R;
        g->new_id.swap(nid);
        g->old_id.swap(old);
        g->score_caller.swap(score);
        g->part_caller.swap(part);
        rc = finalize_graph(g);
    } while (0);
    fclose(f);
    mf_dfree(dbad);
    if (rc != MF_OK) {
        mf_graph_destroy(g);
        return rc;
    }
    g->pool.n = n;
    g->pool.arcs = g->arcs;
    g->pool.nhub = g->nhub;
    *out = g;
    return MF_OK;
}

int mf_debug_prune_mask(mf_graph *g, int32_t s, int32_t t, const mf_opts *opts, uint8_t *mask, int *kept) {
    if (!g || !mask) return fail(MF_ERR_ARG, "bad arguments");
    unsigned char *d = nullptr;
    CK(mf_dmalloc(&d, g->n));
    CK(zero(g, d, g->n));
    int64_t f = 0;
    mf_stats st;
    int rc = solve_common(g, 1, &s, &t, opts, &f, &st, KM_PRUNE, d, true);
    if (rc == MF_OK) {
        std::vector<unsigned char> h(g->n);
        down(g, h.data(), d, g->n);
        int k = 0;
        for (int x = 0; x < g->n; ++x) {
            mask[x] = (s < 0 || t < 0 || s >= g->n || t >= g->n) ? 0 : h[g->new_id[x]];
            k += mask[x];
        }
        if (kept) *kept = k;
    }
    mf_dfree(d);
    return rc;
}

int mf_debug_initial_heights(mf_graph *g, int32_t s, int32_t t, const mf_opts *opts, int32_t *heights) {
    if (!g || !heights) return fail(MF_ERR_ARG, "bad arguments");
    int *d = nullptr;
    CK(mf_dmalloc(&d, sizeof(int) * g->n));
    int64_t f = 0;
    mf_stats st;
    int rc = solve_common(g, 1, &s, &t, opts, &f, &st, KM_HEIGHTS, d, true);
    if (rc == MF_OK) {
        std::vector<int> h(g->n);
        down(g, h.data(), d, sizeof(int) * g->n);
        for (int x = 0; x < g->n; ++x) heights[x] = h[g->new_id[x]];
    }
    mf_dfree(d);
    return rc;
}

int mf_solve_residual(mf_graph *g, int32_t s, int32_t t, const mf_opts *opts, int64_t *flow,
                      int64_t *res, mf_stats *stats) {
    if (!g || !res) return fail(MF_ERR_ARG, "bad arguments");
    i64 *d = nullptr;
    CK(mf_dmalloc(&d, sizeof(i64) * (size_t)std::max<i64>(g->arcs, 1)));
    int64_t f = 0;
    mf_stats st;
    int rc = solve_common(g, 1, &s, &t, opts, &f, stats ? stats : &st, KM_RESIDUAL, d, true);
    if (rc == MF_OK && g->arcs) down(g, res, d, sizeof(i64) * g->arcs);
    if (flow) *flow = f;
    mf_dfree(d);
    return rc;
}

int mf_certify(mf_graph *g, int32_t s, int32_t t, const mf_opts *opts, int64_t *flow, mf_stats *stats) {
    int64_t f = 0;
    mf_stats st;
    int rc = solve_common(g, 1, &s, &t, opts, &f, stats ? stats : &st, KM_CERTIFY, nullptr, true);
    if (flow) *flow = f;
    return rc;
}

// ---- capacity updates ------------------------------------------------------

static int resolve_updates(mf_graph *g, int nb, const int32_t *u, const int32_t *v,
                           const int64_t *delta, std::vector<ArcUpdate> &ups, int *skipped) {
    std::vector<int> ui(nb), vi(nb);
    for (int i = 0; i < nb; ++i) {
        bool ok = u[i] >= 0 && u[i] < g->n && v[i] >= 0 && v[i] < g->n && u[i] != v[i];
        ui[i] = ok ? g->new_id[u[i]] : -1;
        vi[i] = ok ? g->new_id[v[i]] : -1;
    }
    // du | dv | darc (int) then dcap (i64), in the graph's update scratch
    const size_t need = sizeof(i64) * (size_t)nb + 3 * sizeof(int) * (size_t)nb + 16;
    if (g->upd_scratch_bytes < need) {
        mf_dfree(g->upd_scratch);
        g->upd_scratch = nullptr;
        g->upd_scratch_bytes = 0;
        CK(mf_dmalloc(&g->upd_scratch, need));
        g->upd_scratch_bytes = need;
    }
    i64 *dcap = reinterpret_cast<i64 *>(g->upd_scratch);
    int *du = reinterpret_cast<int *>(dcap + nb), *dv = du + nb, *darc = dv + nb;
    CK(up(g, du, ui.data(), sizeof(int) * nb));
    CK(up(g, dv, vi.data(), sizeof(int) * nb));
    k_find_arcs<<<(unsigned)((nb + 7) / 8), 256, 0, g->stream>>>(nb, du, dv, g->row, g->col, g->rev, g->fwd, g->cap, darc, dcap);
    std::vector<int> arc(nb);
    std::vector<i64> capv(nb);
    CK(cudaMemcpyAsync(arc.data(), darc, sizeof(int) * nb, cudaMemcpyDeviceToHost, g->stream));
    CK(cudaMemcpyAsync(capv.data(), dcap, sizeof(i64) * nb, cudaMemcpyDeviceToHost, g->stream));
    CK(cudaStreamSynchronize(g->stream));
    // apply sequentially (clamp at 0 after each change), one entry per arc
    std::unordered_map<int, int> at;
    int skip = 0;
    for (int i = 0; i < nb; ++i) {
        if (arc[i] < 0) {
            ++skip;
            continue;
        }
        auto it = at.find(arc[i]);
        if (it == at.end()) {
            ArcUpdate a;
            a.arc = arc[i];
            a.pad = 0;
            a.old_cap = capv[i];
            a.new_cap = capv[i];
            at[arc[i]] = (int)ups.size();
            ups.push_back(a);
            it = at.find(arc[i]);
        }
        ArcUpdate &a = ups[it->second];
        a.new_cap = std::max<i64>(0, a.new_cap + delta[i]);
    }
    if (skipped) *skipped = skip;
    return MF_OK;
}

static int apply_updates(mf_graph *g, const std::vector<ArcUpdate> &ups, ArcUpdate **d_out) {
    *d_out = nullptr;
    if (ups.empty()) return MF_OK;
    // capacities change reachability: the kept-set cache goes stale (rebuilt
    // lazily, in the same buffers)
    if (g->kc_valid || g->kc_tried) {
        invalidate_kept_cache(g);
        int rc = upload_dgraph(g);
        if (rc) return rc;
    }
    if (g->upd_recs_cap < ups.size()) {
        mf_dfree(g->upd_recs);
        g->upd_recs = nullptr;
        g->upd_recs_cap = 0;
        CK(mf_dmalloc(&g->upd_recs, sizeof(ArcUpdate) * ups.size()));
        g->upd_recs_cap = ups.size();
    }
    ArcUpdate *d = g->upd_recs;  // owned by the graph: valid until its next update batch
    CK(up(g, d, ups.data(), sizeof(ArcUpdate) * ups.size()));
    k_apply_caps<<<((int)ups.size() + 255) / 256, 256, 0, g->stream>>>((int)ups.size(), d, g->cap);
    CK(cudaStreamSynchronize(g->stream));
    *d_out = d;
    return MF_OK;
}

int mf_update_caps(mf_graph *g, int nb, const int32_t *u, const int32_t *v, const int64_t *delta,
                   int *skipped) {
    if (!g) return fail(MF_ERR_ARG, "graph is NULL");
    if (nb <= 0) return MF_OK;
    if (!u || !v || !delta) return fail(MF_ERR_ARG, "bad update arrays");
    std::vector<ArcUpdate> ups;
    int rc = resolve_updates(g, nb, u, v, delta, ups, skipped);
    if (rc) return rc;
    ArcUpdate *d = nullptr;
    rc = apply_updates(g, ups, &d);
    return rc;
}

// ---- sessions ----------------------------------------------------------------

int mf_session_create(mf_graph *g, int nq, const int32_t *s, const int32_t *t, const mf_opts *opts,
                      mf_session **out) {
    if (!g || !out || nq <= 0 || !s || !t) return fail(MF_ERR_ARG, "bad arguments");
    mf_session *ss = new mf_session();
    ss->g = g;
    ss->nq = nq;
    ss->s.resize(nq);
    ss->t.resize(nq);
    for (int i = 0; i < nq; ++i) to_internal(g, s[i], t[i], ss->s[i], ss->t[i]);
    if (opts) ss->opts = *opts;
    else mf_opts_default(&ss->opts);
    ss->pool.n = g->n;
    ss->pool.arcs = g->arcs;
    ss->pool.nhub = g->nhub;
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    if ((double)slot_bytes(g->n, g->arcs, g->nhub) * nq > 0.9 * (double)fr) {
        delete ss;
        return fail(MF_ERR_NOMEM, "admission: %d resident queries need %.1f GB, %.1f GB free", nq,
                    slot_bytes(g->n, g->arcs, g->nhub) * (double)nq / 1e9, fr / 1e9);
    }
    int rc = ss->pool.grow(nq);
    if (rc) {
        ss->pool.release();
        delete ss;
        return rc;
    }
    *out = ss;
    return MF_OK;
}

static int session_run(mf_session *ss, int mode, const ArcUpdate *d_upd, int nupd, int64_t *flows,
                       mf_stats *stats) {
    mf_graph *g = ss->g;
    // a solve from scratch uses the kept-set cache (dropped by capacity
    // updates, rebuilt here); a repair finds its kept sets itself
    if (mode == KM_SOLVE) {
        int rc = ensure_kept_cache(g, ss->opts);
        if (rc) return rc;
    }
    std::vector<QOut> outs(ss->nq);
    int G = ss->opts.group_ctas > 0 ? ss->opts.group_ctas : 8;
    int rc = launch(g, ss->pool, ss->nq, ss->s.data(), ss->t.data(), true, ss->opts, mode, nullptr,
                    d_upd, nupd, G, outs.data());
    if (rc) return rc;
    int worst = MF_OK;
    for (int i = 0; i < ss->nq; ++i) {
        if (flows) flows[i] = outs[i].flow;
        if (stats) fill_stats(&stats[i], outs[i], 0.0, 0);
        int st = status_from_err(outs[i].status);
        if (st != MF_OK && worst == MF_OK) worst = st;
    }
    if (worst != MF_OK) return fail(worst, "a resident query ended with status %d", worst);
    return MF_OK;
}

int mf_session_solve(mf_session *ss, int64_t *flows, mf_stats *stats) {
    if (!ss) return fail(MF_ERR_ARG, "session is NULL");
    int rc = session_run(ss, KM_SOLVE, nullptr, 0, flows, stats);
    if (rc == MF_OK) ss->solved = true;
    return rc;
}

int mf_session_update(mf_session *ss, int nb, const int32_t *u, const int32_t *v, const int64_t *delta,
                      int64_t *flows, mf_stats *stats) {
    if (!ss) return fail(MF_ERR_ARG, "session is NULL");
    if (!ss->solved) {
        int rc = mf_update_caps(ss->g, nb, u, v, delta, nullptr);
        if (rc) return rc;
        return mf_session_solve(ss, flows, stats);
    }
    std::vector<ArcUpdate> ups;
    int rc = MF_OK;
    if (nb > 0) {
        if (!u || !v || !delta) return fail(MF_ERR_ARG, "bad update arrays");
        rc = resolve_updates(ss->g, nb, u, v, delta, ups, nullptr);
        if (rc) return rc;
    }
    ArcUpdate *d = nullptr;
    rc = apply_updates(ss->g, ups, &d);
    if (rc) return rc;
    // A batch touching more than 1/2000 of the graph's arcs re-solves the
    // resident queries from scratch: on R-MAT 2^22 (134 M arcs) the
    // incremental repair beat a fresh batch after 1k and 10k changes (81 vs
    // 95 ms) and lost after 100k (560 vs 93 ms: the cancelled flow leaves
    // deficits and excess everywhere, ~9 relabels per query).
    // MF_REPAIR_MAX_UPDATES overrides the limit.
    long long lim = ss->g->arcs / 2000;
    if (const char *e = getenv("MF_REPAIR_MAX_UPDATES")) lim = atoll(e);
    if ((long long)ups.size() > lim) rc = session_run(ss, KM_SOLVE, nullptr, 0, flows, stats);
    else rc = session_run(ss, KM_REPAIR, d, (int)ups.size(), flows, stats);
    return rc;
}

int mf_session_destroy(mf_session *ss) {
    if (!ss) return MF_OK;
    ss->pool.release();
    delete ss;
    return MF_OK;
}

}  // extern "C"

// ---- continuous-batching server ---------------------------------------------
//
// One persistent cooperative launch of all the GPU's query groups serves a
// ring of requests in mapped pinned host memory: (s,t) queries and
// capacity-update batches on any of the server's graphs (device-resident
// for the server's life).  Group i serves with slot i once the host has
// admitted one; groups without a slot are parked.  A request is admitted to
// the ring if its entry is free (the ticket `cap` earlier has finished), and
// slots are admitted one request at a time: whenever more requests are open
// than slots exist, another slot is allocated if free HBM allows
// (cudaMemGetInfo, 85 % rule), stream-ordered on a side stream so the
// running launch is not disturbed, and published to a parked group.

namespace {
constexpr int SRV_RING_DEFAULT = 1 << 16;       // ring entries
constexpr long long SRV_UPD_DEFAULT = 1 << 20;  // update-arena entries
constexpr int SRV_INITIAL_SLOTS = 4;
}  // namespace

struct mf_server {
    std::vector<mf_graph *> graphs;
    DGraph *d_graphs = nullptr;
    GState *d_gstate = nullptr;
    GroupCtl *d_gctl = nullptr;
    SrvCtl *d_srv = nullptr;
    int *d_err = nullptr;
    mf_opts opts;
    KOpts ko;
    int G = 8;
    int threads = 512;
    int ngroups = 0;    // groups of a launch (co-resident CTAs / G)
    int max_slots = 0;  // admission cap (<= ngroups)
    int nslots = 0;     // slots admitted; group i serves with slot i
    int slot_n = 0, slot_nhub = 0;
    i64 slot_arcs = 0;
    size_t slot_size = 0;
    std::vector<void *> slot_mem;
    // mapped pinned host memory
    int cap = 0;
    unsigned long long *h_tail = nullptr;
    int *h_stop = nullptr;
    int *h_done = nullptr;
    RingReq *h_req = nullptr;
    u64 *h_t0 = nullptr;
    QOut *h_out = nullptr;
    DSlot *h_slot_tab = nullptr;
    int *h_slot_ready = nullptr;
    UpdEntry *h_upd = nullptr;
    long long upd_cap = 0;
    // host bookkeeping
    std::vector<long long> tk_of;  // ring entry -> ticket in it (-1: none yet)
    long long submitted = 0;
    long long first_open = 0;      // smallest ticket not known to be finished
    // update arena: batches occupy [lo, hi) of a virtual offset space
    // (physical offset = virtual % upd_cap, a batch never wraps)
    long long upd_lo = 0, upd_hi = 0;
    std::deque<std::pair<long long, long long>> upd_live;  // (ticket, virtual end), oldest first
    std::vector<long long> nq_sub;   // per graph: queries submitted
    std::vector<int> nupd_sub;       // per graph: update batches submitted
    std::vector<char> updated;       // per graph: a batch was submitted
    cudaStream_t stream = nullptr, side = nullptr;
    cudaEvent_t done_ev = nullptr;
    bool running = false;
    bool launched = false;  // a launch has happened (its error word is meaningful)
    // slot admission runs on its own host thread, so a submit never waits
    // for an allocation: the submitting thread raises `want` (slots the open
    // requests could use) and the admission thread allocates up to it
    int device = 0;
    std::atomic<int> nslots_pub{0};  // slots published (mf_server_slots)
    std::atomic<long long> want{0};
    std::atomic<bool> admit_stop{false};
    std::mutex admit_mu;
    std::condition_variable admit_cv;
    std::thread admit_thr;
};

static bool server_alive(mf_server *sv) {
    if (!sv->running) return false;
    cudaError_t q = cudaEventQuery(sv->done_ev);
    if (q == cudaErrorNotReady) return true;
    sv->running = false;
    return false;
}

static int server_launch(mf_server *sv) {
    if (sv->nslots_pub.load() < 1) return fail(MF_ERR_NOMEM, "server: no residual slot admitted");
    CK(cudaMemsetAsync(sv->d_gctl, 0, sizeof(GroupCtl) * sv->ngroups, sv->stream));
    CK(cudaMemsetAsync(&sv->d_srv->live, 0, sizeof(int), sv->stream));
    CK(cudaMemsetAsync(sv->d_err, 0, sizeof(int), sv->stream));
    *(volatile int *)sv->h_stop = 0;
    std::atomic_thread_fence(std::memory_order_seq_cst);
    KParams p{};
    p.graphs = sv->d_graphs;
    p.G = sv->G;
    p.nq = 0;
    p.err = sv->d_err;
    p.bar_limit_ns = 20ull * 1000 * 1000 * 1000;
    p.o = sv->ko;
    p.mode = KM_SOLVE;
    CK(cudaHostGetDevicePointer((void **)&p.ring_tail, sv->h_tail, 0));
    CK(cudaHostGetDevicePointer((void **)&p.ring_stop, sv->h_stop, 0));
    CK(cudaHostGetDevicePointer((void **)&p.ring_done, sv->h_done, 0));
    CK(cudaHostGetDevicePointer((void **)&p.ring_req, sv->h_req, 0));
    CK(cudaHostGetDevicePointer((void **)&p.ring_t0, sv->h_t0, 0));
    CK(cudaHostGetDevicePointer((void **)&p.out, sv->h_out, 0));
    CK(cudaHostGetDevicePointer((void **)&p.slot_tab, sv->h_slot_tab, 0));
    CK(cudaHostGetDevicePointer((void **)&p.slot_ready, sv->h_slot_ready, 0));
    CK(cudaHostGetDevicePointer((void **)&p.srv_upd, sv->h_upd, 0));
    p.ring_cap = sv->cap;
    p.idle_limit_ns = 300ull * 1000 * 1000;  // groups idle this long end the launch
    p.srv = sv->d_srv;
    p.gstate = sv->d_gstate;
    p.gctl = sv->d_gctl;
    p.slot_n = sv->slot_n;
    cudaError_t le = cudaSuccess;
    mf_launch_kernel(p, sv->ngroups * sv->G, sv->threads, sv->stream, sv->G > 1, &le);
    if (le != cudaSuccess) return fail(MF_ERR_CUDA, "server launch: %s", cudaGetErrorString(le));
    CK(cudaEventRecord(sv->done_ev, sv->stream));
    sv->running = true;
    sv->launched = true;
    return MF_OK;
}

// Device status of the last launch once it has ended (0: none).
static int server_error(mf_server *sv) {
    if (!sv->launched) return 0;
    int herr = 0;
    if (cudaMemcpy(&herr, sv->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return MFD_TIMEOUT;
    return herr;
}

// Launch the persistent kernel if it is not running (after reporting an
// error of the last launch).
static int server_ensure_running(mf_server *sv) {
    if (server_alive(sv)) return MF_OK;
    int herr = server_error(sv);
    if (herr) return fail(status_from_err(herr), "server kernel aborted (status %d)", herr);
    return server_launch(sv);
}

// Advance first_open over finished tickets; free the arena space of
// finished update batches (oldest first).
static void server_advance(mf_server *sv) {
    while (sv->first_open < sv->submitted &&
           *(volatile int *)&sv->h_done[sv->first_open % sv->cap] == 1)
        ++sv->first_open;
    while (!sv->upd_live.empty() && sv->upd_live.front().first < sv->first_open) {
        sv->upd_lo = sv->upd_live.front().second;
        sv->upd_live.pop_front();
    }
    if (sv->upd_live.empty()) sv->upd_lo = sv->upd_hi = 0;  // no batch in use: restart at 0
}

// Admission of residual slots by free HBM: allocate slots (each only if
// cudaMemGetInfo shows room for it under the 85 % rule) until `want` are
// admitted; returns the slots admitted.  Runs on the admission thread (or
// at creation, before that thread exists).
static int server_grow_slots(mf_server *sv, long long want) {
    while (sv->nslots < sv->max_slots && want > sv->nslots) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess || (double)fr * 0.85 < (double)sv->slot_size) break;
        void *m = nullptr;
        if (mf_dmalloc_async_raw(&m, sv->slot_size, sv->side) != cudaSuccess ||
            cudaStreamSynchronize(sv->side) != cudaSuccess) {
            cudaGetLastError();
            if (m) mf_dfree_async(m, sv->side);
            break;
        }
        sv->slot_mem.push_back(m);
        sv->h_slot_tab[sv->nslots] = carve_slot((char *)m, sv->slot_n, sv->slot_arcs, sv->slot_nhub);
        std::atomic_thread_fence(std::memory_order_seq_cst);
        *(volatile int *)&sv->h_slot_ready[sv->nslots] = 1;  // the group clears it before use
        ++sv->nslots;
        sv->nslots_pub.store(sv->nslots);
    }
    return sv->nslots;
}

static void server_admit_loop(mf_server *sv) {
    cudaSetDevice(sv->device);
    std::unique_lock<std::mutex> lk(sv->admit_mu);
    for (;;) {
        sv->admit_cv.wait(lk, [&] { return sv->admit_stop.load() || sv->want.load() > sv->nslots_pub.load(); });
        if (sv->admit_stop.load()) return;
        const long long want = sv->want.load();
        lk.unlock();
        const int before = sv->nslots;
        server_grow_slots(sv, want);
        lk.lock();
        // no room (or the cap): wait for a larger want rather than retrying
        if (sv->nslots == before && !sv->admit_stop.load()) {
            sv->admit_cv.wait_for(lk, std::chrono::milliseconds(20));
            if (sv->want.load() <= want) sv->want.store(sv->nslots);
        }
    }
}

// Called on every submit: more requests are open than slots exist -> ask
// the admission thread for more.
static void server_admit_slots(mf_server *sv) {
    server_advance(sv);
    const long long open = std::min<long long>(sv->submitted - sv->first_open, sv->max_slots);
    if (open > sv->nslots_pub.load() && open > sv->want.load()) {
        {
            std::lock_guard<std::mutex> lk(sv->admit_mu);
            sv->want.store(open);
        }
        sv->admit_cv.notify_one();
    }
}

// Reserve the ring entry of the next ticket (its previous ticket finished).
static int server_reserve(mf_server *sv, int &e) {
    server_advance(sv);
    const long long k = sv->submitted;
    e = (int)(k % sv->cap);
    if (k - sv->first_open >= sv->cap)
        return fail(MF_ERR_NOMEM, "server ring full: %d requests open (ticket %lld not finished)", sv->cap,
                    sv->first_open);
    return MF_OK;
}

static int server_publish(mf_server *sv, int e, long long *ticket) {
    const long long k = sv->submitted;
    sv->tk_of[e] = k;
    std::atomic_thread_fence(std::memory_order_seq_cst);
    sv->submitted = k + 1;
    *(volatile unsigned long long *)sv->h_tail = (unsigned long long)sv->submitted;
    std::atomic_thread_fence(std::memory_order_seq_cst);
    if (ticket) *ticket = k;
    server_admit_slots(sv);
    return server_ensure_running(sv);
}

extern "C" {

int mf_server_create(mf_graph **graphs, int ngraphs, const mf_opts *opts, int max_slots,
                     mf_server **out) {
    if (!graphs || ngraphs <= 0 || !out) return fail(MF_ERR_ARG, "bad arguments");
    *out = nullptr;
    mf_server *sv = new mf_server();
    if (opts) sv->opts = *opts;
    else mf_opts_default(&sv->opts);
    i64 arcs_sum = 0, n_sum = 0;
    std::vector<DGraph> dg(ngraphs);
    for (int i = 0; i < ngraphs; ++i) {
        mf_graph *g = graphs[i];
        if (!g) {
            delete sv;
            return fail(MF_ERR_ARG, "graph %d is NULL", i);
        }
        sv->graphs.push_back(g);
        sv->slot_n = std::max(sv->slot_n, g->n);
        sv->slot_arcs = std::max(sv->slot_arcs, g->arcs);
        sv->slot_nhub = std::max(sv->slot_nhub, g->nhub);
        arcs_sum += g->arcs;
        n_sum += g->n;
        int rc0 = ensure_kept_cache(g, sv->opts);
        if (rc0) {
            delete sv;
            return rc0;
        }
        dg[i] = make_dgraph(g);
    }
    sv->ko = resolve_opts(sv->opts, (int)(arcs_sum / std::max<i64>(1, n_sum)));
    DevInfo di;
    sv->threads = sv->opts.threads > 0 ? sv->opts.threads : 512;
    int rc = dev_info(di, sv->threads);
    if (rc) {
        delete sv;
        return rc;
    }
    sv->G = sv->opts.group_ctas > 0 ? sv->opts.group_ctas : 8;
    sv->ngroups = std::max(1, di.sms * di.bps / sv->G);
    sv->max_slots = max_slots > 0 ? std::min(max_slots, sv->ngroups) : sv->ngroups;
    sv->slot_size = slot_bytes(sv->slot_n, sv->slot_arcs, sv->slot_nhub);
    sv->cap = SRV_RING_DEFAULT;
    if (const char *e = getenv("MF_SERVER_RING")) sv->cap = std::max(16, atoi(e));
    sv->upd_cap = SRV_UPD_DEFAULT;
    if (const char *e = getenv("MF_SERVER_UPDATE_ARENA")) sv->upd_cap = std::max(1024LL, atoll(e));
    sv->tk_of.assign(sv->cap, -1);
    sv->nq_sub.assign(ngraphs, 0);
    sv->nupd_sub.assign(ngraphs, 0);
    sv->updated.assign(ngraphs, 0);
    auto bail = [&](int code, const char *what) {
        mf_server_destroy(sv);
        return fail(code, "server creation: %s", what);
    };
    if (mf_dmalloc(&sv->d_graphs, sizeof(DGraph) * ngraphs) != cudaSuccess ||
        mf_dmalloc(&sv->d_gstate, sizeof(GState) * ngraphs) != cudaSuccess ||
        mf_dmalloc(&sv->d_gctl, sizeof(GroupCtl) * sv->ngroups) != cudaSuccess ||
        mf_dmalloc(&sv->d_srv, sizeof(SrvCtl)) != cudaSuccess || mf_dmalloc(&sv->d_err, sizeof(int)) != cudaSuccess)
        return bail(MF_ERR_NOMEM, "device tables");
    bool ok = mf_hostalloc(&sv->h_tail, sizeof(unsigned long long) * 2, cudaHostAllocMapped) == cudaSuccess &&
              mf_hostalloc(&sv->h_done, sizeof(int) * sv->cap, cudaHostAllocMapped) == cudaSuccess &&
              mf_hostalloc(&sv->h_req, sizeof(RingReq) * sv->cap, cudaHostAllocMapped) == cudaSuccess &&
              mf_hostalloc(&sv->h_t0, sizeof(u64) * 2 * sv->cap, cudaHostAllocMapped) == cudaSuccess &&
              mf_hostalloc(&sv->h_out, sizeof(QOut) * sv->cap, cudaHostAllocMapped) == cudaSuccess &&
              mf_hostalloc(&sv->h_slot_tab, sizeof(DSlot) * sv->ngroups, cudaHostAllocMapped) == cudaSuccess &&
              mf_hostalloc(&sv->h_slot_ready, sizeof(int) * sv->ngroups, cudaHostAllocMapped) == cudaSuccess &&
              mf_hostalloc(&sv->h_upd, sizeof(UpdEntry) * sv->upd_cap, cudaHostAllocMapped) == cudaSuccess;
    if (!ok) return bail(MF_ERR_NOMEM, "mapped ring allocation failed");
    sv->h_stop = reinterpret_cast<int *>(sv->h_tail + 1);
    memset(sv->h_tail, 0, sizeof(unsigned long long) * 2);
    memset(sv->h_done, 0, sizeof(int) * sv->cap);
    memset(sv->h_slot_ready, 0, sizeof(int) * sv->ngroups);
    if (cudaMemcpy(sv->d_graphs, dg.data(), sizeof(DGraph) * ngraphs, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(sv->d_gstate, 0, sizeof(GState) * ngraphs) != cudaSuccess ||
        cudaMemset(sv->d_srv, 0, sizeof(SrvCtl)) != cudaSuccess ||
        cudaMemset(sv->d_err, 0, sizeof(int)) != cudaSuccess || cudaStreamSynchronize(0) != cudaSuccess ||
        cudaStreamCreateWithFlags(&sv->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&sv->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&sv->done_ev, cudaEventDisableTiming) != cudaSuccess)
        return bail(MF_ERR_CUDA, "device set-up failed");
    // the first slots (more are admitted as requests open up)
    cudaGetDevice(&sv->device);
    server_grow_slots(sv, std::min(SRV_INITIAL_SLOTS, sv->max_slots));
    if (sv->nslots < 1) {
        mf_server_destroy(sv);
        return fail(MF_ERR_NOMEM, "admission: no HBM for one residual slot (%zu bytes)", sv->slot_size);
    }
    sv->want.store(sv->nslots);
    sv->admit_thr = std::thread(server_admit_loop, sv);
    *out = sv;
    return MF_OK;
}

int mf_server_slots(const mf_server *sv, int *slots) {
    if (!sv || !slots) return fail(MF_ERR_ARG, "bad arguments");
    *slots = sv->nslots_pub.load();
    return MF_OK;
}

int mf_server_submit(mf_server *sv, int graph, int32_t s, int32_t t, long long *ticket) {
    if (!sv) return fail(MF_ERR_ARG, "server is NULL");
    if (graph < 0 || graph >= (int)sv->graphs.size()) return fail(MF_ERR_ARG, "graph index %d", graph);
    int e = 0;
    int rc = server_reserve(sv, e);
    if (rc) return rc;
    mf_graph *g = sv->graphs[graph];
    int si = -1, ti = -1;
    to_internal(g, s, t, si, ti);
    RingReq r{};
    r.kind = RQ_QUERY;
    r.graph = graph;
    r.s = si;
    r.t = ti;
    r.epoch = sv->nupd_sub[graph];
    sv->h_req[e] = r;
    sv->h_done[e] = 0;
    sv->nq_sub[graph]++;
    return server_publish(sv, e, ticket);
}

int mf_server_update(mf_server *sv, int graph, int nb, const int32_t *u, const int32_t *v,
                     const int64_t *delta, long long *ticket) {
    if (!sv) return fail(MF_ERR_ARG, "server is NULL");
    if (graph < 0 || graph >= (int)sv->graphs.size()) return fail(MF_ERR_ARG, "graph index %d", graph);
    if (nb < 0 || (nb > 0 && (!u || !v || !delta))) return fail(MF_ERR_ARG, "bad update arrays");
    mf_graph *g = sv->graphs[graph];
    // fold the changes of each (u, v) pair, in order, into cap -> max(a, cap + b)
    std::map<std::pair<int, int>, std::pair<i64, i64>> fold;
    std::vector<std::pair<int, int>> order;
    for (int i = 0; i < nb; ++i) {
        if (u[i] < 0 || u[i] >= g->n || v[i] < 0 || v[i] >= g->n || u[i] == v[i]) continue;
        const std::pair<int, int> key(g->new_id[u[i]], g->new_id[v[i]]);
        auto it = fold.find(key);
        if (it == fold.end()) {
            fold[key] = std::make_pair((i64)0, (i64)delta[i]);
            order.push_back(key);
        } else {
            const i64 a = it->second.first, b = it->second.second;
            it->second = std::make_pair(std::max<i64>(0, a + delta[i]), b + delta[i]);
        }
    }
    const long long n = (long long)order.size();
    if (n > sv->upd_cap)
        return fail(MF_ERR_ARG, "update batch of %lld arcs exceeds the server's update arena (%lld)", n,
                    sv->upd_cap);
    int e = 0;
    int rc = server_reserve(sv, e);
    if (rc) return rc;
    // arena space: a batch is contiguous; wait (bounded) for older batches
    long long off = 0;
    for (auto t0 = std::chrono::steady_clock::now();;) {
        server_advance(sv);
        off = sv->upd_hi;
        if (off % sv->upd_cap + n > sv->upd_cap) off += sv->upd_cap - off % sv->upd_cap;
        if (off + n - sv->upd_lo <= sv->upd_cap) break;
        rc = server_ensure_running(sv);
        if (rc) return rc;
        std::this_thread::sleep_for(std::chrono::microseconds(50));
        if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(60))
            return fail(MF_ERR_TIMEOUT, "server update arena stayed full for 60 s");
    }
    const long long phys = off % sv->upd_cap;
    for (long long i = 0; i < n; ++i) {
        const auto &kv = *fold.find(order[i]);
        UpdEntry x;
        x.u = kv.first.first;
        x.v = kv.first.second;
        x.a = kv.second.first;
        x.b = kv.second.second;
        sv->h_upd[phys + i] = x;
    }
    sv->upd_hi = off + n;
    sv->upd_live.push_back(std::make_pair(sv->submitted, sv->upd_hi));
    RingReq r{};
    r.kind = RQ_UPDATE;
    r.graph = graph;
    r.s = r.t = -1;
    r.epoch = sv->nupd_sub[graph];
    r.upd_n = (int)n;
    r.upd_off = phys;
    r.need_done = (unsigned long long)sv->nq_sub[graph];
    sv->h_req[e] = r;
    sv->h_done[e] = 0;
    sv->nupd_sub[graph]++;
    sv->updated[graph] = 1;
    return server_publish(sv, e, ticket);
}

int mf_server_poll(mf_server *sv, long long ticket, int *done, int64_t *flow, double *latency_ms,
                   int *status) {
    if (!sv || ticket < 0 || ticket >= sv->submitted) return fail(MF_ERR_ARG, "bad ticket");
    const int e = (int)(ticket % sv->cap);
    if (sv->tk_of[e] != ticket) return fail(MF_ERR_ARG, "ticket %lld expired (its ring entry was reused)", ticket);
    int d = *(volatile int *)&sv->h_done[e];
    if (d != 1) {
        int rc = server_ensure_running(sv);
        if (rc) return rc;
        if (done) *done = 0;
        return MF_OK;
    }
    std::atomic_thread_fence(std::memory_order_seq_cst);
    const QOut &q = sv->h_out[e];
    if (done) *done = 1;
    if (flow) *flow = q.flow;
    if (status) *status = status_from_err(q.status);
    if (latency_ms) {
        volatile u64 *t0 = sv->h_t0;
        *latency_ms = (double)(t0[2 * e + 1] - t0[2 * e]) * 1e-6;
    }
    return MF_OK;
}

int mf_server_drain(mf_server *sv) {
    if (!sv) return fail(MF_ERR_ARG, "server is NULL");
    for (;;) {
        server_advance(sv);
        if (sv->first_open >= sv->submitted) return MF_OK;
        int rc = server_ensure_running(sv);
        if (rc) return rc;
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

int mf_server_destroy(mf_server *sv) {
    if (!sv) return MF_OK;
    if (sv->admit_thr.joinable()) {
        {
            std::lock_guard<std::mutex> lk(sv->admit_mu);
            sv->admit_stop.store(true);
        }
        sv->admit_cv.notify_one();
        sv->admit_thr.join();
    }
    if (sv->h_stop) *(volatile int *)sv->h_stop = 1;
    std::atomic_thread_fence(std::memory_order_seq_cst);
    if (sv->stream) cudaStreamSynchronize(sv->stream);
    // capacities changed under the graphs' kept-set caches: drop them (the
    // next solve on the graph rebuilds its cache)
    for (size_t i = 0; i < sv->graphs.size() && i < sv->updated.size(); ++i) {
        if (!sv->updated[i]) continue;
        mf_graph *g = sv->graphs[i];
        invalidate_kept_cache(g);
        upload_dgraph(g);
    }
    for (void *m : sv->slot_mem) mf_dfree_async(m, sv->side ? sv->side : sv->stream);
    if (sv->side) cudaStreamSynchronize(sv->side);
    mf_dfree(sv->d_graphs);
    mf_dfree(sv->d_gstate);
    mf_dfree(sv->d_gctl);
    mf_dfree(sv->d_srv);
    mf_dfree(sv->d_err);
    mf_hfree(sv->h_tail);
    mf_hfree(sv->h_done);
    mf_hfree(sv->h_req);
    mf_hfree(sv->h_t0);
    mf_hfree(sv->h_out);
    mf_hfree(sv->h_slot_tab);
    mf_hfree(sv->h_slot_ready);
    mf_hfree(sv->h_upd);
    if (sv->done_ev) cudaEventDestroy(sv->done_ev);
    if (sv->stream) cudaStreamDestroy(sv->stream);
    if (sv->side) cudaStreamDestroy(sv->side);
    delete sv;
    return MF_OK;
}

}  // extern "C"
