// Allocation-free solve (mf_solve_csr_noalloc).
//
// Some callers cannot call cudaMalloc on the path where they need a max flow:
// a host framework that owns the device memory pool and forbids allocations
// outside it, a latency-critical service that allocates everything at start-up
// (cudaMalloc may synchronize the device and fragment a pool it does not
// own), or a plugin that is only handed device pointers.  For them this entry
// point solves one (s,t) query on a CSR the caller already holds in device
// memory, using as scratch only a fixed file-scope device array.
//
// The array below holds one residual slot (residuals, excesses, heights,
// stamps, worklists, control words) for graphs of at most NA_MAX_N vertices
// and NA_MAX_ARCS arcs: about 11 MB that every GPU which loads this library
// keeps until the process exits.  Calls share it and it keeps the previous
// call's contents, so calls whose work overlaps on the GPU (concurrent calls
// from several host threads, or on several streams of one device) race and
// must be serialized by the caller.
//
// Before the solve, a check kernel validates the caller's CSR (offsets,
// head and reverse-arc ranges, the reverse pairing, non-negative
// capacities), so a malformed graph is rejected with MF_ERR_ARG instead of
// steering the solver's indexing outside its scratch regions.
#include <cstdio>
#include <cstring>

#include "../../include/maxflow_b200.h"
#include "mf_solver.cuh"

#include <mutex>

// mf_api.cu: the last-error text of this thread, and the option resolution,
// launch time limit and status mapping every entry point shares.
void mf_set_last_error(const char *msg);
KOpts mf_resolve_opts(const mf_opts &o, int avg_deg);
u64 mf_launch_time_limit_ns();
int mf_status_from_err(int e);

namespace {

constexpr int NA_MAX_N = 1 << 16;
constexpr long long NA_MAX_ARCS = 1 << 20;

constexpr size_t na_align(size_t x) { return (x + 255) & ~(size_t)255; }

// byte offsets inside the scratch array
constexpr size_t OFF_GRAPH = 0;
constexpr size_t OFF_SLOT = OFF_GRAPH + na_align(sizeof(DGraph));
constexpr size_t OFF_OUT = OFF_SLOT + na_align(sizeof(DSlot));
constexpr size_t OFF_CTL = OFF_OUT + na_align(sizeof(QOut));      // err, q_next, s, t
constexpr size_t OFF_ROF = OFF_CTL + na_align(sizeof(int) * 8);   // region_of (all zero, R = 1)
constexpr size_t OFF_RES = OFF_ROF + na_align(sizeof(int) * NA_MAX_N);
constexpr size_t OFF_EX = OFF_RES + na_align(sizeof(i64) * NA_MAX_ARCS);
constexpr size_t OFF_H = OFF_EX + na_align(sizeof(i64) * NA_MAX_N);
constexpr size_t OFF_MARK = OFF_H + na_align(sizeof(int) * NA_MAX_N);
constexpr size_t OFF_QMARK = OFF_MARK + na_align(sizeof(int) * NA_MAX_N);
constexpr size_t OFF_CLAIM = OFF_QMARK + na_align(sizeof(int) * NA_MAX_N);
constexpr size_t OFF_VLIST = OFF_CLAIM + na_align(sizeof(int) * NA_MAX_N);
constexpr size_t OFF_QA = OFF_VLIST + na_align(sizeof(int) * NA_MAX_N);
constexpr size_t OFF_QB = OFF_QA + na_align(sizeof(int) * NA_MAX_N);
constexpr size_t OFF_HOT = OFF_QB + na_align(sizeof(int) * NA_MAX_N);
constexpr size_t OFF_RACT = OFF_HOT + na_align(sizeof(int) * 1024);
constexpr size_t OFF_CNT = OFF_RACT + na_align(sizeof(int) * 1024);
constexpr size_t OFF_ACC = OFF_CNT + na_align(sizeof(int) * CNT_WORDS);
constexpr size_t OFF_BAR = OFF_ACC + na_align(sizeof(i64) * 128);
constexpr size_t OFF_CLOCK = OFF_BAR + na_align(sizeof(GroupBar));
constexpr size_t OFF_META = OFF_CLOCK + na_align(sizeof(unsigned));
// a hub has more than HUB_T arcs, so at most NA_MAX_ARCS / (HUB_T + 1) exist
constexpr int NA_MAX_HUBS = (int)(NA_MAX_ARCS / (HUB_T + 1)) + 1;
constexpr size_t OFF_HUBW = OFF_META + na_align(sizeof(int) * 8);
constexpr size_t OFF_BITS = OFF_HUBW + na_align(sizeof(HubWork) * NA_MAX_HUBS);
constexpr size_t NA_BYTES = OFF_BITS + na_align(sizeof(unsigned) * 5 * ((NA_MAX_N + 31) / 32));

}  // namespace

// The scratch itself.  Host code must not use this name as an address: it
// is a host-side stand-in.  The device address comes from
// cudaGetSymbolAddress, once per device (na_base below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

// CSR defects found by k_na_check (bits of the check word).
#define NA_BAD_ROW 1   // offsets not 0 .. arcs, or decreasing
#define NA_BAD_COL 2   // head outside [0, n)
#define NA_BAD_REV 4   // reverse arc outside [0, arcs), outside its head's range, or not paired back
#define NA_BAD_CAP 8   // negative capacity

// One warp per vertex: its offsets, then every arc e = v -> w: w in [0, n),
// r = rev[e] inside w's arc range, col[r] == v, rev[r] == e, cap[e] >= 0.
// Every load is guarded by the checks before it, so a malformed CSR is
// reported, never indexed out of bounds.
__global__ void k_na_check(int n, long long arcs, const int *row, const int *col, const int *rev,
                           const i64 *cap, int *bad) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += nw) {
        const long long b = row[v], e1 = row[v + 1];
        if (b < 0 || b > e1 || e1 > arcs || (v == 0 && b != 0) || (v == n - 1 && e1 != arcs)) {
            if (lane == 0) atomicOr(bad, NA_BAD_ROW);
            continue;
        }
        int flags = 0;
        for (long long e = b + lane; e < e1; e += 32) {
            const int w = col[e];
            if (cap[e] < 0) flags |= NA_BAD_CAP;
            if (w < 0 || w >= n) {
                flags |= NA_BAD_COL;
                continue;
            }
            const long long r = rev[e];
            if (r < 0 || r >= arcs || r < row[w] || r >= row[w + 1] || col[r] != v || rev[r] != e)
                flags |= NA_BAD_REV;
        }
        if (flags) atomicOr(bad, flags);
    }
}

namespace {

char *na_base[64];  // per device: address of g_noalloc_scratch
int na_sms[64], na_bps[64];
std::mutex na_mu;   // guards the first-call set-up of every device

thread_local char na_msg[256];
int na_fail(int code, const char *msg) {
    mf_set_last_error(msg);
    return code;
}

// First call on a device: resolve the scratch address and zero it.  Under
// na_mu, so two host threads making their first call at once set it up
// exactly once.  The address is kept for the life of the process: after a
// cudaDeviceReset of that device it would be stale (unsupported).
int na_setup(int dev, cudaStream_t st) {
    if (dev < 0 || dev >= 64) return na_fail(MF_ERR_ARG, "mf_solve_csr_noalloc: device index out of range");
    std::lock_guard<std::mutex> lk(na_mu);
    if (na_base[dev]) return MF_OK;
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        snprintf(na_msg, sizeof na_msg, "mf_solve_csr_noalloc: cudaGetSymbolAddress failed: %s",
                 cudaGetErrorString(e));
        mf_set_last_error(na_msg);
        return MF_ERR_CUDA;
    }
    e = cudaMemsetAsync(p, 0, NA_BYTES, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&na_sms[dev], cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) {
        snprintf(na_msg, sizeof na_msg, "mf_solve_csr_noalloc: set-up failed: %s", cudaGetErrorString(e));
        mf_set_last_error(na_msg);
        return MF_ERR_CUDA;
    }
    na_bps[dev] = mf_kernel_max_blocks_per_sm(512);
    if (na_bps[dev] <= 0) return na_fail(MF_ERR_CUDA, "mf_solve_csr_noalloc: solver kernel cannot be resident");
    na_base[dev] = (char *)p;
    return MF_OK;
}

}  // namespace

extern "C" int mf_solve_csr_noalloc(int n, long long arcs, const int32_t *d_row, const int32_t *d_col,
                                    const int32_t *d_rev, const int64_t *d_cap, int32_t s, int32_t t,
                                    const mf_opts *opts, void *stream, int64_t *flow, mf_stats *stats) {
    if (flow) *flow = 0;
    if (stats) memset(stats, 0, sizeof(*stats));
    if (n < 1 || n > NA_MAX_N) {
        snprintf(na_msg, sizeof na_msg,
                 "mf_solve_csr_noalloc: n=%d is outside [1, %d], the allocation-free limit", n, NA_MAX_N);
        mf_set_last_error(na_msg);
        return MF_ERR_ARG;
    }
    if (arcs < 0 || arcs > NA_MAX_ARCS) {
        snprintf(na_msg, sizeof na_msg,
                 "mf_solve_csr_noalloc: %lld arcs is outside [0, %lld], the allocation-free limit", arcs,
                 NA_MAX_ARCS);
        mf_set_last_error(na_msg);
        return MF_ERR_ARG;
    }
    if (!d_row || (arcs > 0 && (!d_col || !d_rev || !d_cap)))
        return na_fail(MF_ERR_ARG, "mf_solve_csr_noalloc: NULL CSR array");
    if (s < 0 || t < 0 || s >= n || t >= n || s == t) return MF_OK;  // flow 0 (RA:2659-2663)
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return na_fail(MF_ERR_CUDA, "mf_solve_csr_noalloc: no device");
    int rc = na_setup(dev, st);
    if (rc) return rc;
    char *b = na_base[dev];
    mf_opts o;
    if (opts) o = *opts;
    else mf_opts_default(&o);

    // validate the caller's CSR on the device (the check word is ctl[4])
    {
        int *dbad = (int *)(b + OFF_CTL) + 4;
        int hbad = 0;
        cudaError_t e = cudaMemsetAsync(dbad, 0, sizeof(int), st);
        if (e == cudaSuccess) {
            k_na_check<<<(unsigned)((n + 7) / 8), 256, 0, st>>>(n, arcs, d_row, d_col, d_rev,
                                                               (const i64 *)d_cap, dbad);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(&hbad, dbad, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            snprintf(na_msg, sizeof na_msg, "mf_solve_csr_noalloc: CSR check failed: %s", cudaGetErrorString(e));
            mf_set_last_error(na_msg);
            return MF_ERR_CUDA;
        }
        if (hbad) {
            snprintf(na_msg, sizeof na_msg,
                     "mf_solve_csr_noalloc: malformed CSR:%s%s%s%s",
                     (hbad & NA_BAD_ROW) ? " row offsets not 0..arcs non-decreasing;" : "",
                     (hbad & NA_BAD_COL) ? " head outside [0, n);" : "",
                     (hbad & NA_BAD_REV) ? " reverse arcs not paired;" : "",
                     (hbad & NA_BAD_CAP) ? " negative capacity;" : "");
            mf_set_last_error(na_msg);
            return MF_ERR_ARG;
        }
    }

    DGraph g{n, 1, arcs, d_row, d_col, d_rev, (const i64 *)d_cap, (const int *)(b + OFF_ROF)};
    DSlot sl;
    sl.res = (i64 *)(b + OFF_RES);
    sl.ex = (i64 *)(b + OFF_EX);
    sl.h = (int *)(b + OFF_H);
    sl.mark = (unsigned *)(b + OFF_MARK);
    sl.qmark = (unsigned *)(b + OFF_QMARK);
    sl.claim = (unsigned *)(b + OFF_CLAIM);
    sl.vlist = (int *)(b + OFF_VLIST);
    sl.qa = (int *)(b + OFF_QA);
    sl.qb = (int *)(b + OFF_QB);
    sl.hot = (int *)(b + OFF_HOT);
    sl.ract = (int *)(b + OFF_RACT);
    sl.cnt = (int *)(b + OFF_CNT);
    sl.acc = (i64 *)(b + OFF_ACC);
    sl.bar = (GroupBar *)(b + OFF_BAR);
    sl.clock = (unsigned *)(b + OFF_CLOCK);
    sl.meta = (int *)(b + OFF_META);
    sl.hubw = (HubWork *)(b + OFF_HUBW);
    sl.nhub = NA_MAX_HUBS;
    sl.bits = (unsigned *)(b + OFF_BITS);
    int ctl[4] = {0, 0, s, t};  // err, q_next, s, t
    GroupBar bar0 = {0, 0, 0, 0};
    cudaError_t e = cudaMemcpyAsync(b + OFF_GRAPH, &g, sizeof g, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b + OFF_SLOT, &sl, sizeof sl, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b + OFF_CTL, ctl, sizeof ctl, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b + OFF_BAR, &bar0, sizeof bar0, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
        snprintf(na_msg, sizeof na_msg, "mf_solve_csr_noalloc: upload failed: %s", cudaGetErrorString(e));
        mf_set_last_error(na_msg);
        return MF_ERR_CUDA;
    }

    const KOpts k = mf_resolve_opts(o, (int)(arcs / n));

    int *dctl = (int *)(b + OFF_CTL);
    KParams p{};
    p.graphs = (const DGraph *)(b + OFF_GRAPH);
    p.slots = (DSlot *)(b + OFF_SLOT);
    p.G = na_sms[dev] * na_bps[dev];  // one group: the whole GPU
    p.nq = 1;
    p.q_s = dctl + 2;
    p.q_t = dctl + 3;
    p.q_next = dctl + 1;
    p.out = (QOut *)(b + OFF_OUT);
    p.err = dctl;
    p.bar_limit_ns = 20ull * 1000 * 1000 * 1000;
    p.time_limit_ns = mf_launch_time_limit_ns();
    p.o = k;
    p.mode = KM_SOLVE;
    cudaError_t le = cudaSuccess;
    mf_launch_kernel(p, p.G, 512, st, true, &le);
    if (le != cudaSuccess) {
        snprintf(na_msg, sizeof na_msg, "mf_solve_csr_noalloc: launch failed: %s", cudaGetErrorString(le));
        mf_set_last_error(na_msg);
        return MF_ERR_CUDA;
    }
    QOut q;
    int herr = 0;
    unsigned clk = 0;
    e = cudaMemcpyAsync(&q, b + OFF_OUT, sizeof q, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, dctl, sizeof herr, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&clk, b + OFF_CLOCK, sizeof clk, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        snprintf(na_msg, sizeof na_msg, "mf_solve_csr_noalloc: %s", cudaGetErrorString(e));
        mf_set_last_error(na_msg);
        return MF_ERR_CUDA;
    }
    if (herr) {
        snprintf(na_msg, sizeof na_msg, "mf_solve_csr_noalloc: device solve aborted (status %d)", herr);
        mf_set_last_error(na_msg);
        return mf_status_from_err(herr);
    }
    // stamps are compared against a monotonic 32-bit clock kept in the
    // scratch; zero them (and the clock) well before it could wrap
    if (clk > (1u << 30)) {
        e = cudaMemsetAsync(b + OFF_MARK, 0, OFF_VLIST - OFF_MARK, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(b + OFF_CLOCK, 0, sizeof(unsigned), st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return na_fail(MF_ERR_CUDA, "mf_solve_csr_noalloc: stamp reset failed");
    }
    if (flow) *flow = q.flow;
    if (stats) {
        stats->flow = q.flow;
        stats->status = mf_status_from_err(q.status);
        stats->mask_vertices = q.mask_n;
        stats->mask_arcs = q.mask_arcs;
        stats->rounds = q.rounds;
        stats->global_relabels = q.relabels;
        stats->arcs_examined = q.arcs_ex;
        stats->vertices_examined = q.verts_ex;
        stats->pushes = q.pushes;
        stats->service_ms = (double)(q.t_done - q.t_begin) * 1e-6;
    }
    if (q.status != 0) {
        snprintf(na_msg, sizeof na_msg, "mf_solve_csr_noalloc: solve ended with status %d", q.status);
        mf_set_last_error(na_msg);
        return mf_status_from_err(q.status);
    }
    return MF_OK;
}
