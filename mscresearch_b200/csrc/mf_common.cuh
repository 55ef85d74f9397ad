// Shared device-side definitions for the B200 max-flow engine.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

typedef long long i64;
typedef unsigned long long u64;

#define MF_FULL 0xffffffffu
#define MF_INF_H 0x7fffffff

// Device-side status codes written into the launch error word / per-query
// status (same numbers as the MF_ERR_* codes of the C ABI).
#define MFD_OK 0
#define MFD_ITER_LIMIT 5
#define MFD_TIMEOUT 6
#define MFD_INEXACT 7
#define MFD_CERTIFY 8

// ---------------------------------------------------------------------------
// Loads.  Graph topology is immutable during a launch: read-only path (nc).
// Residual/excess/height/stamps are written by other CTAs during a launch:
// L2-coherent loads (cg) so that no SM serves a stale L1 line.
__device__ __forceinline__ int ldro(const int *p) { return __ldg(p); }
__device__ __forceinline__ i64 ldro(const i64 *p) { return __ldg(p); }
__device__ __forceinline__ unsigned char ldro_u8(const unsigned char *p) { return __ldg(p); }
__device__ __forceinline__ int ldcg(const int *p) { return __ldcg(p); }
__device__ __forceinline__ unsigned ldcg(const unsigned *p) { return __ldcg(p); }
__device__ __forceinline__ i64 ldcg(const i64 *p) { return __ldcg(p); }
// Capacities.  The serving kernel (mf_serve_kernel.cu, MF_SERVE_TU) applies
// capacity updates to the graphs it reads while it runs, so it reads them
// through L2 (coherent); every other launch treats them as read-only.
#ifdef MF_SERVE_TU
__device__ __forceinline__ i64 ldcap(const i64 *p) { return __ldcg(p); }
__device__ __forceinline__ longlong2 ldcap2(const longlong2 *p) { return __ldcg(p); }
#else
__device__ __forceinline__ i64 ldcap(const i64 *p) { return __ldg(p); }
__device__ __forceinline__ longlong2 ldcap2(const longlong2 *p) { return __ldg(p); }
#endif

// ---------------------------------------------------------------------------
// Self-check builds (-DMF_CHECKS, libmfb200_chk.so): every warp records the
// last site it reached into host-mapped memory (readable after a failed
// launch), and list/vertex indices are range-checked; a bad index is recorded
// and the access skipped.  Production builds compile these to nothing.
#ifdef MF_CHECKS
struct MfChk {
    volatile unsigned *trace;  // [warp][4]: site, aux, count, -
    volatile int *bad;         // [0]: count, [1]: site, [2]: index, [3]: limit
};
static __device__ MfChk g_chk;  // per translation unit (no -rdc); the solver TU installs it
__device__ __forceinline__ void mf_trace(int site, int aux) {
    if (g_chk.trace && (threadIdx.x & 31) == 0) {
        unsigned w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        g_chk.trace[4 * w + 0] = site;
        g_chk.trace[4 * w + 1] = (unsigned)aux;
        g_chk.trace[4 * w + 2] += 1;
        __threadfence_system();
    }
}
__device__ __forceinline__ bool mf_ok_idx(long long i, long long lim, int site) {
    if (i >= 0 && i < lim) return true;
    if (g_chk.bad) {
        if (atomicAdd((int *)&g_chk.bad[0], 1) == 0) {
            g_chk.bad[1] = site;
            g_chk.bad[2] = (int)i;
            g_chk.bad[3] = (int)lim;
        }
        __threadfence_system();
    }
    return false;
}
#define MF_TRACE(site, aux) mf_trace((site), (int)(aux))
#define MF_OK_IDX(i, lim, site) mf_ok_idx((i), (lim), (site))
#else
#define MF_TRACE(site, aux) ((void)0)
#define MF_OK_IDX(i, lim, site) true
#endif

__device__ __forceinline__ i64 atomic_add_i64(i64 *p, i64 v) {
    return (i64)atomicAdd(reinterpret_cast<u64 *>(p), (u64)v);
}

__device__ __forceinline__ u64 globaltimer_ns() {
    u64 t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ i64 warp_incl_scan_i64(i64 x) {
    const int lane = lane_id();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        i64 y = __shfl_up_sync(MF_FULL, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

__device__ __forceinline__ i64 warp_sum_i64(i64 x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(MF_FULL, x, o);
    return x;
}

// Warp-aggregated append: every lane with flag != 0 writes val to
// list[base + rank]; one atomicAdd per warp on *tail.  Must be called by all
// 32 lanes.
__device__ __forceinline__ void warp_append(bool flag, int val, int *list, int *tail, int cap = 0x7fffffff) {
    unsigned b = __ballot_sync(MF_FULL, flag);
    if (b == 0) return;
    int leader = __ffs(b) - 1;
    int base = 0;
    if (lane_id() == leader) base = atomicAdd(tail, __popc(b));
    base = __shfl_sync(MF_FULL, base, leader);
    if (flag) {
        int pos = base + __popc(b & lanemask_lt());
        if (MF_OK_IDX(pos, cap, 90)) list[pos] = val;
    }
}

// ---------------------------------------------------------------------------
// Group barrier.  A query group is G consecutive CTAs of a cooperative
// (co-resident) launch.  G == 1 is a plain __syncthreads.  Otherwise a
// sense-free generation barrier in global memory: thread 0 of each CTA
// arrives with a fenced atomicAdd; the last arriver resets the count and
// bumps the generation.  Every wait is bounded: past the deadline (or when
// another CTA has already raised *err) the waiter records MFD_TIMEOUT and
// leaves, and callers then unwind via gsync()'s return value.
struct GroupBar {
    unsigned arrive;
    unsigned gen;
    int snap;      // values captured by the last arriver (gsync_snap)
    int snap2;
    int snap3;
    int snap4;
};

// gsync_snap additionally returns, to every thread of the group, the values
// of *src and *src2 at the moment the last CTA arrived: all appends made
// before the barrier are counted and none made after it (a CTA that leaves
// the barrier early may already be appending).
__device__ __forceinline__ bool gsync_impl(int G, GroupBar *bar, int *err, u64 limit_ns,
                                           const int *src, const int *src2, int *snap_out,
                                           int *snap2_out, const int *src3 = nullptr,
                                           int *snap3_out = nullptr, const int *src4 = nullptr,
                                           int *snap4_out = nullptr) {
    __shared__ int s_ok;
    __shared__ int s_snap, s_snap2, s_snap3, s_snap4;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        if (G == 1 && src) {
            s_snap = *(volatile const int *)src;
            s_snap2 = *(volatile const int *)src2;
            if (src3) s_snap3 = *(volatile const int *)src3;
            if (src4) s_snap4 = *(volatile const int *)src4;
        }
        if (G > 1) {
            volatile unsigned *vgen = &bar->gen;
            unsigned gen0 = *vgen;
            __threadfence();
            unsigned prev = atomicAdd(&bar->arrive, 1u);
            if (prev == (unsigned)(G - 1)) {
                if (src) {
                    __threadfence();
                    *(volatile int *)&bar->snap = *(volatile const int *)src;
                    *(volatile int *)&bar->snap2 = *(volatile const int *)src2;
                    if (src3) *(volatile int *)&bar->snap3 = *(volatile const int *)src3;
                    if (src4) *(volatile int *)&bar->snap4 = *(volatile const int *)src4;
                }
                atomicExch(&bar->arrive, 0u);
                __threadfence();
                atomicAdd(&bar->gen, 1u);
            } else {
                u64 t0 = globaltimer_ns();
                unsigned spins = 0;
                while (*vgen == gen0) {
                    if (*(volatile int *)err) {
                        ok = 0;
                        break;
                    }
                    __nanosleep(40);
                    if ((++spins & 255u) == 0 && globaltimer_ns() - t0 > limit_ns) {
                        atomicCAS(err, 0, MFD_TIMEOUT);
                        ok = 0;
                        break;
                    }
                }
            }
            __threadfence();
            if (src) {
                s_snap = *(volatile int *)&bar->snap;
                s_snap2 = *(volatile int *)&bar->snap2;
                if (src3) s_snap3 = *(volatile int *)&bar->snap3;
                if (src4) s_snap4 = *(volatile int *)&bar->snap4;
            }
        }
        if (*(volatile int *)err) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    if (snap_out) {
        *snap_out = s_snap;
        *snap2_out = s_snap2;
    }
    if (snap3_out) *snap3_out = s_snap3;
    if (snap4_out) *snap4_out = s_snap4;
    return s_ok != 0;
}

__device__ __forceinline__ bool gsync(int G, GroupBar *bar, int *err, u64 limit_ns) {
    return gsync_impl(G, bar, err, limit_ns, nullptr, nullptr, nullptr, nullptr);
}

__device__ __forceinline__ bool gsync_snap(int G, GroupBar *bar, int *err, u64 limit_ns,
                                           const int *src, const int *src2, int *snap_out,
                                           int *snap2_out) {
    return gsync_impl(G, bar, err, limit_ns, src, src2, snap_out, snap2_out);
}

// ---------------------------------------------------------------------------
// Capacity-degree score, evaluated with a fixed sequence of IEEE double
// operations (no contraction) so that host and device agree bit for bit.
// ln(x) = k*ln2 + 2*atanh(z), x = m*2^k, m in [sqrt(1/2), sqrt(2)),
// z = (m-1)/(m+1), atanh summed as the odd power series up to z^23.
#ifdef __CUDA_ARCH__
#define MF_DMUL(a, b) __dmul_rn((a), (b))
#define MF_DADD(a, b) __dadd_rn((a), (b))
#define MF_DSUB(a, b) __dsub_rn((a), (b))
#define MF_DDIV(a, b) __ddiv_rn((a), (b))
#define MF_DSQRT(a) __dsqrt_rn((a))
#else
#define MF_DMUL(a, b) ((a) * (b))
#define MF_DADD(a, b) ((a) + (b))
#define MF_DSUB(a, b) ((a) - (b))
#define MF_DDIV(a, b) ((a) / (b))
#define MF_DSQRT(a) sqrt((a))
#endif

__host__ __device__ inline double mf_det_log(double x) {
    int k;
    double m = frexp(x, &k);
    if (m < 0.70710678118654752440) {
        m = MF_DMUL(m, 2.0);
        k = k - 1;
    }
    double z = MF_DDIV(MF_DSUB(m, 1.0), MF_DADD(m, 1.0));
    double z2 = MF_DMUL(z, z);
    double p = MF_DDIV(1.0, 23.0);
    for (int j = 21; j >= 1; j -= 2) {
        double t = MF_DMUL(p, z2);
        p = MF_DADD(t, MF_DDIV(1.0, (double)j));
    }
    double r = MF_DMUL(MF_DMUL(2.0, z), p);
    double kl = MF_DMUL((double)k, 0.69314718055994530942);
    return MF_DADD(kl, r);
}

// score = (ln(so*do+1) + ln(si*di+1)) / ln(sqrt(do*di)+1), 1 when the
// denominator is 0 (Region_Aware_PR_with_Pruning_BoundaryCore.cu:1141-1159).
__host__ __device__ inline double mf_score(i64 so, i64 si, int dout, int din) {
    double dso = (double)so, dsi = (double)si, ddo = (double)dout, ddi = (double)din;
    double a = MF_DMUL(dso, ddo);
    double b = MF_DMUL(dsi, ddi);
    double num = MF_DADD(mf_det_log(MF_DADD(a, 1.0)), mf_det_log(MF_DADD(b, 1.0)));
    double pd = MF_DMUL(ddo, ddi);
    double den = mf_det_log(MF_DADD(MF_DSQRT(pd), 1.0));
    if (den > 0.0) return MF_DDIV(num, den);
    return 1.0;
}
