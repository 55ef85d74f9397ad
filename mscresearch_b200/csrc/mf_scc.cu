// Strongly connected components of a device-resident graph and its SCC
// contraction, on the GPU.
//
// Reference: SCC_CONTRACT/scc_contract.cpp ("SC"), an offline host tool:
// Kosaraju over the input edges with capacity > 0 (SC:33-96), then one arc
// per ordered pair of distinct components with the summed capacity
// (SC:98-128).  Kosaraju's depth-first passes are sequential, so the device
// decomposition here is the usual data-parallel one:
//   1. trim: a vertex with no live out-arc or no live in-arc is a component
//      by itself (repeated while it removes vertices, a few passes);
//   2. forward-backward: the live vertices both reached from and reaching
//      the highest-degree live vertex form its component (two level-
//      synchronous searches);
//   3. colouring, until no vertex is left: every live vertex takes the
//      largest id of a live vertex that reaches it (max propagation over
//      in-arcs); a vertex whose colour is its own id is a root, and the live
//      vertices of that colour that reach it (a backward search that stays
//      on its colour) are its component; trim again.
// The arcs are the paired-arc CSR's: arc e = v -> col[e] with cap[e] > 0 is
// an edge v -> w, and cap[rev[e]] > 0 is an edge w -> v, so both directions
// read v's own arc list.  Components are numbered in the order of their
// smallest caller vertex id (Kosaraju's numbering depends on its search
// order; the partition and the contracted graph are the same up to that
// numbering).  Every loop ends by convergence of a monotone quantity (live
// vertices, colours, search frontiers); no kernel waits on another.
#include <algorithm>
#include <climits>
#include <vector>

#include "mf_alloc.h"
#include "mf_build.cuh"
#include "mf_scc.cuh"

namespace {

constexpr int ST = 256;  // threads per block

int blocks_for_warps(long long warps) {
    long long b = (warps * 32 + ST - 1) / ST;
    return (int)std::max(1LL, std::min(b, 148LL * 64));
}
int blocks_for(long long items) { return (int)std::max(1LL, std::min((items + ST - 1) / ST, 148LL * 64)); }

// A live vertex without a live out-neighbour or without a live in-neighbour
// becomes a component by itself (comp = its id).  One warp per vertex.
__global__ void k_trim(int n, const int *row, const int *col, const int *rev, const i64 *cap, int *comp,
                       int *changed) {
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int v = gw; v < n; v += nw) {
        if (comp[v] >= 0) continue;
        const int b = row[v], e1 = row[v + 1];
        bool o = false, in = false;
        for (int base = b; base < e1 && !(o && in); base += 32) {
            const int e = base + lane;
            bool lo = false, li = false;
            if (e < e1) {
                const int w = col[e];
                if (w != v && comp[w] < 0) {
                    lo = cap[e] > 0;
                    li = cap[rev[e]] > 0;
                }
            }
            o = o || __any_sync(MF_FULL, lo);
            in = in || __any_sync(MF_FULL, li);
        }
        if (!(o && in) && lane == 0) {
            comp[v] = v;
            *changed = 1;
        }
    }
}

// Live vertex count and the live vertex of highest degree (smaller id on
// ties), packed as (degree << 32) | (~id).
__global__ void k_pick(int n, const int *row, const int *comp, unsigned long long *best, int *live) {
    unsigned long long b = 0;
    int cnt = 0;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        if (comp[v] >= 0) continue;
        ++cnt;
        const unsigned long long k = ((unsigned long long)(unsigned)(row[v + 1] - row[v]) << 32) |
                                     (unsigned long long)(0xffffffffu - (unsigned)v);
        b = k > b ? k : b;
    }
    cnt = __reduce_add_sync(MF_FULL, cnt);
    for (int o = 16; o; o >>= 1) {
        const unsigned long long x = __shfl_xor_sync(MF_FULL, b, o);
        b = x > b ? x : b;
    }
    if ((threadIdx.x & 31) == 0) {
        if (cnt) atomicAdd(live, cnt);
        if (b) atomicMax(best, b);
    }
}

// Warp-aggregated append of w (flagged lanes) to Q.
__device__ __forceinline__ void push(bool f, int w, int *Q, int *qn) {
    const unsigned m = __ballot_sync(MF_FULL, f);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    int base = 0;
    if (lane == __ffs(m) - 1) base = atomicAdd(qn, __popc(m));
    base = __shfl_sync(MF_FULL, base, __ffs(m) - 1);
    if (f) Q[base + __popc(m & ((1u << lane) - 1))] = w;
}

// One level of the forward (bit 1, out-arcs) or backward (bit 2, in-arcs)
// search from the pivot over live vertices; one warp per frontier vertex.
__global__ void k_fb_level(const int *Q, int qn, int *Q2, int *q2n, const int *row, const int *col,
                           const int *rev, const i64 *cap, const int *comp, int *mark, int bit) {
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = gw; i < qn; i += nw) {
        const int x = Q[i];
        const int b = row[x], e1 = row[x + 1];
        for (int base = b; base < e1; base += 32) {
            const int e = base + lane;
            bool f = false;
            int w = 0;
            if (e < e1) {
                w = col[e];
                const bool arc = bit == 1 ? cap[e] > 0 : cap[rev[e]] > 0;
                if (arc && comp[w] < 0 && !(mark[w] & bit)) f = !(atomicOr(&mark[w], bit) & bit);
            }
            push(f, w, Q2, q2n);
        }
    }
}

// Vertices both searches reached join the pivot's component.
__global__ void k_fb_assign(int n, const int *mark, int *comp, int pivot) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        if (comp[v] < 0 && mark[v] == 3) comp[v] = pivot;
}

__global__ void k_color_init(int n, const int *comp, int *color) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        color[v] = comp[v] < 0 ? v : -1;
}

// color[v] = max(color[v], colours of its live in-neighbours); one warp per
// live vertex.  Only v's warp writes color[v]; colours only grow.
__global__ void k_color_prop(int n, const int *row, const int *col, const int *rev, const i64 *cap,
                             const int *comp, int *color, int *changed) {
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int v = gw; v < n; v += nw) {
        if (comp[v] >= 0) continue;
        const int b = row[v], e1 = row[v + 1];
        int m = -1;
        for (int e = b + lane; e < e1; e += 32) {
            const int w = col[e];
            if (comp[w] < 0 && cap[rev[e]] > 0) m = max(m, color[w]);
        }
        m = __reduce_max_sync(MF_FULL, m);
        if (lane == 0 && m > color[v]) {
            color[v] = m;
            *changed = 1;
        }
    }
}

// Roots (colour == own id) take their own component and start the search.
__global__ void k_color_roots(int n, int *comp, const int *color, int *Q, int *qn) {
    for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const int v = base + threadIdx.x;
        const bool r = v < n && comp[v] < 0 && color[v] == v;
        if (r) comp[v] = v;
        push(r, v, Q, qn);
    }
}

// One level of the backward searches from the roots: a live in-neighbour
// of the same colour joins the root's component.
__global__ void k_color_level(const int *Q, int qn, int *Q2, int *q2n, const int *row, const int *col,
                              const int *rev, const i64 *cap, int *comp, const int *color) {
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = gw; i < qn; i += nw) {
        const int x = Q[i];
        const int r = comp[x];
        const int b = row[x], e1 = row[x + 1];
        for (int base = b; base < e1; base += 32) {
            const int e = base + lane;
            bool f = false;
            int w = 0;
            if (e < e1) {
                w = col[e];
                if (comp[w] < 0 && color[w] == r && cap[rev[e]] > 0) f = atomicCAS(&comp[w], -1, r) == -1;
            }
            push(f, w, Q2, q2n);
        }
    }
}

// Smallest caller id per component (indexed by the representative).
__global__ void k_minc(int n, const int *comp, const int *old_id, int *minc) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        if (comp[v] >= 0) atomicMin(&minc[comp[v]], old_id[v]);
}

// first[x] = 1 when caller vertex x is its component's smallest.
__global__ void k_first(int n, const int *new_id, const int *comp, const int *minc, int *first) {
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n; x += gridDim.x * blockDim.x)
        first[x] = minc[comp[new_id[x]]] == x;
}

// Component numbers: cid[v] (internal ids) and label[x] (caller ids).
__global__ void k_number(int n, const int *new_id, const int *comp, const int *minc, const int *rank, int *cid,
                         int *label) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        cid[v] = rank[minc[comp[v]]];
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n; x += gridDim.x * blockDim.x)
        label[x] = rank[minc[comp[new_id[x]]]];
}

// Arcs between distinct components (one entry per edge with capacity > 0);
// one warp per vertex.
__global__ void k_emit(int n, const int *row, const int *col, const i64 *cap, const int *cid, int *ea, int *eb,
                       i64 *ec, int *cnt) {
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int v = gw; v < n; v += nw) {
        const int a = cid[v];
        const int b0 = row[v], e1 = row[v + 1];
        for (int base = b0; base < e1; base += 32) {
            const int e = base + lane;
            bool f = false;
            int b = 0;
            i64 c = 0;
            if (e < e1) {
                c = cap[e];
                b = cid[col[e]];
                f = c > 0 && b != a;
            }
            const unsigned m = __ballot_sync(MF_FULL, f);
            if (!m) continue;
            int pos = 0;
            if (lane == __ffs(m) - 1) pos = atomicAdd(cnt, __popc(m));
            pos = __shfl_sync(MF_FULL, pos, __ffs(m) - 1) + __popc(m & ((1u << lane) - 1));
            if (f) {
                ea[pos] = a;
                eb[pos] = b;
                ec[pos] = c;
            }
        }
    }
}

__global__ void k_iota(int N, int *a) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) a[i] = i;
}

__global__ void k_gather(int N, const int *idx, const int *src, int *dst) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) dst[i] = src[idx[i]];
}

// head[i] = 1 where the sorted pair (a, b) differs from the one before.
__global__ void k_heads(int N, const int *idx, const int *ea, const int *eb, int *head) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const int j = idx[i];
        head[i] = i == 0 || ea[j] != ea[idx[i - 1]] || eb[j] != eb[idx[i - 1]];
    }
}

// Sums each run of equal pairs into one contracted arc (pos: exclusive scan
// of head, so the run of item i is pos[i] + head[i] - 1).
__global__ void k_sum(int N, const int *idx, const int *ea, const int *eb, const i64 *ec, const int *head,
                      const int *pos, int *ou, int *ov, i64 *oc) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const int j = idx[i];
        const int k = pos[i] + head[i] - 1;
        if (head[i]) {
            ou[k] = ea[j];
            ov[k] = eb[j];
        }
        atomic_add_i64(&oc[k], ec[j]);
    }
}

int scan_tmp_ints(int n) { return n / 1024 + 2; }

}  // namespace

#define SCC_CK(x)                            \
    do {                                     \
        cudaError_t e_ = (x);                \
        if (e_ != cudaSuccess) return e_;    \
    } while (0)

cudaError_t mf_scc_run(const SccIn &in, cudaStream_t st, SccOut &out) {
    const int n = in.n;
    out = SccOut{};
    if (n <= 0) return cudaSuccess;
    DevScope t;
    int *comp, *mark, *color, *Q, *Q2, *qn, *flag, *live, *minc, *first, *rank, *cid, *label, *nid, *oid, *stmp;
    unsigned long long *best;
    SCC_CK(t.alloc(&comp, sizeof(int) * n));
    SCC_CK(t.alloc(&mark, sizeof(int) * n));
    SCC_CK(t.alloc(&color, sizeof(int) * n));
    SCC_CK(t.alloc(&Q, sizeof(int) * n));
    SCC_CK(t.alloc(&Q2, sizeof(int) * n));
    SCC_CK(t.alloc(&qn, sizeof(int) * 2));
    SCC_CK(t.alloc(&flag, sizeof(int)));
    SCC_CK(t.alloc(&live, sizeof(int)));
    SCC_CK(t.alloc(&best, sizeof(unsigned long long)));
    SCC_CK(cudaMemsetAsync(comp, 0xff, sizeof(int) * n, st));
    SCC_CK(cudaMemsetAsync(mark, 0, sizeof(int) * n, st));
    const int *row = in.row, *col = in.col, *rev = in.rev;
    const i64 *cap = in.cap;
    const int BW = blocks_for_warps(n), B = blocks_for(n);
    auto get = [&](const int *d, int &h) -> cudaError_t {
        cudaError_t e = cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, st);
        return e ? e : cudaStreamSynchronize(st);
    };
    auto trim = [&](int passes) -> cudaError_t {
        for (int p = 0; p < passes; ++p) {
            int ch = 0;
            SCC_CK(cudaMemsetAsync(flag, 0, sizeof(int), st));
            k_trim<<<BW, ST, 0, st>>>(n, row, col, rev, cap, comp, flag);
            SCC_CK(get(flag, ch));
            if (!ch) break;
        }
        return cudaSuccess;
    };
    // level-synchronous search from the n0 vertices in Q; kern runs a level
    auto search = [&](int n0, auto kern) -> cudaError_t {
        int *a = Q, *b = Q2, qa = n0;
        while (qa > 0) {
            SCC_CK(cudaMemsetAsync(qn, 0, sizeof(int), st));
            kern(a, qa, b, qn);
            int qb = 0;
            SCC_CK(get(qn, qb));
            std::swap(a, b);
            qa = qb;
        }
        return cudaSuccess;
    };
    // 1. trim
    SCC_CK(trim(8));
    // 2. forward-backward from the highest-degree live vertex
    {
        SCC_CK(cudaMemsetAsync(live, 0, sizeof(int), st));
        SCC_CK(cudaMemsetAsync(best, 0, sizeof(unsigned long long), st));
        k_pick<<<B, ST, 0, st>>>(n, row, comp, best, live);
        unsigned long long hb = 0;
        int hl = 0;
        SCC_CK(cudaMemcpyAsync(&hb, best, sizeof(hb), cudaMemcpyDeviceToHost, st));
        SCC_CK(get(live, hl));
        if (hl > 0) {
            const int pivot = (int)(0xffffffffu - (unsigned)(hb & 0xffffffffull));
            // the pivot starts each search marked with that search's bit
            // only, and holds both once they are done
            for (int bit = 1; bit <= 2; bit <<= 1) {
                SCC_CK(cudaMemcpyAsync(Q, &pivot, sizeof(int), cudaMemcpyHostToDevice, st));
                const int pm = bit;
                SCC_CK(cudaMemcpyAsync(mark + pivot, &pm, sizeof(int), cudaMemcpyHostToDevice, st));
                SCC_CK(search(1, [&](int *a, int qa, int *b, int *qb) {
                    k_fb_level<<<blocks_for_warps(qa), ST, 0, st>>>(a, qa, b, qb, row, col, rev, cap, comp, mark, bit);
                }));
            }
            const int both = 3;
            SCC_CK(cudaMemcpyAsync(mark + pivot, &both, sizeof(int), cudaMemcpyHostToDevice, st));
            k_fb_assign<<<B, ST, 0, st>>>(n, mark, comp, pivot);
        }
    }
    // 3. colouring rounds until no live vertex is left (each round settles
    // at least the component of the live vertex with the largest id)
    bool settled = false;
    for (int round = 0; round <= n && !settled; ++round) {
        SCC_CK(trim(2));
        int hl = 0;
        SCC_CK(cudaMemsetAsync(live, 0, sizeof(int), st));
        SCC_CK(cudaMemsetAsync(best, 0, sizeof(unsigned long long), st));
        k_pick<<<B, ST, 0, st>>>(n, row, comp, best, live);
        SCC_CK(get(live, hl));
        settled = hl == 0;
        if (settled) break;
        k_color_init<<<B, ST, 0, st>>>(n, comp, color);
        for (int it = 0; it <= n; ++it) {
            int ch = 0;
            SCC_CK(cudaMemsetAsync(flag, 0, sizeof(int), st));
            k_color_prop<<<BW, ST, 0, st>>>(n, row, col, rev, cap, comp, color, flag);
            SCC_CK(get(flag, ch));
            if (!ch) break;
        }
        SCC_CK(cudaMemsetAsync(qn, 0, sizeof(int), st));
        k_color_roots<<<B, ST, 0, st>>>(n, comp, color, Q, qn);
        int nr = 0;
        SCC_CK(get(qn, nr));
        SCC_CK(search(nr, [&](int *a, int qa, int *b, int *qb) {
            k_color_level<<<blocks_for_warps(qa), ST, 0, st>>>(a, qa, b, qb, row, col, rev, cap, comp, color);
        }));
    }
    if (!settled) return cudaErrorUnknown;  // not reached: every round settles a component
    // numbering by smallest caller id
    SCC_CK(t.alloc(&minc, sizeof(int) * n));
    SCC_CK(t.alloc(&first, sizeof(int) * n));
    SCC_CK(t.alloc(&rank, sizeof(int) * n));
    SCC_CK(t.alloc(&cid, sizeof(int) * n));
    SCC_CK(t.alloc(&label, sizeof(int) * n));
    SCC_CK(t.alloc(&nid, sizeof(int) * n));
    SCC_CK(t.alloc(&oid, sizeof(int) * n));
    SCC_CK(t.alloc(&stmp, sizeof(int) * scan_tmp_ints(n)));
    SCC_CK(cudaMemcpyAsync(nid, in.new_id, sizeof(int) * n, cudaMemcpyHostToDevice, st));
    SCC_CK(cudaMemcpyAsync(oid, in.old_id, sizeof(int) * n, cudaMemcpyHostToDevice, st));
    SCC_CK(cudaMemsetAsync(minc, 0x7f, sizeof(int) * n, st));  // 0x7f7f7f7f > any id
    k_minc<<<B, ST, 0, st>>>(n, comp, oid, minc);
    k_first<<<B, ST, 0, st>>>(n, nid, comp, minc, first);
    mf_exclusive_scan(n, first, rank, stmp, st);
    k_number<<<B, ST, 0, st>>>(n, nid, comp, minc, rank, cid, label);
    int last_rank = 0, last_first = 0;
    SCC_CK(cudaMemcpyAsync(&last_rank, rank + n - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    SCC_CK(get(first + n - 1, last_first));
    out.ncomp = last_rank + last_first;
    out.comp.resize(n);
    SCC_CK(cudaMemcpyAsync(out.comp.data(), label, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    // contraction
    const i64 A = std::max<i64>(in.arcs, 1);
    int *ea, *eb, *ka, *kb, *va, *vb, *cnt, *head, *pos, *ou, *ov;
    i64 *ec, *oc;
    SCC_CK(t.alloc(&ea, sizeof(int) * A));
    SCC_CK(t.alloc(&eb, sizeof(int) * A));
    SCC_CK(t.alloc(&ec, sizeof(i64) * A));
    SCC_CK(t.alloc(&cnt, sizeof(int)));
    SCC_CK(cudaMemsetAsync(cnt, 0, sizeof(int), st));
    k_emit<<<BW, ST, 0, st>>>(n, row, col, cap, cid, ea, eb, ec, cnt);
    int M = 0;
    SCC_CK(get(cnt, M));
    if (M > 0) {
        SCC_CK(t.alloc(&ka, sizeof(int) * M));
        SCC_CK(t.alloc(&kb, sizeof(int) * M));
        SCC_CK(t.alloc(&va, sizeof(int) * M));
        SCC_CK(t.alloc(&vb, sizeof(int) * M));
        SCC_CK(t.alloc(&head, sizeof(int) * M));
        SCC_CK(t.alloc(&pos, sizeof(int) * M));
        SCC_CK(t.alloc(&ou, sizeof(int) * M));
        SCC_CK(t.alloc(&ov, sizeof(int) * M));
        SCC_CK(t.alloc(&oc, sizeof(i64) * M));
        int *st2 = nullptr;
        SCC_CK(t.alloc(&st2, sizeof(int) * scan_tmp_ints(M)));
        const int BM = blocks_for(M);
        // by b, then stably by a: the order (a, b)
        SCC_CK(cudaMemcpyAsync(ka, eb, sizeof(int) * M, cudaMemcpyDeviceToDevice, st));
        k_iota<<<BM, ST, 0, st>>>(M, va);
        int *k1 = ka, *v1 = va, *k2 = kb, *v2 = vb;
        SCC_CK(mf_radix_sort_pairs(M, out.ncomp - 1, k1, v1, k2, v2, st));
        k_gather<<<BM, ST, 0, st>>>(M, v1, ea, k1);
        SCC_CK(mf_radix_sort_pairs(M, out.ncomp - 1, k1, v1, k2, v2, st));
        k_heads<<<BM, ST, 0, st>>>(M, v1, ea, eb, head);
        mf_exclusive_scan(M, head, pos, st2, st);
        int lp = 0, lh = 0;
        SCC_CK(cudaMemcpyAsync(&lp, pos + M - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        SCC_CK(cudaMemcpyAsync(&lh, head + M - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        SCC_CK(cudaMemsetAsync(oc, 0, sizeof(i64) * M, st));
        k_sum<<<BM, ST, 0, st>>>(M, v1, ea, eb, ec, head, pos, ou, ov, oc);
        SCC_CK(cudaStreamSynchronize(st));
        const int K = lp + lh;
        out.cu.resize(K);
        out.cv.resize(K);
        out.cap.resize(K);
        SCC_CK(cudaMemcpyAsync(out.cu.data(), ou, sizeof(int) * K, cudaMemcpyDeviceToHost, st));
        SCC_CK(cudaMemcpyAsync(out.cv.data(), ov, sizeof(int) * K, cudaMemcpyDeviceToHost, st));
        SCC_CK(cudaMemcpyAsync(out.cap.data(), oc, sizeof(i64) * K, cudaMemcpyDeviceToHost, st));
    }
    SCC_CK(cudaStreamSynchronize(st));
    return cudaGetLastError();
}
