// Device-side graph ingest: graph.txt token parse and the paired-arc CSR
// build, both on the GPU.
//
// Reference (Region_Aware_PR_with_Pruning_BoundaryCore.cu, "RA"):
//   build_graph RA:1044-1126 -- an "n m" header, then up to m "u v cap"
//   triples read as an fscanf token stream, stopping at the first triple
//   that does not scan (RA:1068-1075); edges with an endpoint outside
//   [0, n), u == v or cap <= 0 are skipped; every kept edge appends its
//   forward arc to u's list and a zero-capacity reverse arc to v's list, in
//   input order (RA:1090-1122).
//
// Token stream on the device.  fscanf("%d"/"%lld") skips white space, takes
// an optional sign and one or more digits, and fails on anything else.  So
// the stream is valid up to the first byte that is neither white space, a
// digit, nor a sign followed by a digit; an integer starts at a sign
// followed by a digit, or at a digit preceded by neither a digit nor a sign.
// Both tests look at one byte and its neighbours, so every byte is
// classified in parallel; the token index of a start is a prefix count.
//
// CSR on the device.  Vertex x's arc list in the host build is every kept
// edge incident to x in input order.  Half-arc h = 2 * i + side (side 0:
// the forward arc, keyed by u[i]; side 1: the reverse arc, keyed by v[i];
// skipped edges keyed n) sorted stably by key gives exactly that order, so
// a stable LSD radix sort (8-bit digits, per-chunk histograms, a scan, and
// warp-stable placement with __match_any_sync) yields the CSR positions.
#include <algorithm>
#include <cstdio>
#include <vector>

#include "mf_alloc.h"
#include "mf_build.cuh"

namespace {

__device__ __forceinline__ bool tk_space(unsigned c) { return c == ' ' || (c >= '\t' && c <= '\r'); }
__device__ __forceinline__ bool tk_digit(unsigned c) { return c - '0' < 10u; }
__device__ __forceinline__ bool tk_sign(unsigned c) { return c == '+' || c == '-'; }

#define TOK_B 1024

// Per byte: does an integer start here, and does the token stream end here?
__device__ __forceinline__ void tk_classify(i64 S, const unsigned char *txt, i64 i, bool &start, bool &bad) {
    start = bad = false;
    if (i >= S) return;
    unsigned c = txt[i];
    unsigned nx = (i + 1 < S) ? txt[i + 1] : 0u;
    unsigned pv = (i > 0) ? txt[i - 1] : (unsigned)' ';
    bool sg = tk_sign(c) && tk_digit(nx);
    bad = !tk_space(c) && !tk_digit(c) && !sg;
    start = sg || (tk_digit(c) && !tk_digit(pv) && !tk_sign(pv));
}

// Pass 1: integer starts per block, and the first byte that ends the stream.
__global__ void k_tok_count(i64 S, const unsigned char *txt, int *bcount, u64 *first_bad) {
    i64 i = (i64)blockIdx.x * TOK_B + threadIdx.x;
    bool st, bad;
    tk_classify(S, txt, i, st, bad);
    int c = __syncthreads_count(st);
    if (threadIdx.x == 0) bcount[blockIdx.x] = c;
    unsigned bb = __ballot_sync(MF_FULL, bad);
    if (bb && (threadIdx.x & 31) == __ffs(bb) - 1) atomicMin(first_bad, (u64)i);
}

// Pass 2: each start before the stream's end parses its integer as fscanf
// does: the magnitude saturates at the 64-bit limit of its sign (strtoll's
// rule), then the sign applies.
__global__ void k_tok_values(i64 S, const unsigned char *txt, const int *boff, const u64 *first_bad,
                             i64 *tok, int *ntok) {
    __shared__ int wsum[TOK_B / 32];
    i64 i = (i64)blockIdx.x * TOK_B + threadIdx.x;
    bool st, bad;
    tk_classify(S, txt, i, st, bad);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned b = __ballot_sync(MF_FULL, st);
    if (lane == 0) wsum[warp] = __popc(b);
    __syncthreads();
    if (threadIdx.x < 32) {
        int x = (lane < TOK_B / 32) ? wsum[lane] : 0;
        int incl = x;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(MF_FULL, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane < TOK_B / 32) wsum[lane] = incl - x;
    }
    __syncthreads();
    if (!st || (u64)i >= *first_bad) return;
    int idx = boff[blockIdx.x] + wsum[warp] + __popc(b & lanemask_lt());
    i64 p = i;
    bool neg = false;
    if (tk_sign(txt[p])) {
        neg = txt[p] == '-';
        ++p;
    }
    const u64 lim = neg ? (1ull << 63) : (1ull << 63) - 1ull;
    u64 x = 0;
    bool over = false;
    while (p < S && tk_digit(txt[p])) {
        const u64 d = (u64)(txt[p] - '0');
        if (x > (lim - d) / 10ull) over = true;
        else x = x * 10ull + d;
        ++p;
    }
    if (over) x = lim;
    tok[idx] = (i64)(neg ? (~x + 1ull) : x);
    atomicMax(ntok, idx + 1);
}

// Triples after the header: u, v are 1-based in the file; "%d" keeps the
// low 32 bits of the scanned value.
__global__ void k_tok_edges(i64 m, const i64 *tok, int *u, int *v, i64 *c) {
    for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (i64)gridDim.x * blockDim.x) {
        u[e] = (int)((unsigned)tok[2 + 3 * e] - 1u);
        v[e] = (int)((unsigned)tok[3 + 3 * e] - 1u);
        c[e] = tok[4 + 3 * e];
    }
}

// ---- stable LSD radix sort of (key, half-arc) pairs ------------------------
#define RS_CHUNK 4096
#define RS_WARPS 16
#define RS_BINS 256

__device__ __forceinline__ bool edge_kept(int n, int a, int b, i64 c) {
    return a >= 0 && a < n && b >= 0 && b < n && a != b && c > 0;
}

// Half-arcs in input order: h = 2 i + side, key = tail (n when skipped).
__global__ void k_halfarcs(int n, i64 m, const int *u, const int *v, const i64 *c, int *key, int *val) {
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (i64)gridDim.x * blockDim.x) {
        int a = u[i], b = v[i];
        bool k = edge_kept(n, a, b, c[i]);
        key[2 * i] = k ? a : n;
        key[2 * i + 1] = k ? b : n;
        val[2 * i] = (int)(2 * i);
        val[2 * i + 1] = (int)(2 * i + 1);
    }
}

__global__ void k_rs_hist(int N, const int *key, int shift, int nchunks, int *cnt) {
    __shared__ int h[RS_BINS];
    for (int b = threadIdx.x; b < RS_BINS; b += blockDim.x) h[b] = 0;
    __syncthreads();
    const i64 base = (i64)blockIdx.x * RS_CHUNK;
    for (int t = threadIdx.x; t < RS_CHUNK; t += blockDim.x) {
        i64 i = base + t;
        if (i < N) atomicAdd(&h[(key[i] >> shift) & (RS_BINS - 1)], 1);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < RS_BINS; b += blockDim.x) cnt[(size_t)b * nchunks + blockIdx.x] = h[b];
}

// Warp w of chunk c places items [c*CHUNK + w*per, +per) in order: equal
// digits inside a 32-item step rank by lane (peer mask), steps in order,
// warps in order (prefix over the per-warp digit totals), chunks in order
// (the digit-major scan of the histograms).
__global__ void k_rs_place(int N, const int *key, const int *val, int shift, int nchunks, const int *off,
                           int *key2, int *val2) {
    __shared__ int wc[RS_WARPS * RS_BINS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < RS_WARPS * RS_BINS; i += blockDim.x) wc[i] = 0;
    __syncthreads();
    const int per = RS_CHUNK / RS_WARPS;
    const i64 base = (i64)blockIdx.x * RS_CHUNK + warp * per;
    for (int s = 0; s < per; s += 32) {
        i64 i = base + s + lane;
        int d = (i < N) ? ((key[i] >> shift) & (RS_BINS - 1)) : -1;
        unsigned peers = __match_any_sync(MF_FULL, d);
        if (d >= 0 && (peers & lanemask_lt()) == 0) wc[warp * RS_BINS + d] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    for (int b = threadIdx.x; b < RS_BINS; b += blockDim.x) {
        int acc = off[(size_t)b * nchunks + blockIdx.x];
        for (int w = 0; w < RS_WARPS; ++w) {
            int x = wc[w * RS_BINS + b];
            wc[w * RS_BINS + b] = acc;
            acc += x;
        }
    }
    __syncthreads();
    for (int s = 0; s < per; s += 32) {
        i64 i = base + s + lane;
        int k = 0, vv = 0, d = -1;
        if (i < N) {
            k = key[i];
            vv = val[i];
            d = (k >> shift) & (RS_BINS - 1);
        }
        unsigned peers = __match_any_sync(MF_FULL, d);
        if (d >= 0) {
            int pos = wc[warp * RS_BINS + d] + __popc(peers & lanemask_lt());
            key2[pos] = k;
            val2[pos] = vv;
        }
        __syncwarp();
        if (d >= 0 && (peers & lanemask_lt()) == 0) wc[warp * RS_BINS + d] += __popc(peers);
        __syncwarp();
    }
}

// Degrees from the sorted keys: each run of key x (x < n) spans [first, last].
__global__ void k_runs_deg(int N, int n, const int *key, int *deg) {
    for (i64 p = (i64)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (i64)gridDim.x * blockDim.x) {
        int x = key[p];
        if (x >= n) continue;
        // deg[x] = (last + 1) - first, one add at each end of the run
        if (p + 1 == N || key[p + 1] != x) atomicAdd(&deg[x], (int)(p + 1));
        if (p == 0 || key[p - 1] != x) atomicAdd(&deg[x], -(int)p);
    }
}

__global__ void k_pos_of(int arcs, const int *val, int *pos_of) {
    for (i64 p = (i64)blockIdx.x * blockDim.x + threadIdx.x; p < arcs; p += (i64)gridDim.x * blockDim.x)
        pos_of[val[p]] = (int)p;
}

__global__ void k_csr_arcs(int arcs, const int *val, const int *pos_of, const int *u, const int *v,
                           const i64 *c, int *col, i64 *cap, int *rev, unsigned char *fwd) {
    for (i64 p = (i64)blockIdx.x * blockDim.x + threadIdx.x; p < arcs; p += (i64)gridDim.x * blockDim.x) {
        int h = val[p];
        i64 i = h >> 1;
        bool back = h & 1;
        col[p] = back ? u[i] : v[i];
        cap[p] = back ? 0 : c[i];
        fwd[p] = back ? 0 : 1;
        rev[p] = pos_of[h ^ 1];
    }
}

int grid_of(i64 work, int threads) {
    i64 b = (work + threads - 1) / threads;
    return (int)std::max<i64>(1, std::min<i64>(b, 148 * 16));
}

}  // namespace

cudaError_t mf_device_csr(int n, i64 m, const int *u, const int *v, const i64 *c, cudaStream_t st,
                          DevCsr &out) {
    out = DevCsr{};
    const i64 N = 2 * m;
    if (N > 0x7fffffffLL) return cudaErrorInvalidValue;
    cudaError_t e = cudaSuccess;
    int *key = nullptr, *val = nullptr, *key2 = nullptr, *val2 = nullptr, *cnt = nullptr, *off = nullptr,
        *tmp = nullptr, *deg = nullptr, *pos = nullptr;
    const int nchunks = (int)std::max<i64>(1, (N + RS_CHUNK - 1) / RS_CHUNK);
    const int nbins = RS_BINS * nchunks;
    int passes = 0;
    for (unsigned x = (unsigned)n; x; x >>= 8) ++passes;
    do {
        const size_t NN = (size_t)std::max<i64>(N, 1);
        if ((e = mf_dmalloc(&key, sizeof(int) * NN)) || (e = mf_dmalloc(&val, sizeof(int) * NN)) ||
            (e = mf_dmalloc(&key2, sizeof(int) * NN)) || (e = mf_dmalloc(&val2, sizeof(int) * NN)) ||
            (e = mf_dmalloc(&cnt, sizeof(int) * (size_t)nbins)) ||
            (e = mf_dmalloc(&off, sizeof(int) * ((size_t)nbins + 1))) ||
            (e = mf_dmalloc(&tmp, sizeof(int) * ((size_t)std::max(nbins, n + 1) / 1024 + 2))) ||
            (e = mf_dmalloc(&deg, sizeof(int) * ((size_t)n + 1))) ||
            (e = mf_dmalloc(&out.row, sizeof(int) * ((size_t)n + 1))))
            break;
        if (m > 0) k_halfarcs<<<grid_of(m, 256), 256, 0, st>>>(n, m, u, v, c, key, val);
        for (int ps = 0; ps < passes && N > 0; ++ps) {
            const int shift = 8 * ps;
            k_rs_hist<<<nchunks, 512, 0, st>>>((int)N, key, shift, nchunks, cnt);
            mf_exclusive_scan(nbins, cnt, off, tmp, st);
            k_rs_place<<<nchunks, 32 * RS_WARPS, 0, st>>>((int)N, key, val, shift, nchunks, off, key2, val2);
            std::swap(key, key2);
            std::swap(val, val2);
        }
        if ((e = cudaMemsetAsync(deg, 0, sizeof(int) * ((size_t)n + 1), st))) break;
        if (N > 0) k_runs_deg<<<grid_of(N, 256), 256, 0, st>>>((int)N, n, key, deg);
        mf_exclusive_scan(n, deg, out.row, tmp, st);
        int arcs = 0;
        if ((e = cudaMemcpyAsync(&arcs, out.row + n, sizeof(int), cudaMemcpyDeviceToHost, st)) ||
            (e = cudaStreamSynchronize(st)))
            break;
        out.arcs = arcs;
        const size_t A = (size_t)std::max(arcs, 1);
        if ((e = mf_dmalloc(&out.col, sizeof(int) * A)) || (e = mf_dmalloc(&out.cap, sizeof(i64) * A)) ||
            (e = mf_dmalloc(&out.rev, sizeof(int) * A)) || (e = mf_dmalloc(&out.fwd, A)) ||
            (e = mf_dmalloc(&pos, sizeof(int) * NN)))
            break;
        if (arcs > 0) {
            k_pos_of<<<grid_of(arcs, 256), 256, 0, st>>>(arcs, val, pos);
            k_csr_arcs<<<grid_of(arcs, 256), 256, 0, st>>>(arcs, val, pos, u, v, c, out.col, out.cap, out.rev,
                                                            out.fwd);
        }
        e = cudaStreamSynchronize(st);
        if (e == cudaSuccess) e = cudaGetLastError();
    } while (0);
    mf_dfree(key);
    mf_dfree(val);
    mf_dfree(key2);
    mf_dfree(val2);
    mf_dfree(cnt);
    mf_dfree(off);
    mf_dfree(tmp);
    mf_dfree(deg);
    mf_dfree(pos);
    if (e != cudaSuccess) mf_free_dev_csr(out);
    return e;
}

cudaError_t mf_radix_sort_pairs(int N, int key_max, int *&key, int *&val, int *&key2, int *&val2,
                                cudaStream_t st) {
    if (N <= 0 || key_max <= 0) return cudaSuccess;
    const int nchunks = (N + RS_CHUNK - 1) / RS_CHUNK;
    const int nbins = RS_BINS * nchunks;
    DevScope tmp;
    int *cnt = nullptr, *off = nullptr, *stmp = nullptr;
    cudaError_t e;
    if ((e = tmp.alloc(&cnt, sizeof(int) * (size_t)nbins)) || (e = tmp.alloc(&off, sizeof(int) * ((size_t)nbins + 1))) ||
        (e = tmp.alloc(&stmp, sizeof(int) * ((size_t)nbins / 1024 + 2))))
        return e;
    for (unsigned x = (unsigned)key_max, shift = 0; x; x >>= 8, shift += 8) {
        k_rs_hist<<<nchunks, 512, 0, st>>>(N, key, (int)shift, nchunks, cnt);
        mf_exclusive_scan(nbins, cnt, off, stmp, st);
        k_rs_place<<<nchunks, 32 * RS_WARPS, 0, st>>>(N, key, val, (int)shift, nchunks, off, key2, val2);
        std::swap(key, key2);
        std::swap(val, val2);
    }
    if ((e = cudaGetLastError())) return e;
    return cudaStreamSynchronize(st);  // the scratch is freed on return
}

void mf_free_dev_csr(DevCsr &c) {
    mf_dfree(c.row);
    mf_dfree(c.col);
    mf_dfree(c.cap);
    mf_dfree(c.rev);
    mf_dfree(c.fwd);
    c = DevCsr{};
}

cudaError_t mf_parse_graph_text(const unsigned char *txt, i64 S, cudaStream_t st, TextEdges &out) {
    out = TextEdges{};
    cudaError_t e = cudaSuccess;
    int *bcount = nullptr, *boff = nullptr, *tmp = nullptr, *ntok = nullptr;
    u64 *first_bad = nullptr;
    i64 *tok = nullptr;
    const i64 nb64 = std::max<i64>(1, (S + TOK_B - 1) / TOK_B);
    if (nb64 > 0x7fffffffLL) return cudaErrorInvalidValue;
    const int nb = (int)nb64;
    do {
        if ((e = mf_dmalloc(&bcount, sizeof(int) * (size_t)nb)) ||
            (e = mf_dmalloc(&boff, sizeof(int) * ((size_t)nb + 1))) ||
            (e = mf_dmalloc(&tmp, sizeof(int) * ((size_t)nb / 1024 + 2))) || (e = mf_dmalloc(&ntok, sizeof(int))) ||
            (e = mf_dmalloc(&first_bad, sizeof(u64))))
            break;
        const u64 none = ~0ull;
        if ((e = cudaMemcpyAsync(first_bad, &none, sizeof(u64), cudaMemcpyHostToDevice, st)) ||
            (e = cudaMemsetAsync(ntok, 0, sizeof(int), st)))
            break;
        k_tok_count<<<nb, TOK_B, 0, st>>>(S, txt, bcount, first_bad);
        mf_exclusive_scan(nb, bcount, boff, tmp, st);
        int total = 0;
        if ((e = cudaMemcpyAsync(&total, boff + nb, sizeof(int), cudaMemcpyDeviceToHost, st)) ||
            (e = cudaStreamSynchronize(st)))
            break;
        if ((e = mf_dmalloc(&tok, sizeof(i64) * (size_t)std::max(total, 2)))) break;
        k_tok_values<<<nb, TOK_B, 0, st>>>(S, txt, boff, first_bad, tok, ntok);
        int K = 0;
        i64 hdr[2] = {0, 0};
        if ((e = cudaMemcpyAsync(&K, ntok, sizeof(int), cudaMemcpyDeviceToHost, st)) ||
            (e = cudaMemcpyAsync(hdr, tok, sizeof(hdr), cudaMemcpyDeviceToHost, st)) ||
            (e = cudaStreamSynchronize(st)))
            break;
        if (K < 2) {
            out.header_ok = false;
            break;
        }
        out.header_ok = true;
        out.n = (int)hdr[0];
        out.m_header = (int)hdr[1];
        i64 m = std::min<i64>(std::max<i64>(out.m_header, 0), (K - 2) / 3);
        out.m = m;
        const size_t M = (size_t)std::max<i64>(m, 1);
        if ((e = mf_dmalloc(&out.u, sizeof(int) * M)) || (e = mf_dmalloc(&out.v, sizeof(int) * M)) ||
            (e = mf_dmalloc(&out.c, sizeof(i64) * M)))
            break;
        if (m > 0) k_tok_edges<<<grid_of(m, 256), 256, 0, st>>>(m, tok, out.u, out.v, out.c);
        e = cudaStreamSynchronize(st);
        if (e == cudaSuccess) e = cudaGetLastError();
    } while (0);
    mf_dfree(bcount);
    mf_dfree(boff);
    mf_dfree(tmp);
    mf_dfree(ntok);
    mf_dfree(first_bad);
    mf_dfree(tok);
    if (e != cudaSuccess) mf_free_text_edges(out);
    return e;
}

void mf_free_text_edges(TextEdges &t) {
    mf_dfree(t.u);
    mf_dfree(t.v);
    mf_dfree(t.c);
    t.u = t.v = nullptr;
    t.c = nullptr;
}
