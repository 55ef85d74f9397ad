// Device-side region partitioning and region-ordered CSR reorder.
//
// Reference (Region_Aware_PR_with_Pruning_BoundaryCore.cu, "RA"):
//   per-vertex capacity/degree statistics ........ RA:2707-2720 (RA:1085-1088 at parse)
//   capacity-degree score + greedy least-loaded ... build_capacity_degree_partition_from_stats RA:1130-1178
//   region-contiguous renumbering + CSR scatter ... partition_and_reorder RA:1182-1260
//   region id per vertex .......................... build_region_id RA:1263-1276
// Differences by design: the score's logarithm is evaluated with a fixed
// operation sequence (mf_det_log) so host and device agree bit for bit, and
// equal scores are ordered by increasing vertex id (the reference's
// std::sort leaves their order unspecified).
#include <cstdio>
#include <cstring>
#include <vector>

#include "mf_build.cuh"

namespace {

// src[e] = row owning arc e (warp per vertex, coalesced stores).
__global__ void k_fill_src(int n, const int *__restrict__ row, int *__restrict__ src) {
    int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    int nw = (gridDim.x * blockDim.x) >> 5;
    for (int v = w; v < n; v += nw) {
        int b = row[v], e1 = row[v + 1];
        for (int e = b + lane; e < e1; e += 32) src[e] = v;
    }
}

// Statistics over arcs with cap > 0: four arcs per thread with 128-bit
// loads of src/col (int4) and cap (2 x longlong2); scalar tail.
__global__ void k_stats(i64 arcs, const int *__restrict__ src, const int *__restrict__ col,
                        const i64 *__restrict__ cap, i64 *so, i64 *si, int *dout, int *din) {
    i64 nvec = arcs >> 2;
    i64 stride = (i64)gridDim.x * blockDim.x;
    const int4 *src4 = reinterpret_cast<const int4 *>(src);
    const int4 *col4 = reinterpret_cast<const int4 *>(col);
    const longlong2 *cap2 = reinterpret_cast<const longlong2 *>(cap);
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < nvec; i += stride) {
        int4 s4 = __ldg(&src4[i]);
        int4 c4 = __ldg(&col4[i]);
        longlong2 a = __ldg(&cap2[2 * i]);
        longlong2 b = __ldg(&cap2[2 * i + 1]);
        int ss[4] = {s4.x, s4.y, s4.z, s4.w};
        int cc[4] = {c4.x, c4.y, c4.z, c4.w};
        i64 kk[4] = {a.x, a.y, b.x, b.y};
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (kk[j] > 0) {
                atomic_add_i64(&so[ss[j]], kk[j]);
                atomic_add_i64(&si[cc[j]], kk[j]);
                atomicAdd(&dout[ss[j]], 1);
                atomicAdd(&din[cc[j]], 1);
            }
    }
    for (i64 e = (nvec << 2) + (i64)blockIdx.x * blockDim.x + threadIdx.x; e < arcs; e += stride) {
        i64 k = cap[e];
        if (k > 0) {
            atomic_add_i64(&so[src[e]], k);
            atomic_add_i64(&si[col[e]], k);
            atomicAdd(&dout[src[e]], 1);
            atomicAdd(&din[col[e]], 1);
        }
    }
}

// Sort keys: descending score, then ascending id.  Positive doubles order
// like their bit patterns, so key = ~bits sorts descending.  Padding keys
// sort last.
__global__ void k_scores(int n, int P, const i64 *so, const i64 *si, const int *dout,
                         const int *din, u64 *key, int *id, double *score) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < P; v += gridDim.x * blockDim.x) {
        if (v < n) {
            double s = mf_score(so[v], si[v], dout[v], din[v]);
            score[v] = s;
            key[v] = ~(u64)__double_as_longlong(s);
            id[v] = v;
        } else {
            key[v] = ~0ull;
            id[v] = 0x7fffffff;
        }
    }
}

__device__ __forceinline__ bool kv_less(u64 ka, int ia, u64 kb, int ib) {
    return ka < kb || (ka == kb && ia < ib);
}

// One bitonic compare-exchange step over the whole array (global memory).
__global__ void k_bitonic_global(int P, int k, int j, u64 *key, int *id) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P; i += gridDim.x * blockDim.x) {
        int l = i ^ j;
        if (l > i) {
            u64 a = key[i], b = key[l];
            int ia = id[i], ib = id[l];
            bool up = (i & k) == 0;
            bool sw = up ? kv_less(b, ib, a, ia) : kv_less(a, ia, b, ib);
            if (sw) {
                key[i] = b;
                key[l] = a;
                id[i] = ib;
                id[l] = ia;
            }
        }
    }
}

// All steps with j < 1024 of stage k inside one 2048-element tile in shared
// memory (tile = blockIdx.x).
__global__ void k_bitonic_shared(int k, int jstart, u64 *key, int *id) {
    __shared__ u64 sk[2048];
    __shared__ int si_[2048];
    int base = blockIdx.x * 2048;
    for (int t = threadIdx.x; t < 2048; t += blockDim.x) {
        sk[t] = key[base + t];
        si_[t] = id[base + t];
    }
    __syncthreads();
    for (int j = jstart; j > 0; j >>= 1) {
        for (int t = threadIdx.x; t < 2048; t += blockDim.x) {
            int i = base + t;
            int l = i ^ j;
            if (l > i) {
                int tl = l - base;
                u64 a = sk[t], b = sk[tl];
                int ia = si_[t], ib = si_[tl];
                bool up = (i & k) == 0;
                bool sw = up ? kv_less(b, ib, a, ia) : kv_less(a, ia, b, ib);
                if (sw) {
                    sk[t] = b;
                    sk[tl] = a;
                    si_[t] = ib;
                    si_[tl] = ia;
                }
            }
        }
        __syncthreads();
    }
    for (int t = threadIdx.x; t < 2048; t += blockDim.x) {
        key[base + t] = sk[t];
        id[base + t] = si_[t];
    }
}

// Greedy least-loaded packing (RA:1168-1177): vertices in decreasing score
// order (the device sort's order) each go to the region with the least load,
// the lowest region on ties.  Every choice depends on all earlier ones, so
// the step is a single dependency chain; it runs on the host with a binary
// heap over (load, region), O(n log R), instead of serialising one GPU warp
// through n shuffle reductions.  Loads add in IEEE double round-to-nearest,
// exactly as the oracle does, so the packing is bit-identical.
static cudaError_t host_lpt(int n, int R, const u64 *d_key, const int *d_id, int *d_part, cudaStream_t st) {
    std::vector<u64> key((size_t)n);
    std::vector<int> id((size_t)n), part((size_t)n);
    cudaError_t e = cudaMemcpyAsync(key.data(), d_key, sizeof(u64) * (size_t)n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(id.data(), d_id, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    std::vector<double> load((size_t)R, 0.0);
    std::vector<int> heap((size_t)R);
    for (int r = 0; r < R; ++r) heap[r] = r;  // equal loads: index order is a heap
    auto less = [&](int x, int y) { return load[x] < load[y] || (load[x] == load[y] && x < y); };
    for (int i = 0; i < n; ++i) {
        const int r = heap[0];
        u64 bits = ~key[i];
        double w;
        memcpy(&w, &bits, sizeof w);
        part[id[i]] = r;
        load[r] = load[r] + w;
        // sift the grown root down
        int k = 0;
        for (;;) {
            int c = 2 * k + 1;
            if (c >= R) break;
            if (c + 1 < R && less(heap[c + 1], heap[c])) ++c;
            if (!less(heap[c], heap[k])) break;
            int tmp = heap[c];
            heap[c] = heap[k];
            heap[k] = tmp;
            k = c;
        }
    }
    e = cudaMemcpyAsync(d_part, part.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e;
}

#define CHUNK 4096
#define CHUNK_WARPS 16

// Per-chunk region counts (chunk = CHUNK consecutive old ids).
__global__ void k_chunk_counts(int n, int R, const int *part, int *ccount) {
    extern __shared__ int sc[];
    for (int r = threadIdx.x; r < R; r += blockDim.x) sc[r] = 0;
    __syncthreads();
    int base = blockIdx.x * CHUNK;
    for (int t = threadIdx.x; t < CHUNK; t += blockDim.x) {
        int v = base + t;
        if (v < n) {
            int r = part[v];
            if (r < 0 || r >= R) r = 0;
            atomicAdd(&sc[r], 1);
        }
    }
    __syncthreads();
    for (int r = threadIdx.x; r < R; r += blockDim.x) ccount[(size_t)blockIdx.x * R + r] = sc[r];
}

// region_start (R+1) and per-(chunk, region) offsets, one thread per region.
__global__ void k_chunk_offsets(int R, int nchunks, const int *ccount, int *coff, int *region_start) {
    // serial over regions for region_start (R <= 1024): thread 0
    __shared__ int rs[1025];
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int r = 0; r < R; ++r) {
            rs[r] = acc;
            int tot = 0;
            for (int c = 0; c < nchunks; ++c) tot += ccount[(size_t)c * R + r];
            acc += tot;
        }
        rs[R] = acc;
        for (int r = 0; r <= R; ++r) region_start[r] = rs[r];
    }
    __syncthreads();
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        int acc = rs[r];
        for (int c = 0; c < nchunks; ++c) {
            coff[(size_t)c * R + r] = acc;
            acc += ccount[(size_t)c * R + r];
        }
    }
}

// Stable placement inside a chunk: warp w handles CHUNK/CHUNK_WARPS
// consecutive ids in 32-wide steps; __match_any_sync groups equal regions,
// ranks come from popc of the peer mask; per-warp region totals are prefix
// summed across warps in shared memory.
__global__ void k_chunk_place(int n, int R, const int *part, const int *coff, int *new_id,
                              int *old_id) {
    extern __shared__ int sm[];
    int *wcnt = sm;                    // [CHUNK_WARPS][R]
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < CHUNK_WARPS * R; i += blockDim.x) wcnt[i] = 0;
    __syncthreads();
    const int per = CHUNK / CHUNK_WARPS;
    int base = blockIdx.x * CHUNK + warp * per;
    for (int step = 0; step < per; step += 32) {
        int v = base + step + lane;
        int r = (v < n) ? part[v] : -1;
        if (r >= R) r = 0;
        if (v < n && r < 0) r = 0;
        unsigned peers = __match_any_sync(MF_FULL, r);
        if (r >= 0 && (peers & lanemask_lt()) == 0) wcnt[warp * R + r] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // exclusive prefix over warps per region
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        int acc = 0;
        for (int w = 0; w < CHUNK_WARPS; ++w) {
            int c = wcnt[w * R + r];
            wcnt[w * R + r] = acc;
            acc += c;
        }
    }
    __syncthreads();
    const int *off = coff + (size_t)blockIdx.x * R;
    for (int step = 0; step < per; step += 32) {
        int v = base + step + lane;
        int r = (v < n) ? part[v] : -1;
        if (r >= R) r = 0;
        if (v < n && r < 0) r = 0;
        unsigned peers = __match_any_sync(MF_FULL, r);
        if (r >= 0) {
            int pos = off[r] + wcnt[warp * R + r] + __popc(peers & lanemask_lt());
            new_id[v] = pos;
            old_id[pos] = v;
        }
        __syncwarp();
        if (r >= 0 && (peers & lanemask_lt()) == 0) wcnt[warp * R + r] += __popc(peers);
        __syncwarp();
    }
}

__global__ void k_new_degrees(int n, const int *row0, const int *new_id, int *deg) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        deg[new_id[v]] = row0[v + 1] - row0[v];
}

// Exclusive scan helpers (n+1 outputs: out[0] = 0, out[i+1] = sum in[0..i]).
#define SCAN_B 1024
__global__ void k_scan_blocks(int n, const int *in, int *out, int *bsum) {
    __shared__ int s[SCAN_B];
    int i = blockIdx.x * SCAN_B + threadIdx.x;
    int x = (i < n) ? in[i] : 0;
    s[threadIdx.x] = x;
    __syncthreads();
    for (int o = 1; o < SCAN_B; o <<= 1) {
        int y = (threadIdx.x >= o) ? s[threadIdx.x - o] : 0;
        __syncthreads();
        s[threadIdx.x] += y;
        __syncthreads();
    }
    if (i < n) out[i + 1] = s[threadIdx.x];
    if (threadIdx.x == SCAN_B - 1) bsum[blockIdx.x] = s[threadIdx.x];
}
__global__ void k_scan_sums(int nb, int *bsum) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        int acc = 0;
        for (int b = 0; b < nb; ++b) {
            int x = bsum[b];
            bsum[b] = acc;
            acc += x;
        }
    }
}
__global__ void k_scan_add(int n, int *out, const int *bsum) {
    int i = blockIdx.x * SCAN_B + threadIdx.x;
    if (i < n) out[i + 1] += bsum[blockIdx.x];
    if (i == 0) out[0] = 0;
}

// Arc scatter into region order: four arcs per thread with 128-bit loads of
// src/col/isfwd-free fields; e2n records each arc's new position.
__global__ void k_scatter_arcs(i64 arcs, const int *__restrict__ src, const int *__restrict__ row0,
                               const int *__restrict__ col0, const i64 *__restrict__ cap0,
                               const unsigned char *__restrict__ fwd0, const int *__restrict__ new_id,
                               const int *__restrict__ row, int *__restrict__ col,
                               i64 *__restrict__ cap, unsigned char *__restrict__ fwd,
                               int *__restrict__ e2n) {
    i64 nvec = arcs >> 2;
    i64 stride = (i64)gridDim.x * blockDim.x;
    const int4 *src4 = reinterpret_cast<const int4 *>(src);
    const int4 *col4 = reinterpret_cast<const int4 *>(col0);
    const longlong2 *cap2 = reinterpret_cast<const longlong2 *>(cap0);
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < nvec; i += stride) {
        int4 s4 = __ldg(&src4[i]);
        int4 c4 = __ldg(&col4[i]);
        longlong2 a = __ldg(&cap2[2 * i]);
        longlong2 b = __ldg(&cap2[2 * i + 1]);
        int ss[4] = {s4.x, s4.y, s4.z, s4.w};
        int cc[4] = {c4.x, c4.y, c4.z, c4.w};
        i64 kk[4] = {a.x, a.y, b.x, b.y};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            i64 e = 4 * i + j;
            int u = ss[j];
            int pos = __ldg(&row[__ldg(&new_id[u])]) + (int)(e - __ldg(&row0[u]));
            col[pos] = __ldg(&new_id[cc[j]]);
            cap[pos] = kk[j];
            fwd[pos] = fwd0[e];
            e2n[e] = pos;
        }
    }
    for (i64 e = (nvec << 2) + (i64)blockIdx.x * blockDim.x + threadIdx.x; e < arcs; e += stride) {
        int u = src[e];
        int pos = row[new_id[u]] + (int)(e - row0[u]);
        col[pos] = new_id[col0[e]];
        cap[pos] = cap0[e];
        fwd[pos] = fwd0[e];
        e2n[e] = pos;
    }
}

__global__ void k_scatter_rev(i64 arcs, const int *rev0, const int *e2n, int *rev) {
    for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < arcs;
         e += (i64)gridDim.x * blockDim.x)
        rev[e2n[e]] = e2n[rev0[e]];
}

__global__ void k_region_of(int R, const int *region_start, int *region_of) {
    int r = blockIdx.x;
    if (r >= R) return;
    for (int p = region_start[r] + threadIdx.x; p < region_start[r + 1]; p += blockDim.x)
        region_of[p] = r;
}

int grid_for(i64 work, int threads) {
    i64 b = (work + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 32) b = 148 * 32;
    return (int)b;
}

}  // namespace

// Exclusive scan of n ints into out[0..n] on stream st (tmp: >= n/1024+1 ints).
void mf_exclusive_scan(int n, const int *in, int *out, int *tmp, cudaStream_t st) {
    int nb = (n + SCAN_B - 1) / SCAN_B;
    if (nb < 1) nb = 1;
    k_scan_blocks<<<nb, SCAN_B, 0, st>>>(n, in, out, tmp);
    k_scan_sums<<<1, 32, 0, st>>>(nb, tmp);
    k_scan_add<<<nb, SCAN_B, 0, st>>>(n, out, tmp);
}

size_t mf_partition_scratch_bytes(int n, i64 arcs, int R) {
    int P = 2048;
    while (P < n) P <<= 1;
    int nchunks = (n + CHUNK - 1) / CHUNK;
    size_t b = 0;
    b += sizeof(int) * (size_t)arcs;             // src
    b += sizeof(int) * (size_t)arcs;             // e2n
    b += 2 * sizeof(i64) * (size_t)n;            // so, si
    b += 2 * sizeof(int) * (size_t)n;            // dout, din
    b += sizeof(u64) * (size_t)P + sizeof(int) * (size_t)P;  // keys, ids
    b += 2 * sizeof(int) * (size_t)nchunks * R;  // ccount, coff
    b += sizeof(int) * ((size_t)n + 2);          // deg
    b += sizeof(int) * ((size_t)n / SCAN_B + 2); // scan tmp
    return b + 64 * 16;
}

// Partition + reorder (see file header).  in: CSR in any vertex order;
// out: region-ordered CSR.  All device pointers; scratch from
// mf_partition_scratch_bytes.  Returns a cudaError_t.
cudaError_t mf_partition_reorder(const BuildIn &in, const BuildOut &out, void *scratch,
                                 cudaStream_t st) {
    const int n = in.n, R = in.R;
    const i64 arcs = in.arcs;
    int P = 2048;
    while (P < n) P <<= 1;
    int nchunks = (n + CHUNK - 1) / CHUNK;
    char *p = (char *)scratch;
    auto take = [&](size_t bytes) {
        char *r = p;
        p += (bytes + 255) & ~(size_t)255;
        return (void *)r;
    };
    int *src = (int *)take(sizeof(int) * (size_t)(arcs > 0 ? arcs : 1));
    int *e2n = (int *)take(sizeof(int) * (size_t)(arcs > 0 ? arcs : 1));
    i64 *so = (i64 *)take(sizeof(i64) * n);
    i64 *si = (i64 *)take(sizeof(i64) * n);
    int *dout = (int *)take(sizeof(int) * n);
    int *din = (int *)take(sizeof(int) * n);
    u64 *key = (u64 *)take(sizeof(u64) * P);
    int *id = (int *)take(sizeof(int) * P);
    int *ccount = (int *)take(sizeof(int) * (size_t)nchunks * R);
    int *coff = (int *)take(sizeof(int) * (size_t)nchunks * R);
    int *deg = (int *)take(sizeof(int) * ((size_t)n + 2));
    int *stmp = (int *)take(sizeof(int) * ((size_t)n / SCAN_B + 2));

    cudaMemsetAsync(so, 0, sizeof(i64) * n, st);
    cudaMemsetAsync(si, 0, sizeof(i64) * n, st);
    cudaMemsetAsync(dout, 0, sizeof(int) * n, st);
    cudaMemsetAsync(din, 0, sizeof(int) * n, st);
    k_fill_src<<<grid_for((i64)n * 32, 256), 256, 0, st>>>(n, in.row, src);
    k_stats<<<grid_for(arcs / 4 + 1, 256), 256, 0, st>>>(arcs, src, in.col, in.cap, so, si, dout, din);
    k_scores<<<grid_for(P, 256), 256, 0, st>>>(n, P, so, si, dout, din, key, id, out.score);
    for (int k = 2; k <= P; k <<= 1) {
        int j = k >> 1;
        for (; j >= 1024; j >>= 1) k_bitonic_global<<<grid_for(P, 256), 256, 0, st>>>(P, k, j, key, id);
        k_bitonic_shared<<<P / 2048, 1024, 0, st>>>(k, j, key, id);
    }
    {
        cudaError_t e = host_lpt(n, R, key, id, out.part, st);
        if (e != cudaSuccess) return e;
    }
    cudaFuncSetAttribute(k_chunk_place, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(sizeof(int) * CHUNK_WARPS * 1024));
    k_chunk_counts<<<nchunks, 512, sizeof(int) * R, st>>>(n, R, out.part, ccount);
    k_chunk_offsets<<<1, 256, 0, st>>>(R, nchunks, ccount, coff, out.region_start);
    k_chunk_place<<<nchunks, 32 * CHUNK_WARPS, sizeof(int) * CHUNK_WARPS * R, st>>>(
        n, R, out.part, coff, out.new_id, out.old_id);
    k_new_degrees<<<grid_for(n, 256), 256, 0, st>>>(n, in.row, out.new_id, deg);
    mf_exclusive_scan(n, deg, out.row, stmp, st);
    k_scatter_arcs<<<grid_for(arcs / 4 + 1, 256), 256, 0, st>>>(
        arcs, src, in.row, in.col, in.cap, in.fwd, out.new_id, out.row, out.col, out.cap, out.fwd, e2n);
    k_scatter_rev<<<grid_for(arcs, 256), 256, 0, st>>>(arcs, in.rev, e2n, out.rev);
    k_region_of<<<R, 256, 0, st>>>(R, out.region_start, out.region_of);
    return cudaGetLastError();
}
