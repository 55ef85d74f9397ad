// Host-side utilities of the C ABI: seeded synthetic workloads, graph.txt /
// test.txt reading and writing.
//
// Reader semantics follow the reference's build_graph and query loop
// (Region_Aware_PR_with_Pruning_BoundaryCore.cu:1051-1075, 2609-2621): an
// "n m" header, then up to m "u v cap" triples read as a token stream (as
// fscanf would), stopping at the first triple that does not scan.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/maxflow_b200.h"

namespace {

// splitmix64 (seeding) and xoshiro256** (stream), both public-domain
// generators by Vigna / Blackman.
inline uint64_t splitmix64(uint64_t &x) {
    uint64_t z = (x += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        uint64_t x = seed;
        for (int i = 0; i < 4; ++i) s[i] = splitmix64(x);
    }
    static inline uint64_t rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }
    inline uint64_t next() {
        uint64_t r = rotl(s[1] * 5, 7) * 9;
        uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    // uniform in [0, k) by multiply-shift
    inline uint64_t below(uint64_t k) { return (uint64_t)(((unsigned __int128)next() * k) >> 64); }
    inline double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

uint64_t chunk_seed(uint64_t seed, uint64_t chunk) {
    uint64_t x = seed ^ (0xd1b54a32d192ed03ull * (chunk + 1));
    return splitmix64(x);
}

template <class F>
void parallel_chunks(long long nchunks, F f) {
    unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    int T = (int)std::min<long long>(hw, std::max<long long>(1, nchunks));
    std::vector<std::thread> th;
    for (int w = 0; w < T; ++w)
        th.emplace_back([&, w]() {
            for (long long c = w; c < nchunks; c += T) f(c);
        });
    for (auto &x : th) x.join();
}

const long long CH = 1 << 16;

}  // namespace

extern "C" {

int mf_gen_uniform(int n, long long m, long long lo, long long hi, unsigned long long seed,
                   int32_t *u, int32_t *v, int64_t *cap) {
    if (n < 2 || m < 0 || lo > hi || !u || !v || !cap) return MF_ERR_ARG;
    long long nch = (m + CH - 1) / CH;
    parallel_chunks(nch, [&](long long c) {
        Rng r(chunk_seed(seed, (uint64_t)c));
        long long e0 = c * CH, e1 = std::min(m, e0 + CH);
        for (long long i = e0; i < e1; ++i) {
            int a = (int)r.below((uint64_t)n);
            int b = (int)r.below((uint64_t)n);
            while (b == a) b = (int)r.below((uint64_t)n);
            u[i] = a;
            v[i] = b;
            cap[i] = lo + (long long)r.below((uint64_t)(hi - lo + 1));
        }
    });
    return MF_OK;
}

int mf_gen_rmat(int scale, long long m, double a, double b, double c, long long lo, long long hi,
                unsigned long long seed, int32_t *u, int32_t *v, int64_t *cap, long long *kept) {
    if (scale < 1 || scale > 30 || m < 0 || lo > hi || !u || !v || !cap) return MF_ERR_ARG;
    const double ab = a + b, abc = a + b + c;
    long long nch = (m + CH - 1) / CH;
    std::vector<unsigned char> self(m > 0 ? m : 1, 0);
    parallel_chunks(nch, [&](long long ch) {
        Rng r(chunk_seed(seed, (uint64_t)ch));
        long long e0 = ch * CH, e1 = std::min(m, e0 + CH);
        for (long long i = e0; i < e1; ++i) {
            uint32_t x = 0, y = 0;
            for (int l = 0; l < scale; ++l) {
                double p = r.unit();
                uint32_t bx = 0, by = 0;
                if (p < a) {
                } else if (p < ab) {
                    by = 1;
                } else if (p < abc) {
                    bx = 1;
                } else {
                    bx = 1;
                    by = 1;
                }
                x = (x << 1) | bx;
                y = (y << 1) | by;
            }
            u[i] = (int32_t)x;
            v[i] = (int32_t)y;
            cap[i] = lo + (long long)r.below((uint64_t)(hi - lo + 1));
            self[i] = (x == y);
        }
    });
    long long k = 0;
    for (long long i = 0; i < m; ++i) {
        if (self[i]) continue;
        u[k] = u[i];
        v[k] = v[i];
        cap[k] = cap[i];
        ++k;
    }
    if (kept) *kept = k;
    return MF_OK;
}

int mf_gen_grid(int W, int H, unsigned long long seed, int32_t *u, int32_t *v, int64_t *cap,
                long long *m) {
    if (W < 1 || H < 1 || !u || !v || !cap) return MF_ERR_ARG;
    const int S = W * H, T = W * H + 1;
    // per row: 4 neighbour slots + 1 terminal slot per pixel, compacted after
    const long long per_row = 5LL * W;
    std::vector<unsigned char> used((size_t)per_row * H, 0);
    parallel_chunks(H, [&](long long y) {
        Rng r(chunk_seed(seed, (uint64_t)y));
        long long base = y * per_row;
        for (int x = 0; x < W; ++x) {
            int p = (int)y * W + x;
            const int dx[4] = {1, -1, 0, 0}, dy[4] = {0, 0, 1, -1};
            for (int k = 0; k < 4; ++k) {
                long long slot = base + 5LL * x + k;
                int nx = x + dx[k], ny = (int)y + dy[k];
                // d ~ N(0, 40) by Box-Muller
                double u1 = r.unit(), u2 = r.unit();
                if (u1 < 1e-300) u1 = 1e-300;
                double d = 40.0 * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
                if (nx < 0 || nx >= W || ny < 0 || ny >= H) continue;
                u[slot] = p;
                v[slot] = ny * W + nx;
                cap[slot] = 1 + (long long)std::floor(255.0 * std::exp(-d * d / 50.0));
                used[slot] = 1;
            }
            long long slot = base + 5LL * x + 4;
            bool to_src = (r.next() >> 63) != 0;
            long long c = (long long)r.below(256);
            if (to_src) {
                u[slot] = S;
                v[slot] = p;
            } else {
                u[slot] = p;
                v[slot] = T;
            }
            cap[slot] = c;
            used[slot] = 1;
        }
    });
    long long k = 0, tot = per_row * H;
    for (long long i = 0; i < tot; ++i) {
        if (!used[i]) continue;
        u[k] = u[i];
        v[k] = v[i];
        cap[k] = cap[i];
        ++k;
    }
    if (m) *m = k;
    return MF_OK;
}

int mf_gen_queries_hub(int n, long long m, const int32_t *u, const int32_t *v, int nhub, int nuni,
                       unsigned long long seed, int32_t *s, int32_t *t) {
    if (n < 2 || nhub < 0 || nuni < 0 || !s || !t) return MF_ERR_ARG;
    std::vector<long long> dout(n, 0), din(n, 0);
    for (long long i = 0; i < m; ++i) {
        if (u[i] < 0 || u[i] >= n || v[i] < 0 || v[i] >= n || u[i] == v[i]) continue;
        dout[u[i]]++;
        din[v[i]]++;
    }
    int top = std::max(1, n / 100);
    std::vector<int> ord(n);
    for (int i = 0; i < n; ++i) ord[i] = i;
    std::vector<int> tout(ord), tin(ord);
    std::partial_sort(tout.begin(), tout.begin() + top, tout.end(), [&](int a, int b) {
        return dout[a] != dout[b] ? dout[a] > dout[b] : a < b;
    });
    std::partial_sort(tin.begin(), tin.begin() + top, tin.end(), [&](int a, int b) {
        return din[a] != din[b] ? din[a] > din[b] : a < b;
    });
    Rng r(seed ^ 0x5bd1e995ull);
    for (int i = 0; i < nhub; ++i) {
        int a = tout[r.below(top)], b = tin[r.below(top)];
        for (int tries = 0; a == b && tries < 64; ++tries) b = tin[r.below(top)];
        if (a == b) b = (a + 1) % n;
        s[i] = a;
        t[i] = b;
    }
    for (int i = nhub; i < nhub + nuni; ++i) {
        int a = (int)r.below(n), b = (int)r.below(n);
        while (b == a) b = (int)r.below(n);
        s[i] = a;
        t[i] = b;
    }
    return MF_OK;
}

// ---- text I/O ---------------------------------------------------------------

static char *fmt_i64(char *p, long long x) {
    char tmp[24];
    int k = 0;
    bool neg = x < 0;
    unsigned long long ux = neg ? (unsigned long long)(-(x + 1)) + 1 : (unsigned long long)x;
    do {
        tmp[k++] = (char)('0' + ux % 10);
        ux /= 10;
    } while (ux);
    if (neg) *p++ = '-';
    while (k) *p++ = tmp[--k];
    return p;
}

int mf_write_graph_txt(const char *path, int n, long long m, const int32_t *u, const int32_t *v,
                       const int64_t *cap) {
    FILE *f = fopen(path, "wb");
    if (!f) return MF_ERR_IO;
    fprintf(f, "%d %lld\n", n, m);
    std::vector<char> buf(1 << 22);
    size_t pos = 0;
    for (long long i = 0; i < m; ++i) {
        if (pos + 80 > buf.size()) {
            fwrite(buf.data(), 1, pos, f);
            pos = 0;
        }
        char *p = buf.data() + pos;
        p = fmt_i64(p, (long long)u[i] + 1);
        *p++ = ' ';
        p = fmt_i64(p, (long long)v[i] + 1);
        *p++ = ' ';
        p = fmt_i64(p, cap[i]);
        *p++ = '\n';
        pos = p - buf.data();
    }
    fwrite(buf.data(), 1, pos, f);
    return fclose(f) == 0 ? MF_OK : MF_ERR_IO;
}

int mf_write_test_txt(const char *path, int nq, const int32_t *s, const int32_t *t) {
    FILE *f = fopen(path, "wb");
    if (!f) return MF_ERR_IO;
    for (int i = 0; i < nq; ++i) fprintf(f, "%d %d\n", s[i] + 1, t[i] + 1);
    return fclose(f) == 0 ? MF_OK : MF_ERR_IO;
}

namespace {
struct Scanner {
    const char *p, *e;
    // fscanf-style integer: skip white space, optional sign, >= 1 digit.
    bool next(long long &out) {
        while (p < e && isspace((unsigned char)*p)) ++p;
        if (p >= e) return false;
        const char *q = p;
        bool neg = false;
        if (*q == '+' || *q == '-') {
            neg = (*q == '-');
            ++q;
        }
        if (q >= e || !isdigit((unsigned char)*q)) return false;
        // magnitude saturates at the limit of its sign, as strtoll does
        const unsigned long long lim = neg ? (1ull << 63) : (1ull << 63) - 1ull;
        unsigned long long x = 0;
        bool over = false;
        while (q < e && isdigit((unsigned char)*q)) {
            const unsigned long long d = (unsigned)(*q - '0');
            if (x > (lim - d) / 10ull) over = true;
            else x = x * 10ull + d;
            ++q;
        }
        if (over) x = lim;
        p = q;
        out = (long long)(neg ? (~x + 1ull) : x);
        return true;
    }
};

bool slurp(const char *path, std::vector<char> &data) {
    FILE *f = fopen(path, "rb");
    if (!f) return false;
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    data.resize(sz > 0 ? (size_t)sz : 0);
    size_t got = sz > 0 ? fread(data.data(), 1, (size_t)sz, f) : 0;
    fclose(f);
    data.resize(got);
    return true;
}
}  // namespace

int mf_graph_txt_header(const char *path, int *n, long long *m) {
    FILE *f = fopen(path, "r");
    if (!f) return MF_ERR_IO;
    int a, b;
    int ok = fscanf(f, "%d %d", &a, &b);
    fclose(f);
    if (ok != 2) return MF_ERR_IO;
    if (n) *n = a;
    if (m) *m = b;
    return MF_OK;
}

int mf_read_graph_txt(const char *path, int *n, long long *m_read, int32_t *u, int32_t *v,
                      int64_t *cap, long long cap_len) {
    std::vector<char> data;
    if (!slurp(path, data)) return MF_ERR_IO;
    Scanner sc{data.data(), data.data() + data.size()};
    long long a, b;
    if (!sc.next(a) || !sc.next(b)) return MF_ERR_IO;
    if (n) *n = (int)a;
    long long m = b, k = 0;
    for (long long i = 0; i < m && k < cap_len; ++i) {
        long long x, y, c;
        if (!sc.next(x) || !sc.next(y) || !sc.next(c)) break;
        u[k] = (int32_t)((uint32_t)x - 1u);
        v[k] = (int32_t)((uint32_t)y - 1u);
        cap[k] = c;
        ++k;
    }
    if (m_read) *m_read = k;
    return MF_OK;
}


}  // extern "C"
