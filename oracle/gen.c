/*
 * Synthetic workload generators and graph.txt / test.txt writers for the
 * checker side — TEST INFRASTRUCTURE ONLY (built into oracle/liboracle.so).
 *
 * bench.py's reference arm writes the reference program's inputs with these,
 * so that the process timing the reference never loads the engine's library.
 * They restate the engine's own seeded generators (mf_gen_rmat,
 * mf_gen_queries_hub, mf_write_graph_txt, mf_write_test_txt in
 * mscresearch_b200/csrc/mf_host.cpp) output for output: the same
 * splitmix64 seeding, xoshiro256** stream, 65536-edge chunks with one
 * stream per chunk, draw order and byte format.  tests/test_oracle.py checks
 * that both produce identical arrays and identical files.
 *
 * The R-MAT recursion (quadrant probabilities a, b, c, d per level) and the
 * query mix (half between top-1% out-degree and top-1% in-degree vertices,
 * half uniform) are the workload the benchmark measures; the reference
 * itself ships no generator.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

typedef long long i64;

/* splitmix64 (seeding) and xoshiro256** (stream): public-domain generators
 * by Vigna and Blackman. */
static uint64_t gn_splitmix(uint64_t *x) {
    uint64_t z = (*x += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

typedef struct {
    uint64_t s[4];
} gn_rng;

static void gn_seed(gn_rng *r, uint64_t seed) {
    uint64_t x = seed;
    for (int i = 0; i < 4; ++i) r->s[i] = gn_splitmix(&x);
}

static uint64_t gn_rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }

static uint64_t gn_next(gn_rng *r) {
    uint64_t *s = r->s;
    const uint64_t out = gn_rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = gn_rotl(s[3], 45);
    return out;
}

/* uniform in [0, k) by a 64x64 -> 128-bit multiply-shift */
static uint64_t gn_below(gn_rng *r, uint64_t k) {
    return (uint64_t)(((unsigned __int128)gn_next(r) * k) >> 64);
}

/* uniform double in [0, 1) with 53 random bits */
static double gn_unit(gn_rng *r) { return (double)(gn_next(r) >> 11) * (1.0 / 9007199254740992.0); }

static uint64_t gn_chunk_seed(uint64_t seed, uint64_t chunk) {
    uint64_t x = seed ^ (0xd1b54a32d192ed03ull * (chunk + 1));
    return gn_splitmix(&x);
}

#define GN_CHUNK 65536LL

typedef struct {
    int scale;
    i64 m;
    double a, ab, abc;
    i64 lo, hi;
    uint64_t seed;
    int *u, *v;
    i64 *cap;
    unsigned char *self;
    int worker, workers;
} gn_rmat_job;

static void *gn_rmat_worker(void *p) {
    gn_rmat_job *j = (gn_rmat_job *)p;
    const i64 nch = (j->m + GN_CHUNK - 1) / GN_CHUNK;
    for (i64 ch = j->worker; ch < nch; ch += j->workers) {
        gn_rng r;
        gn_seed(&r, gn_chunk_seed(j->seed, (uint64_t)ch));
        const i64 e0 = ch * GN_CHUNK, e1 = e0 + GN_CHUNK < j->m ? e0 + GN_CHUNK : j->m;
        for (i64 i = e0; i < e1; ++i) {
            uint32_t x = 0, y = 0;
            for (int l = 0; l < j->scale; ++l) {
                const double p = gn_unit(&r);
                uint32_t bx = 0, by = 0;
                if (p < j->a) {
                } else if (p < j->ab) {
                    by = 1;
                } else if (p < j->abc) {
                    bx = 1;
                } else {
                    bx = 1;
                    by = 1;
                }
                x = (x << 1) | bx;
                y = (y << 1) | by;
            }
            j->u[i] = (int)x;
            j->v[i] = (int)y;
            j->cap[i] = j->lo + (i64)gn_below(&r, (uint64_t)(j->hi - j->lo + 1));
            j->self[i] = (x == y);
        }
    }
    return NULL;
}

/* R-MAT with n = 2^scale and m draws; self loops dropped (the kept count is
 * returned; the arrays hold m entries).  Returns -1 on bad arguments. */
i64 gn_rmat(int scale, i64 m, double a, double b, double c, i64 lo, i64 hi, uint64_t seed, int *u, int *v,
            i64 *cap) {
    if (scale < 1 || scale > 30 || m < 0 || lo > hi || !u || !v || !cap) return -1;
    unsigned char *self = (unsigned char *)calloc((size_t)(m > 0 ? m : 1), 1);
    if (!self) return -1;
    long hw = sysconf(_SC_NPROCESSORS_ONLN);
    int T = hw > 0 ? (int)hw : 1;
    if (T > 64) T = 64;
    gn_rmat_job jobs[64];
    pthread_t th[64];
    for (int w = 0; w < T; ++w) {
        gn_rmat_job jb = {scale, m, a, a + b, a + b + c, lo, hi, seed, u, v, cap, self, w, T};
        jobs[w] = jb;
        pthread_create(&th[w], NULL, gn_rmat_worker, &jobs[w]);
    }
    for (int w = 0; w < T; ++w) pthread_join(th[w], NULL);
    i64 k = 0;
    for (i64 i = 0; i < m; ++i) {
        if (self[i]) continue;
        u[k] = u[i];
        v[k] = v[i];
        cap[k] = cap[i];
        ++k;
    }
    free(self);
    return k;
}

static const i64 *gn_key;
/* larger key first, then smaller id (a total order) */
static int gn_desc_cmp(const void *pa, const void *pb) {
    const int a = *(const int *)pa, b = *(const int *)pb;
    if (gn_key[a] != gn_key[b]) return gn_key[a] > gn_key[b] ? -1 : 1;
    return (a > b) - (a < b);
}

/* nhub pairs with s among the top 1% of vertices by out-degree and t among
 * the top 1% by in-degree (ties by id), then nuni uniform pairs; s != t.
 * Returns 0, or -1 on bad arguments. */
int gn_queries_hub(int n, i64 m, const int *u, const int *v, int nhub, int nuni, uint64_t seed, int *s,
                   int *t) {
    if (n < 2 || nhub < 0 || nuni < 0 || !s || !t) return -1;
    i64 *dout = (i64 *)calloc((size_t)n, sizeof(i64));
    i64 *din = (i64 *)calloc((size_t)n, sizeof(i64));
    int *tout = (int *)malloc(sizeof(int) * (size_t)n);
    int *tin = (int *)malloc(sizeof(int) * (size_t)n);
    if (!dout || !din || !tout || !tin) {
        free(dout);
        free(din);
        free(tout);
        free(tin);
        return -1;
    }
    for (i64 i = 0; i < m; ++i) {
        if (u[i] < 0 || u[i] >= n || v[i] < 0 || v[i] >= n || u[i] == v[i]) continue;
        dout[u[i]]++;
        din[v[i]]++;
    }
    for (int i = 0; i < n; ++i) tout[i] = tin[i] = i;
    gn_key = dout;
    qsort(tout, (size_t)n, sizeof(int), gn_desc_cmp);
    gn_key = din;
    qsort(tin, (size_t)n, sizeof(int), gn_desc_cmp);
    const int top = n / 100 > 1 ? n / 100 : 1;
    gn_rng r;
    gn_seed(&r, seed ^ 0x5bd1e995ull);
    for (int i = 0; i < nhub; ++i) {
        int a = tout[gn_below(&r, (uint64_t)top)], b = tin[gn_below(&r, (uint64_t)top)];
        for (int tries = 0; a == b && tries < 64; ++tries) b = tin[gn_below(&r, (uint64_t)top)];
        if (a == b) b = (a + 1) % n;
        s[i] = a;
        t[i] = b;
    }
    for (int i = nhub; i < nhub + nuni; ++i) {
        int a = (int)gn_below(&r, (uint64_t)n), b = (int)gn_below(&r, (uint64_t)n);
        while (b == a) b = (int)gn_below(&r, (uint64_t)n);
        s[i] = a;
        t[i] = b;
    }
    free(dout);
    free(din);
    free(tout);
    free(tin);
    return 0;
}

/* graph.txt: "n m" then one "u v cap" line per edge, 1-based ids. */
int gn_write_graph_txt(const char *path, int n, i64 m, const int *u, const int *v, const i64 *cap) {
    FILE *f = fopen(path, "wb");
    if (!f) return -1;
    static char buf[1 << 20];
    setvbuf(f, buf, _IOFBF, sizeof buf);
    fprintf(f, "%d %lld\n", n, m);
    for (i64 i = 0; i < m; ++i) fprintf(f, "%lld %lld %lld\n", (i64)u[i] + 1, (i64)v[i] + 1, cap[i]);
    return fclose(f) == 0 ? 0 : -1;
}

/* test.txt: one "s t" line per query, 1-based ids. */
int gn_write_test_txt(const char *path, int nq, const int *s, const int *t) {
    FILE *f = fopen(path, "wb");
    if (!f) return -1;
    for (int i = 0; i < nq; ++i) fprintf(f, "%d %d\n", s[i] + 1, t[i] + 1);
    return fclose(f) == 0 ? 0 : -1;
}
