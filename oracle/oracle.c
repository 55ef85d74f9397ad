/*
 * CPU oracle for the exact max-flow hot path — TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker, never the product: only tests/, the smoke check
 * in __graft_entry__.py and the cpu_baseline leg of bench.py load it.  The
 * engine under mscresearch_b200/ never links, loads or calls it.
 *
 * It restates, in plain C, the reference's host-side semantics for the path
 * (file:line cites are into the reference project,
 * Region_Aware_PR_with_Pruning_BoundaryCore.cu, abbreviated RA):
 *   - graph.txt parsing and filtering .......... RA:1051-1075
 *   - paired-arc CSR construction (rev) ........ RA:1078-1122
 *   - per-vertex capacity/degree statistics .... RA:2707-2720 (and RA:1085-1088)
 *   - capacity-degree score + greedy packing ... RA:1130-1178
 *   - region-contiguous reorder ................ RA:1182-1260
 *   - query reachability prune mask ............ RA:1391-1445
 *   - induced subgraph by mask ................. RA:2477-2551
 *   - boundary-aware core mask ................. RA:2340-2475 (restated only to
 *     show it is not flow preserving; the engine does not apply it)
 * and provides two independent exact max-flow solvers on the same CSR:
 *   - Dinic (BFS levels + blocking flow with current-arc pointers), and
 *   - a sequential FIFO push-relabel with exact global relabeling, which is
 *     the sequential form of the reference's algorithm (RA:432-515 discharge,
 *     RA:203-348 BFS relabel from the sink).
 * plus a certifier (feasibility, conservation, equal-capacity s-t cut).
 *
 * Parity anchor: the reference ships no tests or golden vectors.  The oracle
 * is pinned against outputs of the reference's own CUDA build run on a B200
 * (tests/golden/, generated by tests/golden/make_golden.py + oracle/build_ref.sh).
 *
 * Flows, capacities and excesses are int64 throughout (RA:18).
 *
 * Compile with -ffp-contract=off: or_score must round exactly like the
 * engine's device score (see det_log below).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef long long i64;

/* ------------------------------------------------------------------------ */
/* graph.txt parsing (RA:1051-1075).  Reads the "n m" header and then up to m
 * "u v cap" lines, stopping at the first line that does not scan as three
 * numbers.  Ids are returned as read (1-based); filtering happens in
 * or_build_csr.  Returns the number of edge lines read, or -1 on a missing
 * file / bad header. */
i64 or_parse_graph(const char *path, int *n_out, i64 *m_hdr, int *u, int *v, i64 *c,
                   i64 cap_len) {
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    int n, m;
    if (fscanf(f, "%d %d", &n, &m) != 2) {
        fclose(f);
        return -1;
    }
    *n_out = n;
    *m_hdr = m;
    i64 k = 0;
    for (int i = 0; i < m && k < cap_len; ++i) {
        int a, b;
        long long w;
        if (fscanf(f, "%d %d %lld", &a, &b, &w) != 3) break;
        u[k] = a;
        v[k] = b;
        c[k] = w;
        ++k;
    }
    fclose(f);
    return k;
}

/* test.txt parsing (RA:2609-2621): pairs until the first failed scan. */
i64 or_parse_queries(const char *path, int *s, int *t, i64 cap_len) {
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    i64 k = 0;
    int a, b;
    while (k < cap_len && fscanf(f, "%d %d", &a, &b) == 2) {
        s[k] = a;
        t[k] = b;
        ++k;
    }
    fclose(f);
    return k;
}

/* ------------------------------------------------------------------------ */
/* Paired-arc CSR (RA:1068-1122).  u,v are 0-based.  An edge is skipped when
 * an endpoint is out of range, u == v, or cap <= 0 (RA:1073-1075).  Each kept
 * edge i appends a forward arc (cap) to row u and a reverse arc (0) to row v;
 * within a row, arcs keep input order.  rev pairs the two.  Output arrays
 * must hold 2*m entries (row: n+1).  Also fills the parse-time statistics
 * sum_cap_out/in and deg_out/in (RA:1085-1088) when non-NULL.
 * Returns the arc count. */
i64 or_build_csr(int n, i64 m, const int *u, const int *v, const i64 *c, int *row, int *col,
                 i64 *cap, int *rev) {
    int *deg = (int *)calloc((size_t)n + 1, sizeof(int));
    for (i64 i = 0; i < m; ++i) {
        int a = u[i], b = v[i];
        if (a < 0 || a >= n || b < 0 || b >= n) continue;
        if (a == b) continue;
        if (c[i] <= 0) continue;
        deg[a]++;
        deg[b]++;
    }
    row[0] = 0;
    for (int x = 0; x < n; ++x) row[x + 1] = row[x] + deg[x];
    int *cur = deg; /* reuse as cursor */
    for (int x = 0; x < n; ++x) cur[x] = row[x];
    for (i64 i = 0; i < m; ++i) {
        int a = u[i], b = v[i];
        if (a < 0 || a >= n || b < 0 || b >= n) continue;
        if (a == b) continue;
        if (c[i] <= 0) continue;
        int ea = cur[a]++;
        int eb = cur[b]++;
        col[ea] = b;
        cap[ea] = c[i];
        rev[ea] = eb;
        col[eb] = a;
        cap[eb] = 0;
        rev[eb] = ea;
    }
    i64 arcs = row[n];
    free(deg);
    return arcs;
}

/* Statistics over arcs with cap > 0 (RA:2707-2720). */
void or_degree_stats(int n, const int *row, const int *col, const i64 *cap, i64 *so, i64 *si,
                     int *dout, int *din) {
    memset(so, 0, sizeof(i64) * (size_t)n);
    memset(si, 0, sizeof(i64) * (size_t)n);
    memset(dout, 0, sizeof(int) * (size_t)n);
    memset(din, 0, sizeof(int) * (size_t)n);
    for (int x = 0; x < n; ++x)
        for (int e = row[x]; e < row[x + 1]; ++e)
            if (cap[e] > 0) {
                int y = col[e];
                so[x] += cap[e];
                si[y] += cap[e];
                dout[x]++;
                din[y]++;
            }
}

/* ------------------------------------------------------------------------ */
/* Capacity-degree score (RA:1141-1159):
 *   score = (ln(so*do + 1) + ln(si*di + 1)) / ln(sqrt(do*di) + 1),  1 if the
 *   denominator is 0.
 * The natural log is evaluated with a fixed sequence of IEEE double
 * operations so that CPU and GPU produce identical bits (the greedy packing
 * below is sensitive to the order of near-equal scores).  Method: x = m*2^k
 * with m in [sqrt(1/2), sqrt(2)); ln(m) = 2*atanh(z), z = (m-1)/(m+1),
 * summed as the odd power series 2z(1 + z^2/3 + z^4/5 + ... + z^22/23),
 * truncation below 1e-20 relative for |z| <= 0.1716. */
static const double OR_LN2 = 0.69314718055994530942;

double or_det_log(double x) {
    int k;
    double m = frexp(x, &k);
    if (m < 0.70710678118654752440) {
        m = m * 2.0;
        k = k - 1;
    }
    double z = (m - 1.0) / (m + 1.0);
    double z2 = z * z;
    double p = 1.0 / 23.0;
    for (int j = 21; j >= 1; j -= 2) {
        double t = p * z2;
        p = t + 1.0 / (double)j;
    }
    double r = (2.0 * z) * p;
    double kl = (double)k * OR_LN2;
    return kl + r;
}

double or_score(i64 so, i64 si, int dout, int din) {
    double dso = (double)so, dsi = (double)si, ddo = (double)dout, ddi = (double)din;
    double a = dso * ddo;
    double b = dsi * ddi;
    double num = or_det_log(a + 1.0) + or_det_log(b + 1.0);
    double pd = ddo * ddi;
    double den = or_det_log(sqrt(pd) + 1.0);
    if (den > 0.0) return num / den;
    return 1.0;
}

typedef struct {
    double s;
    int v;
} or_vinfo;

static int or_vinfo_cmp(const void *pa, const void *pb) {
    const or_vinfo *a = (const or_vinfo *)pa, *b = (const or_vinfo *)pb;
    if (a->s > b->s) return -1;
    if (a->s < b->s) return 1;
    return (a->v < b->v) ? -1 : (a->v > b->v);
}

/* Greedy least-loaded packing (RA:1162-1177): vertices in decreasing score
 * order (ties: increasing id — the reference's std::sort leaves ties in an
 * unspecified order), each to the region with the smallest load, lowest
 * index on equal loads; load += score. */
void or_partition(int n, int R, const i64 *so, const i64 *si, const int *dout, const int *din,
                  int *part, double *score_out) {
    or_vinfo *vi = (or_vinfo *)malloc(sizeof(or_vinfo) * (size_t)(n > 0 ? n : 1));
    for (int x = 0; x < n; ++x) {
        vi[x].s = or_score(so[x], si[x], dout[x], din[x]);
        vi[x].v = x;
        if (score_out) score_out[x] = vi[x].s;
    }
    qsort(vi, (size_t)n, sizeof(or_vinfo), or_vinfo_cmp);
    double *load = (double *)calloc((size_t)R, sizeof(double));
    for (int i = 0; i < n; ++i) {
        int best = 0;
        double bl = load[0];
        for (int r = 1; r < R; ++r)
            if (load[r] < bl) {
                bl = load[r];
                best = r;
            }
        part[vi[i].v] = best;
        load[best] += vi[i].s;
    }
    free(load);
    free(vi);
}

/* The same packing with the reference's own score arithmetic: libm log and
 * sqrt (std::log / std::sqrt, RA:1147-1151) instead of or_det_log.  Ties in
 * the decreasing-score order are again broken by increasing id.  Used only
 * to measure how far the deterministic log moves the partition. */
void or_partition_libm(int n, int R, const i64 *so, const i64 *si, const int *dout, const int *din,
                       int *part, double *score_out) {
    or_vinfo *vi = (or_vinfo *)malloc(sizeof(or_vinfo) * (size_t)(n > 0 ? n : 1));
    for (int x = 0; x < n; ++x) {
        double dso = (double)so[x], dsi = (double)si[x], ddo = (double)dout[x], ddi = (double)din[x];
        double num = log(dso * ddo + 1.0) + log(dsi * ddi + 1.0);
        double den = log(sqrt(ddo * ddi) + 1.0);
        vi[x].s = den > 0.0 ? num / den : 1.0;
        vi[x].v = x;
        if (score_out) score_out[x] = vi[x].s;
    }
    qsort(vi, (size_t)n, sizeof(or_vinfo), or_vinfo_cmp);
    double *load = (double *)calloc((size_t)R, sizeof(double));
    for (int i = 0; i < n; ++i) {
        int best = 0;
        double bl = load[0];
        for (int r = 1; r < R; ++r)
            if (load[r] < bl) {
                bl = load[r];
                best = r;
            }
        part[vi[i].v] = best;
        load[best] += vi[i].s;
    }
    free(load);
    free(vi);
}

/* Region-contiguous renumbering (RA:1193-1214) and CSR scatter with rev
 * remap (RA:1216-1259).  region_start has R+1 entries ([start,end) = entries
 * r, r+1).  Within a region vertices keep increasing old id; within a row
 * arcs keep their order. */
void or_reorder(int n, int R, const int *part, const int *row, const int *col, const i64 *cap,
                const int *rev, int *new_id, int *old_id, int *region_start, int *row2, int *col2,
                i64 *cap2, int *rev2) {
    int *cnt = (int *)calloc((size_t)R + 1, sizeof(int));
    for (int x = 0; x < n; ++x) {
        int r = part[x];
        if (r < 0 || r >= R) r = 0;
        cnt[r]++;
    }
    region_start[0] = 0;
    for (int r = 0; r < R; ++r) region_start[r + 1] = region_start[r] + cnt[r];
    for (int r = 0; r < R; ++r) cnt[r] = region_start[r];
    for (int x = 0; x < n; ++x) {
        int r = part[x];
        if (r < 0 || r >= R) r = 0;
        int p = cnt[r]++;
        new_id[x] = p;
        old_id[p] = x;
    }
    free(cnt);
    row2[0] = 0;
    for (int p = 0; p < n; ++p) {
        int x = old_id[p];
        row2[p + 1] = row2[p] + (row[x + 1] - row[x]);
    }
    i64 arcs = row[n];
    int *o2n = (int *)malloc(sizeof(int) * (size_t)(arcs > 0 ? arcs : 1));
    for (int x = 0; x < n; ++x) {
        int base = row2[new_id[x]];
        for (int e = row[x]; e < row[x + 1]; ++e) {
            int pos = base + (e - row[x]);
            col2[pos] = new_id[col[e]];
            cap2[pos] = cap[e];
            o2n[e] = pos;
        }
    }
    for (i64 e = 0; e < arcs; ++e) rev2[o2n[e]] = o2n[rev[e]];
    free(o2n);
}

/* ------------------------------------------------------------------------ */
/* Query prune masks.
 * mode 0 (RA:1391-1445): forward reach from s over arcs with cap > 0,
 *   intersected with the undirected component of t (all arcs, both
 *   directions exist as paired arcs), plus s and t.
 * mode 1 (engine default): forward reach from s over cap > 0 intersected
 *   with backward reach to t over cap > 0 — the vertices on some s-t path —
 *   plus s and t.  Contained in mode 0; both preserve the max-flow value.
 * Returns the number of marked vertices; mask is 0/1. */
static int *or_queue_buf(int n) { return (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1)); }

int or_prune_mask(int n, const int *row, const int *col, const i64 *cap, const int *rev, int s,
                  int t, int mode, unsigned char *mask) {
    memset(mask, 0, (size_t)n);
    if (s < 0 || s >= n || t < 0 || t >= n) return 0;
    unsigned char *fwd = (unsigned char *)calloc((size_t)n, 1);
    unsigned char *oth = (unsigned char *)calloc((size_t)n, 1);
    int *q = or_queue_buf(n);
    int qh = 0, qt = 0;
    fwd[s] = 1;
    q[qt++] = s;
    while (qh < qt) {
        int x = q[qh++];
        for (int e = row[x]; e < row[x + 1]; ++e) {
            int y = col[e];
            if (cap[e] > 0 && !fwd[y]) {
                fwd[y] = 1;
                q[qt++] = y;
            }
        }
    }
    qh = qt = 0;
    oth[t] = 1;
    q[qt++] = t;
    while (qh < qt) {
        int x = q[qh++];
        for (int e = row[x]; e < row[x + 1]; ++e) {
            int y = col[e];
            int ok = (mode == 0) ? 1 : (cap[rev[e]] > 0); /* mode 1: arc y->x has cap */
            if (ok && !oth[y]) {
                oth[y] = 1;
                q[qt++] = y;
            }
        }
    }
    int kept = 0;
    for (int x = 0; x < n; ++x)
        if (fwd[x] && oth[x]) mask[x] = 1;
    mask[s] = 1;
    mask[t] = 1;
    for (int x = 0; x < n; ++x) kept += mask[x];
    free(q);
    free(fwd);
    free(oth);
    return kept;
}

/* Induced subgraph by mask (RA:2477-2551).  Kept vertices are renumbered in
 * increasing old id; arcs keep row order; rev remapped.  Returns sub arcs;
 * *sub_n receives the vertex count. old2sub: n entries (-1 when dropped). */
i64 or_induced_subgraph(int n, const int *row, const int *col, const i64 *cap, const int *rev,
                        const unsigned char *mask, int *sub_n, int *old2sub, int *sub2old,
                        int *row2, int *col2, i64 *cap2, int *rev2) {
    int k = 0;
    for (int x = 0; x < n; ++x) {
        old2sub[x] = -1;
        if (mask[x]) {
            old2sub[x] = k;
            sub2old[k] = x;
            ++k;
        }
    }
    *sub_n = k;
    row2[0] = 0;
    for (int i = 0; i < k; ++i) {
        int x = sub2old[i], d = 0;
        for (int e = row[x]; e < row[x + 1]; ++e)
            if (old2sub[col[e]] != -1) ++d;
        row2[i + 1] = row2[i] + d;
    }
    i64 arcs = row[n];
    int *o2s = (int *)malloc(sizeof(int) * (size_t)(arcs > 0 ? arcs : 1));
    for (i64 e = 0; e < arcs; ++e) o2s[e] = -1;
    for (int i = 0; i < k; ++i) {
        int x = sub2old[i], pos = row2[i];
        for (int e = row[x]; e < row[x + 1]; ++e) {
            int y = old2sub[col[e]];
            if (y != -1) {
                col2[pos] = y;
                cap2[pos] = cap[e];
                o2s[e] = pos;
                ++pos;
            }
        }
    }
    for (i64 e = 0; e < arcs; ++e)
        if (o2s[e] != -1) rev2[o2s[e]] = o2s[rev[e]];
    free(o2s);
    return row2[k];
}

/* Boundary-aware core mask (RA:2340-2475), restated for the record.  region_of
 * gives each vertex's region.  keep_region = regions on some s-region ->
 * t-region path of the region graph; seeds = kept-region vertices that are in
 * s's or t's region or have an arc leaving their region; then up to hop_limit
 * intra-region hops.  s and t always kept. */
int or_boundary_core_mask(int n, int R, const int *row, const int *col, const int *region_of,
                          int s, int t, int hop_limit, unsigned char *mask) {
    memset(mask, 0, (size_t)n);
    if (s < 0 || s >= n || t < 0 || t >= n) return 0;
    unsigned char *adj = (unsigned char *)calloc((size_t)R * R, 1);
    unsigned char *bnd = (unsigned char *)calloc((size_t)n, 1);
    for (int x = 0; x < n; ++x)
        for (int e = row[x]; e < row[x + 1]; ++e) {
            int rx = region_of[x], ry = region_of[col[e]];
            if (rx != ry) {
                adj[(size_t)rx * R + ry] = 1;
                bnd[x] = 1;
            }
        }
    unsigned char *fs = (unsigned char *)calloc((size_t)R, 1), *tt = (unsigned char *)calloc((size_t)R, 1);
    int *rq = or_queue_buf(R);
    int qh = 0, qt = 0;
    fs[region_of[s]] = 1;
    rq[qt++] = region_of[s];
    while (qh < qt) {
        int r = rq[qh++];
        for (int r2 = 0; r2 < R; ++r2)
            if (adj[(size_t)r * R + r2] && !fs[r2]) {
                fs[r2] = 1;
                rq[qt++] = r2;
            }
    }
    qh = qt = 0;
    tt[region_of[t]] = 1;
    rq[qt++] = region_of[t];
    while (qh < qt) {
        int r = rq[qh++];
        for (int r2 = 0; r2 < R; ++r2)
            if (adj[(size_t)r2 * R + r] && !tt[r2]) {
                tt[r2] = 1;
                rq[qt++] = r2;
            }
    }
    int *dist = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int *q = or_queue_buf(n);
    qh = qt = 0;
    int rs = region_of[s], rt = region_of[t];
    for (int x = 0; x < n; ++x) {
        dist[x] = -1;
        int r = region_of[x];
        if (!(fs[r] && tt[r])) continue;
        if (r == rs || r == rt || bnd[x]) {
            mask[x] = 1;
            dist[x] = 0;
            q[qt++] = x;
        }
    }
    while (qh < qt) {
        int x = q[qh++];
        if (dist[x] >= hop_limit) continue;
        int rx = region_of[x];
        for (int e = row[x]; e < row[x + 1]; ++e) {
            int y = col[e];
            if (region_of[y] != rx) continue;
            if (!(fs[rx] && tt[rx])) continue;
            if (dist[y] == -1) {
                dist[y] = dist[x] + 1;
                mask[y] = 1;
                q[qt++] = y;
            }
        }
    }
    mask[s] = 1;
    mask[t] = 1;
    int kept = 0;
    for (int x = 0; x < n; ++x) kept += mask[x];
    free(adj);
    free(bnd);
    free(fs);
    free(tt);
    free(rq);
    free(dist);
    free(q);
    return kept;
}

/* ------------------------------------------------------------------------ */
/* Exact backward BFS distances to the seed set over residual arcs: dist[t] =
 * 0; x gets d+1 when some arc x->y with res > 0 has dist[y] = d.  Vertices
 * with seed[x] != 0 are extra level-0 seeds (the sink's role in RA:224-231,
 * where negative-excess vertices also seed); blocked[x] != 0 vertices are
 * never labeled.  Unreached vertices get n. */
void or_bfs_heights(int n, const int *row, const int *col, const int *rev, const i64 *res, int t,
                    const unsigned char *seed, const unsigned char *blocked, int *dist) {
    int *q = or_queue_buf(n);
    int qh = 0, qt = 0;
    for (int x = 0; x < n; ++x) dist[x] = n;
    for (int x = 0; x < n; ++x)
        if ((x == t || (seed && seed[x])) && !(blocked && blocked[x])) {
            dist[x] = 0;
            q[qt++] = x;
        }
    while (qh < qt) {
        int x = q[qh++];
        for (int e = row[x]; e < row[x + 1]; ++e) {
            int y = col[e];
            if (res[rev[e]] > 0 && dist[y] == n && !(blocked && blocked[y])) {
                dist[y] = dist[x] + 1;
                q[qt++] = y;
            }
        }
    }
    free(q);
}

/* ------------------------------------------------------------------------ */
/* Dinic.  res (2m, optional) receives the final residual capacities. */
typedef struct {
    int n;
    const int *row, *col, *rev;
    i64 *res;
    int *lvl, *it, *q;
    int *stk_v, *stk_e;
} or_dinic_ws;

static int or_dinic_bfs(or_dinic_ws *w, int s, int t) {
    for (int x = 0; x < w->n; ++x) w->lvl[x] = -1;
    int qh = 0, qt = 0;
    w->lvl[s] = 0;
    w->q[qt++] = s;
    while (qh < qt) {
        int x = w->q[qh++];
        for (int e = w->row[x]; e < w->row[x + 1]; ++e) {
            int y = w->col[e];
            if (w->res[e] > 0 && w->lvl[y] < 0) {
                w->lvl[y] = w->lvl[x] + 1;
                w->q[qt++] = y;
            }
        }
    }
    return w->lvl[t] >= 0;
}

/* Iterative blocking-flow DFS with current-arc pointers. */
static i64 or_dinic_augment(or_dinic_ws *w, int s, int t) {
    i64 total = 0;
    for (;;) {
        int depth = 0;
        w->stk_v[0] = s;
        int found = 0;
        while (depth >= 0) {
            int x = w->stk_v[depth];
            if (x == t) {
                found = 1;
                break;
            }
            int advanced = 0;
            for (; w->it[x] < w->row[x + 1]; ++w->it[x]) {
                int e = w->it[x];
                int y = w->col[e];
                if (w->res[e] > 0 && w->lvl[y] == w->lvl[x] + 1) {
                    w->stk_e[depth] = e;
                    w->stk_v[++depth] = y;
                    advanced = 1;
                    break;
                }
            }
            if (!advanced) {
                w->lvl[x] = -1; /* dead end */
                --depth;
                if (depth >= 0) ++w->it[w->stk_v[depth]];
            }
        }
        if (!found) break;
        i64 d = INT64_MAX;
        for (int i = 0; i < depth; ++i)
            if (w->res[w->stk_e[i]] < d) d = w->res[w->stk_e[i]];
        for (int i = 0; i < depth; ++i) {
            int e = w->stk_e[i];
            w->res[e] -= d;
            w->res[w->rev[e]] += d;
        }
        total += d;
    }
    return total;
}

i64 or_dinic(int n, const int *row, const int *col, const i64 *cap, const int *rev, int s, int t,
             i64 *res_out) {
    if (s < 0 || s >= n || t < 0 || t >= n || s == t) return 0;
    i64 arcs = row[n];
    or_dinic_ws w;
    w.n = n;
    w.row = row;
    w.col = col;
    w.rev = rev;
    w.res = res_out ? res_out : (i64 *)malloc(sizeof(i64) * (size_t)(arcs > 0 ? arcs : 1));
    memcpy(w.res, cap, sizeof(i64) * (size_t)arcs);
    w.lvl = (int *)malloc(sizeof(int) * (size_t)n);
    w.it = (int *)malloc(sizeof(int) * (size_t)n);
    w.q = (int *)malloc(sizeof(int) * (size_t)n);
    w.stk_v = (int *)malloc(sizeof(int) * ((size_t)n + 1));
    w.stk_e = (int *)malloc(sizeof(int) * ((size_t)n + 1));
    i64 flow = 0;
    while (or_dinic_bfs(&w, s, t)) {
        for (int x = 0; x < n; ++x) w.it[x] = row[x];
        flow += or_dinic_augment(&w, s, t);
    }
    if (!res_out) free(w.res);
    free(w.lvl);
    free(w.it);
    free(w.q);
    free(w.stk_v);
    free(w.stk_e);
    return flow;
}

/* Multi-threaded batch of independent Dinic solves (queries spread over
 * pthreads), used as the CPU baseline.  Invalid ids or s == t give 0
 * (RA:2659-2663). */
typedef struct {
    int n;
    const int *row, *col, *rev;
    const i64 *cap;
    int nq;
    const int *s, *t;
    i64 *flows;
    int *next;
    pthread_mutex_t *mu;
} or_batch_job;

static void *or_batch_worker(void *p) {
    or_batch_job *j = (or_batch_job *)p;
    for (;;) {
        pthread_mutex_lock(j->mu);
        int q = (*j->next)++;
        pthread_mutex_unlock(j->mu);
        if (q >= j->nq) break;
        j->flows[q] = or_dinic(j->n, j->row, j->col, j->cap, j->rev, j->s[q], j->t[q], NULL);
    }
    return NULL;
}

void or_dinic_batch(int n, const int *row, const int *col, const i64 *cap, const int *rev, int nq,
                    const int *s, const int *t, i64 *flows, int threads) {
    if (threads < 1) threads = 1;
    int next = 0;
    pthread_mutex_t mu;
    pthread_mutex_init(&mu, NULL);
    or_batch_job j = {n, row, col, rev, cap, nq, s, t, flows, &next, &mu};
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)threads);
    for (int i = 0; i < threads; ++i) pthread_create(&th[i], NULL, or_batch_worker, &j);
    for (int i = 0; i < threads; ++i) pthread_join(th[i], NULL);
    free(th);
    pthread_mutex_destroy(&mu);
}

/* ------------------------------------------------------------------------ */
/* Sequential FIFO push-relabel with exact global relabeling from the sink —
 * the one-thread form of the reference's scheme: discharge pushes excess to
 * the lowest residual neighbour and relabels to min+1 (RA:474-512), heights
 * come from a backward residual BFS from t (RA:203-233, 322-348), vertices
 * with height >= n are inactive (RA:466).  Phase 1 only: the flow value is
 * the sink excess (RA:2202-2204).  A global relabel runs every n relabels
 * and whenever the queue empties; the loop ends when a global relabel leaves
 * no active vertex. */
i64 or_push_relabel(int n, const int *row, const int *col, const i64 *cap, const int *rev, int s,
                    int t, i64 *res_out) {
    if (s < 0 || s >= n || t < 0 || t >= n || s == t) return 0;
    i64 arcs = row[n];
    i64 *res = res_out ? res_out : (i64 *)malloc(sizeof(i64) * (size_t)(arcs > 0 ? arcs : 1));
    memcpy(res, cap, sizeof(i64) * (size_t)arcs);
    i64 *ex = (i64 *)calloc((size_t)n, sizeof(i64));
    int *h = (int *)malloc(sizeof(int) * (size_t)n);
    int *inq = (int *)calloc((size_t)n, sizeof(int));
    int *fifo = (int *)malloc(sizeof(int) * ((size_t)n + 1));
    int head = 0, tail = 0, count = 0;
    for (int e = row[s]; e < row[s + 1]; ++e) {
        i64 d = res[e];
        if (d > 0) {
            res[e] -= d;
            res[rev[e]] += d;
            ex[col[e]] += d;
            ex[s] -= d;
        }
    }
    i64 relabels = 0;
    for (;;) {
        /* exact global relabel */
        unsigned char *blk = (unsigned char *)calloc((size_t)n, 1);
        blk[s] = 1;
        or_bfs_heights(n, row, col, rev, res, t, NULL, blk, h);
        free(blk);
        h[s] = n;
        head = tail = count = 0;
        for (int x = 0; x < n; ++x) inq[x] = 0;
        for (int x = 0; x < n; ++x)
            if (x != s && x != t && ex[x] > 0 && h[x] < n) {
                fifo[tail] = x;
                tail = (tail + 1) % (n + 1);
                inq[x] = 1;
                ++count;
            }
        if (count == 0) break;
        relabels = 0;
        while (count > 0 && relabels < n) {
            int x = fifo[head];
            head = (head + 1) % (n + 1);
            --count;
            inq[x] = 0;
            while (ex[x] > 0 && h[x] < n) {
                int minh = 2 * n + 1;
                int pushed_any = 0;
                for (int e = row[x]; e < row[x + 1] && ex[x] > 0; ++e) {
                    if (res[e] <= 0) continue;
                    int y = col[e];
                    if (h[x] == h[y] + 1) {
                        i64 d = ex[x] < res[e] ? ex[x] : res[e];
                        res[e] -= d;
                        res[rev[e]] += d;
                        ex[x] -= d;
                        ex[y] += d;
                        pushed_any = 1;
                        if (y != s && y != t && !inq[y] && ex[y] > 0) {
                            fifo[tail] = y;
                            tail = (tail + 1) % (n + 1);
                            inq[y] = 1;
                            ++count;
                        }
                    }
                }
                if (ex[x] > 0) {
                    for (int e = row[x]; e < row[x + 1]; ++e)
                        if (res[e] > 0 && h[col[e]] < minh) minh = h[col[e]];
                    h[x] = (minh >= n) ? n : minh + 1;
                    ++relabels;
                    (void)pushed_any;
                }
            }
        }
    }
    i64 flow = ex[t];
    if (!res_out) free(res);
    free(ex);
    free(h);
    free(inq);
    free(fifo);
    return flow;
}

/* ------------------------------------------------------------------------ */
/* Certifier.  Given final residual capacities res for the (s,t) problem and a
 * claimed value, checks:
 *   (1) 0 <= res[e] and res[e] + res[rev e] == cap[e] + cap[rev e];
 *   (2) excess(x) = inflow - outflow >= 0 for x != s (preflow), and, when
 *       require_flow != 0, == 0 for every x not in {s,t} (a zero-excess flow);
 *   (3) excess(t) == value;
 *   (4) T = vertices that reach t in the residual graph; s not in T; the
 *       capacity of the cut (V\T -> T) over original arcs equals value.
 * Returns 0 when all hold, else the number (1..4) of the first failed check.
 * *cut_out receives the cut capacity. */
int or_certify(int n, const int *row, const int *col, const i64 *cap, const int *rev, int s, int t,
               const i64 *res, i64 value, int require_flow, i64 *cut_out) {
    i64 arcs = row[n];
    for (i64 e = 0; e < arcs; ++e) {
        if (res[e] < 0) return 1;
        if (res[e] + res[rev[e]] != cap[e] + cap[rev[e]]) return 1;
    }
    i64 *ex = (i64 *)calloc((size_t)n, sizeof(i64));
    for (int x = 0; x < n; ++x)
        for (int e = row[x]; e < row[x + 1]; ++e) {
            i64 f = cap[e] - res[e]; /* net flow on the arc pair, seen from x */
            if (f > 0) {
                ex[x] -= f;
                ex[col[e]] += f;
            }
        }
    int bad = 0;
    for (int x = 0; x < n && !bad; ++x) {
        if (x == s) continue;
        if (ex[x] < 0) bad = 2;
        if (require_flow && x != t && ex[x] != 0) bad = 2;
    }
    if (!bad && ex[t] != value) bad = 3;
    free(ex);
    int *dist = (int *)malloc(sizeof(int) * (size_t)n);
    or_bfs_heights(n, row, col, rev, res, t, NULL, NULL, dist);
    i64 cut = 0;
    for (int x = 0; x < n; ++x) {
        if (dist[x] < n) continue; /* x in T */
        for (int e = row[x]; e < row[x + 1]; ++e)
            if (dist[col[e]] < n && cap[e] > 0) cut += cap[e];
    }
    if (cut_out) *cut_out = cut;
    if (!bad && dist[s] < n) bad = 4;
    if (!bad && cut != value) bad = 4;
    free(dist);
    return bad;
}
