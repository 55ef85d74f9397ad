/*
 * Strongly connected components and SCC contraction on the host — TEST
 * INFRASTRUCTURE ONLY (built into oracle/liboracle.so; the engine never
 * links, loads or calls it).
 *
 * Restates the reference's offline SCC tool,
 * SCC_CONTRACT/scc_contract.cpp ("SC"):
 *   - edge filter (SC:33-39): endpoints outside [0, n), self loops and
 *     capacities <= 0 are skipped; every other edge is an arc u -> v;
 *   - Kosaraju (SC:43-96): a first depth-first pass over the out-arcs (in
 *     input order, vertices in id order) records finishing order; a second
 *     pass over the in-arcs, taking roots in decreasing finishing time,
 *     numbers the components 0, 1, ... in the order it finds them (which is
 *     a topological order of the condensation);
 *   - contraction (SC:98-128): one arc per ordered pair of distinct
 *     components joined by an arc, its capacity the sum of theirs, listed in
 *     increasing (cu, cv).
 * tests/golden/make_scc_golden.py pins this restatement to the reference
 * tool itself (compiled from its source by oracle/build_ref.sh): both write
 * byte-identical files on every golden graph.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef long long i64;

/* Arc lists of the kept edges in input order: out-arcs (head) and in-arcs
 * (tail) as two CSR arrays.  Returns 0, or -1 when out of memory. */
static int sc_lists(int n, i64 m, const int *u, const int *v, const i64 *c, int **orow, int **ocol, int **irow,
                    int **icol) {
    int *od = (int *)calloc((size_t)n + 1, sizeof(int));
    int *id = (int *)calloc((size_t)n + 1, sizeof(int));
    if (!od || !id) {
        free(od);
        free(id);
        return -1;
    }
    i64 k = 0;
    for (i64 i = 0; i < m; ++i) {
        const int a = u[i], b = v[i];
        if (a < 0 || a >= n || b < 0 || b >= n || a == b || c[i] <= 0) continue;
        od[a + 1]++;
        id[b + 1]++;
        ++k;
    }
    for (int x = 0; x < n; ++x) {
        od[x + 1] += od[x];
        id[x + 1] += id[x];
    }
    int *oc = (int *)malloc(sizeof(int) * (size_t)(k > 0 ? k : 1));
    int *ic = (int *)malloc(sizeof(int) * (size_t)(k > 0 ? k : 1));
    int *fo = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int *fi = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    if (!oc || !ic || !fo || !fi) {
        free(od);
        free(id);
        free(oc);
        free(ic);
        free(fo);
        free(fi);
        return -1;
    }
    memcpy(fo, od, sizeof(int) * (size_t)n);
    memcpy(fi, id, sizeof(int) * (size_t)n);
    for (i64 i = 0; i < m; ++i) {
        const int a = u[i], b = v[i];
        if (a < 0 || a >= n || b < 0 || b >= n || a == b || c[i] <= 0) continue;
        oc[fo[a]++] = b;
        ic[fi[b]++] = a;
    }
    free(fo);
    free(fi);
    *orow = od;
    *ocol = oc;
    *irow = id;
    *icol = ic;
    return 0;
}

/* Component of every vertex (0-based, in the second pass's discovery
 * order); returns the number of components, or -1 when out of memory. */
int or_scc_kosaraju(int n, i64 m, const int *u, const int *v, const i64 *c, int *comp) {
    if (n <= 0) return 0;
    int *orow, *ocol, *irow, *icol;
    if (sc_lists(n, m, u, v, c, &orow, &ocol, &irow, &icol)) return -1;
    int *order = (int *)malloc(sizeof(int) * (size_t)n);
    int *stk = (int *)malloc(sizeof(int) * (size_t)n);
    int *nxt = (int *)malloc(sizeof(int) * (size_t)n);  // next out-arc of a vertex on the stack
    unsigned char *seen = (unsigned char *)calloc((size_t)n, 1);
    int C = -1;
    if (order && stk && nxt && seen) {
        /* pass 1: depth-first over out-arcs; a vertex is marked when pushed
         * and finishes once its arcs are exhausted */
        int no = 0;
        for (int r = 0; r < n; ++r) {
            if (seen[r]) continue;
            int sp = 0;
            stk[sp++] = r;
            nxt[r] = orow[r];
            seen[r] = 1;
            while (sp > 0) {
                const int x = stk[sp - 1];
                if (nxt[x] < orow[x + 1]) {
                    const int y = ocol[nxt[x]++];
                    if (!seen[y]) {
                        seen[y] = 1;
                        nxt[y] = orow[y];
                        stk[sp++] = y;
                    }
                } else {
                    order[no++] = x;
                    --sp;
                }
            }
        }
        /* pass 2: roots in decreasing finishing time; everything that reaches
         * a root over in-arcs and has no component yet joins it */
        for (int x = 0; x < n; ++x) comp[x] = -1;
        C = 0;
        for (int i = no - 1; i >= 0; --i) {
            const int r = order[i];
            if (comp[r] != -1) continue;
            int sp = 0;
            stk[sp++] = r;
            comp[r] = C;
            while (sp > 0) {
                const int x = stk[--sp];
                for (int e = irow[x]; e < irow[x + 1]; ++e) {
                    const int y = icol[e];
                    if (comp[y] == -1) {
                        comp[y] = C;
                        stk[sp++] = y;
                    }
                }
            }
            ++C;
        }
    }
    free(order);
    free(stk);
    free(nxt);
    free(seen);
    free(orow);
    free(ocol);
    free(irow);
    free(icol);
    return C;
}

typedef struct {
    int a, b;
    i64 cap;
} sc_arc;

static int sc_arc_cmp(const void *pa, const void *pb) {
    const sc_arc *x = (const sc_arc *)pa, *y = (const sc_arc *)pb;
    if (x->a != y->a) return x->a < y->a ? -1 : 1;
    if (x->b != y->b) return x->b < y->b ? -1 : 1;
    return 0;
}

/* Contracted arcs for a component labelling comp (any numbering): kept
 * edges between distinct components, summed per (comp u, comp v) pair,
 * written in increasing (cu, cv) into cu / cv / ccap (room for m entries).
 * Returns the number of contracted arcs, or -1 when out of memory. */
i64 or_scc_contract(int n, i64 m, const int *u, const int *v, const i64 *c, const int *comp, int *cu, int *cv,
                    i64 *ccap) {
    sc_arc *t = (sc_arc *)malloc(sizeof(sc_arc) * (size_t)(m > 0 ? m : 1));
    if (!t) return -1;
    i64 k = 0;
    for (i64 i = 0; i < m; ++i) {
        const int a = u[i], b = v[i];
        if (a < 0 || a >= n || b < 0 || b >= n || a == b || c[i] <= 0) continue;
        if (comp[a] == comp[b]) continue;
        t[k].a = comp[a];
        t[k].b = comp[b];
        t[k].cap = c[i];
        ++k;
    }
    qsort(t, (size_t)k, sizeof(sc_arc), sc_arc_cmp);
    i64 w = 0;
    for (i64 i = 0; i < k; ++i) {
        if (w > 0 && cu[w - 1] == t[i].a && cv[w - 1] == t[i].b) {
            ccap[w - 1] += t[i].cap;
        } else {
            cu[w] = t[i].a;
            cv[w] = t[i].b;
            ccap[w] = t[i].cap;
            ++w;
        }
    }
    free(t);
    return w;
}
