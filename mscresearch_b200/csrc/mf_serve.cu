// Autotuner for the batched solver: chooses the region count R, the local
// cycle bound K (kernel_cycles_base, RA:1467) and the global-relabel
// frequency (GR_FREQ0, RA:1466, plus the work-based relabel trigger), and the
// query-group width, by timing mf_solve_batch on a sample of queries.
// Coordinate descent: one dimension at a time, keeping the fastest value.
// Every configuration must return the same flows (max-flow values are
// unique); a mismatch is reported as MF_ERR_INEXACT.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/maxflow_b200.h"

namespace {

int time_cfg(mf_graph *g, int nq, const int32_t *s, const int32_t *t, const mf_opts &o,
             std::vector<int64_t> &flows, double &ms) {
    flows.assign(nq, 0);
    int rc = mf_solve_batch(g, nq, s, t, &o, flows.data(), nullptr);  // warm-up
    if (rc) return rc;
    double best = 1e300;
    for (int rep = 0; rep < 2; ++rep) {
        rc = mf_solve_batch(g, nq, s, t, &o, flows.data(), nullptr);
        if (rc) return rc;
        best = std::min(best, mf_last_device_ms(g));
    }
    ms = best;
    return MF_OK;
}

}  // namespace

extern "C" int mf_autotune(mf_graph *g, int nq, const int32_t *s, const int32_t *t,
                           const mf_opts *base, mf_opts *best, int *best_R) {
    if (!g || nq <= 0 || !s || !t || !best) return MF_ERR_ARG;
    mf_opts cur;
    if (base) cur = *base;
    else mf_opts_default(&cur);
    int n = 0, R0 = 0;
    long long arcs = 0;
    mf_graph_info(g, &n, &arcs, &R0);
    std::vector<int64_t> ref, f;
    double best_ms = 0;
    int rc = time_cfg(g, nq, s, t, cur, ref, best_ms);
    if (rc) return rc;
    auto consider = [&](mf_opts cand) -> int {
        double ms = 0;
        int r = time_cfg(g, nq, s, t, cand, f, ms);
        if (r) return r;
        if (f != ref) return MF_ERR_INEXACT;
        if (ms < best_ms) {
            best_ms = ms;
            cur = cand;
        }
        return MF_OK;
    };
    const int groups[] = {1, 2, 4, 8};
    for (int G : groups) {
        if (G == cur.group_ctas) continue;
        mf_opts c = cur;
        c.group_ctas = G;
        if ((rc = consider(c))) return rc;
    }
    const int ks[] = {2, 4, 8, 16};
    for (int K : ks) {
        mf_opts c = cur;
        c.kernel_cycles = K;
        if ((rc = consider(c))) return rc;
    }
    const double alphas[] = {0.25, 0.5, 1.0, 2.0};
    for (double a : alphas) {
        if (a == cur.gr_work_alpha) continue;
        mf_opts c = cur;
        c.gr_work_alpha = a;
        if ((rc = consider(c))) return rc;
    }
    const int freqs[] = {8, 16, 32, 128};
    for (int fq : freqs) {
        if (fq == cur.gr_freq) continue;
        mf_opts c = cur;
        c.gr_freq = fq;
        if ((rc = consider(c))) return rc;
    }
    int bestR = R0;
    const int Rs[] = {32, 64, 128, 256, 512};
    for (int R : Rs) {
        if (R == R0 || R > n) continue;
        if ((rc = mf_graph_repartition(g, R))) return rc;
        double ms = 0;
        if ((rc = time_cfg(g, nq, s, t, cur, f, ms))) return rc;
        if (f != ref) return MF_ERR_INEXACT;
        if (ms < best_ms) {
            best_ms = ms;
            bestR = R;
        }
    }
    if ((rc = mf_graph_repartition(g, bestR))) return rc;
    *best = cur;
    if (best_R) *best_R = bestR;
    return MF_OK;
}
