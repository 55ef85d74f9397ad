// Device solver: one persistent cooperative launch in which groups of CTAs
// each take (s,t) queries from a work queue and solve them to an exact
// maximum preflow (optionally a certified flow) in their own residual slot.
//
// Mapping to the reference (Region_Aware_PR_with_Pruning_BoundaryCore.cu,
// "RA"):
//   prune (fwd/bwd or fwd/undirected BFS) ... build_reachable_refined_from_st RA:1391-1445
//   init + source preflow ................... staticMaxFlow_kernel_1 / _7   RA:151-200
//   global relabel (frontier BFS from sink
//     and deficit vertices, warp-ballot
//     frontier compaction) .................. init_height_level_frontier + bfs_expand_frontier
//                                             RA:203-233, 322-348, driver RA:1499-1581
//   discharge (lane / warp / group per vertex
//     by degree, ballot/shuffle arc scans,
//     native 64-bit atomics) ................ staticMaxFlow_kernel_14_region RA:432-515
//   active worklist + counts ................ build_active_list_and_count RA:664-695
//   hot-region extra sweep .................. count_region_active_kernel + hot pass RA:283-318, 1899-1984
//   sparse-phase path push .................. try_push_along_path / _with_path_push RA:773-955
//   region-aware invalid-arc repair (RM) .... staticMaxFlow_kernel_17_region RA:605-657
//   stagnation / adaptive K, GR frequency ... RA:1845-1891
//   termination + read excess(t) ............ RA:1988, 2114, 2202-2204
//
// Load balance.  Every frontier and worklist holds each vertex at most once
// and is split by degree: vertices with at most HUB_T arcs fill the list
// from the front, "hubs" fill it from the back of the same array.  BFS levels
// give each warp 32 front vertices and spread their combined arcs over the
// lanes; hub arcs are cut into 32-arc chunks spread over all warps of the
// group.  Discharge runs one vertex per lane for vertices with at most
// SMALL_T arcs, one vertex per warp above that, and hubs chunked over the
// whole group with the excess handed out through an atomic budget.
//
// Exactness.  Every kernel keeps residuals non-negative and pairwise
// conserved with atomic updates; only the owner of a vertex (one lane or
// warp per vertex per pass, the budget for hubs, ownership stamps for path
// push) lowers its excess.  RM is the only step that creates negative excess
// (deficits), as in the reference; deficits are relabel seeds, and if any
// remain when no active vertex is left the solver drains them back from the
// sink (phase B) before resuming.  A solve ends only when an exact global
// relabel finds no vertex with positive excess that can reach the sink and
// no deficit: the preflow is then maximum and excess(t) is the max-flow value.
#include "mf_solver.cuh"

#include <climits>
#include <cstring>

// The slot's control words (CNT_WORDS ints):
//   cnt[0..7]    front tails of the list banks, cnt[16..23] their back (hub)
//                tails.  Banks are handed out in rotation; taking bank k
//                zeroes bank k+4 (mod 8), last read at least one group barrier
//                earlier (no code path takes more than three banks between
//                two barriers);
//   cnt[8..12]   query hand-off and serving request words;
//   cnt[30]      total chunks of the current hub pass;
//   cnt[32..38]  level state published by a solo search episode.
#define NBANKS 8
#define CNT_BACK 16
#define CNT_HUBCH 30  // total chunks of the current hub pass
#define CNT_ACT 40    // global relabel: active vertices to label
#define CNT_FOUND 41  // global relabel: active vertices labelled so far
#define CNT_FARCS 42  // global relabel: arcs of the vertices labelled so far
#define CNT_OPENED 43 // repair: an update opened a residual arc or cancelled flow
#define CNT_Q 8      // query handed to the group
#define CNT_FLAG 9   // misc uniform flag
#define CNT_RS 10    // serving: request source / sink / graph
#define CNT_RT 11
#define CNT_RG 12
#define ACC_BANK 16  // i64 fields per accumulator bank
#define ACC_TOT 64   // start of per-query totals (within acc, 64 i64 reserved for banks)
#define ACC_GR_DUR 80  // duration of the last global relabel (ns, leader's clock)
#define ACC_GR_END 81  // leader's clock at its end
#define DEEP_LEVELS 256  // a relabel search deeper than this is "deep" (see run_phases)

// accumulator fields (per bank)
#define A_SUMEX 0
#define A_HIGH 1
#define A_WORK 2
#define A_PUSH 3
#define A_HMIN 4
#define A_HMAX 5
#define A_FIXED 6
#define A_NDEF 7
#define A_VERTS 8
#define A_CUT 9
#define A_BAD 10
#define A_TIME 11   // leader's clock when it finished the round's discharge

// per-query totals
#define T_ARCS 0
#define T_VERTS 1
#define T_PUSH 2
#define T_MASKARCS 3
#define T_RARCS 4
#define T_HARCS 5
#define T_HPASS 6
#define T_HREL 7
#define T_LEVELS 8   // search levels (prune, relabels, certificate)
#define T_BU 9       // of which bottom-up
#define T_SOLO 10    // of which run solo by one CTA

#define SMALL_T 32  // at most this many arcs: one lane per vertex in discharge
#define MAX_WARPS 32

enum Phase { PH_A = 0, PH_B = 1, PH_C = 2 };

struct QCtx {
    // group geometry
    int G, crank, gw, gW, lane, wpc, warp;
    GroupBar *bar;
    int *err;
    u64 lim;
    // graph
    int n, R;
    const int *row, *col, *rev, *rof;
    const i64 *cap;
    const DGraph *gr;
    const int *giants;  // the graph's giant list (gr->giants), ngiant entries
    int ngiant;
    // slot
    DSlot st;
    int vf;  // kept vertices in the front part of vlist (the rest are at the back)
    // uniform control
    unsigned clock;
    int seq;   // list-bank sequence
    int aseq;  // accumulator-bank sequence
    bool leader;
    u64 t_start;
    u64 time_limit;
    u64 q_begin;
    u64 tm_relabel, tm_rounds;  // leader: accumulated phase times
    // per-warp counters (flushed at the end of the query)
    i64 w_arcs, w_verts, w_push;
    int bu_factor;  // direction switch of the searches (KOpts::bu_factor)
    int bu_arcs;    // and its arc criterion (KOpts::bu_arcs)
    bool no_cache;  // the graph's kept-set cache is stale (a served capacity update)
    i64 w_farcs;    // arcs of the vertices this thread labelled (relabel searches)

    __device__ bool sync() { return gsync(G, bar, err, lim); }
    // a vertex with arcs [b, e1) that for_giants covers
    __device__ __forceinline__ bool giant(int b, int e1) const { return giants && e1 - b > GIANT_T; }
    // barrier that also returns the front and back tails of list bank `bank`
    // as of the barrier
    __device__ bool sync_tails(int bank, int &ft, int &bt) {
        return gsync_snap(G, bar, err, lim, &st.cnt[bank], &st.cnt[CNT_BACK + bank], &ft, &bt);
    }
    // the same, also returning the values of the control words cnt[w3] and
    // cnt[w4] as of the barrier
    __device__ bool sync_tails4(int bank, int &ft, int &bt, int w3, int &v3, int w4, int &v4) {
        return gsync_impl(G, bar, err, lim, &st.cnt[bank], &st.cnt[CNT_BACK + bank], &ft, &bt, &st.cnt[w3], &v3,
                          &st.cnt[w4], &v4);
    }
    __device__ int take_bank() {
        int b = seq & (NBANKS - 1);
        if (leader) {
            int z = (seq + 4) & (NBANKS - 1);
            st.cnt[z] = 0;
            st.cnt[CNT_BACK + z] = 0;
        }
        ++seq;
        return b;
    }
    __device__ i64 *take_abank() {
        int b = aseq & 3;
        if (leader) {
            i64 *z = st.acc + ((aseq + 2) & 3) * ACC_BANK;
            for (int i = 0; i < ACC_BANK; ++i) z[i] = 0;
            z[A_HMIN] = INT_MAX;
            z[A_HMAX] = -1;
        }
        ++aseq;
        return st.acc + b * ACC_BANK;
    }
    // All 32 lanes call it: the counters live on the lanes that did the work
    // (lane 0, or the first lane of each 8-lane discharge tile).
    __device__ void flush_warp_counts() {
        i64 a = warp_sum_i64(w_arcs), v = warp_sum_i64(w_verts), p = warp_sum_i64(w_push);
        if (lane == 0) {
            i64 *tot = st.acc + ACC_TOT;
            if (a) atomic_add_i64(&tot[T_ARCS], a);
            if (v) atomic_add_i64(&tot[T_VERTS], v);
            if (p) atomic_add_i64(&tot[T_PUSH], p);
        }
        w_arcs = w_verts = w_push = 0;
    }
    __device__ __forceinline__ int deg(int v) const { return ldro(&row[v + 1]) - ldro(&row[v]); }
    // i-th kept vertex (front part, then back part)
    __device__ __forceinline__ int vat(int i) const {
        return ldcg(i < vf ? &st.vlist[i] : &st.vlist[n - 1 - (i - vf)]);
    }
};

// entry k of a list's back part
__device__ __forceinline__ int back_at(const QCtx &c, const int *L, int k) { return ldcg(&L[c.n - 1 - k]); }

// ---------------------------------------------------------------------------
// Class-aware warp-aggregated append: flagged lanes add w to list L, at the
// front (cnt[bank]) or, when w has more than HUB_T arcs, at the back
// (cnt[CNT_BACK + bank], stored at L[n-1-k]).  One atomicAdd per class per
// warp.  All 32 lanes must call it.
__device__ __forceinline__ void append2(QCtx &c, bool flag, int w, int *L, int bank,
                                        unsigned mask = MF_FULL) {
    unsigned any = __ballot_sync(mask, flag);
    if (any == 0) return;
    bool hub = false;
    if (flag) hub = c.deg(w) > HUB_T;
    unsigned fm = __ballot_sync(mask, flag && !hub);
    unsigned bm = any & ~fm;
    if (fm) {
        int ld = __ffs(fm) - 1, base = 0;
        if (c.lane == ld) base = atomicAdd(&c.st.cnt[bank], __popc(fm));
        base = __shfl_sync(mask, base, ld);
        if (flag && !hub) {
            int pos = base + __popc(fm & lanemask_lt());
            if (MF_OK_IDX(pos, c.n, 91)) L[pos] = w;
        }
    }
    if (bm) {
        int ld = __ffs(bm) - 1, base = 0;
        if (c.lane == ld) base = atomicAdd(&c.st.cnt[CNT_BACK + bank], __popc(bm));
        base = __shfl_sync(mask, base, ld);
        if (flag && hub) {
            int k = base + __popc(bm & lanemask_lt());
            if (MF_OK_IDX(k, c.n, 92)) L[c.n - 1 - k] = w;
        }
    }
}

// Single-lane append (no warp collectives).
__device__ __forceinline__ void append1(QCtx &c, int w, int *L, int bank) {
    if (c.deg(w) > HUB_T) {
        int k = atomicAdd(&c.st.cnt[CNT_BACK + bank], 1);
        if (MF_OK_IDX(k, c.n, 93)) L[c.n - 1 - k] = w;
    } else {
        int k = atomicAdd(&c.st.cnt[bank], 1);
        if (MF_OK_IDX(k, c.n, 94)) L[k] = w;
    }
}

__device__ __forceinline__ int warp_incl_scan_int(int x) {
    const int lane = lane_id();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(MF_FULL, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

// ---------------------------------------------------------------------------
// Level-synchronous frontier BFS over a growing two-ended queue Q: the
// frontier at a level is Q[flo,fhi) plus back entries [blo,bhi).
__shared__ int s_lbs_v[MAX_WARPS][32];
__shared__ int s_lbs_b[MAX_WARPS][32];
__shared__ int s_lbs_x[MAX_WARPS][32];

// One top-down level.  Functor cl(v, e, w, level) returns true when arc
// e = v->w claims w (it performs the claim itself).
// The level's work is spread over warps gw, gw + gW, ... (the whole group,
// or one CTA in a solo level).
template <class Claim>
__device__ void td_level(QCtx &c, int *Q, int bank, int flo, int fhi, int blo, int bhi, int level,
                         Claim cl, int gw, int gW) {
    int *sv = s_lbs_v[c.warp], *sb = s_lbs_b[c.warp], *sx = s_lbs_x[c.warp];
    // front: vpw vertices per warp (the frontier spread over all gW warps,
    // 1 to 32 each), their arcs balanced over the lanes
    const int nf = fhi - flo;
    const int vpw = max(1, min(32, (nf + gW - 1) / gW));
    const int stride = gW * vpw;
    // software-pipelined: the next step's frontier vertex is loaded before
    // this step's scan and its row bounds before this step's arcs
    int v_nx = 0;
    {
        const int i = flo + gw * vpw + c.lane;
        if (c.lane < vpw && i < fhi) v_nx = ldcg(&Q[i]);
    }
    bool have_nx = c.lane < vpw && flo + gw * vpw + c.lane < fhi;
    int b_nx = 0, d_nx = 0;
    if (have_nx && MF_OK_IDX(v_nx, c.n, 11)) {
        b_nx = ldro(&c.row[v_nx]);
        d_nx = ldro(&c.row[v_nx + 1]) - b_nx;
    }
    for (int base = flo + gw * vpw; base < fhi; base += stride) {
        const int v = v_nx, b = b_nx, d = d_nx;
        const int i2 = base + stride + c.lane;
        have_nx = c.lane < vpw && i2 < fhi;
        if (have_nx) v_nx = ldcg(&Q[i2]);
        int incl = warp_incl_scan_int(d);
        int total = __shfl_sync(MF_FULL, incl, 31);
        sv[c.lane] = v;
        sb[c.lane] = b;
        sx[c.lane] = incl - d;
        __syncwarp();
        b_nx = 0;
        d_nx = 0;
        if (have_nx && MF_OK_IDX(v_nx, c.n, 11)) {
            b_nx = ldro(&c.row[v_nx]);
            d_nx = ldro(&c.row[v_nx + 1]) - b_nx;
        }
        for (int k = 0; k < total; k += 32) {
            int j = k + c.lane;
            bool ok = false;
            int w = 0;
            if (j < total) {
                int o = 0;
#pragma unroll
                for (int step = 16; step > 0; step >>= 1)
                    if (sx[o + step] <= j) o += step;
                int e = sb[o] + (j - sx[o]);
                w = ldro(&c.col[e]);
                ok = cl(sv[o], e, w, level);
            }
            append2(c, ok, w, Q, bank);
        }
        __syncwarp();
        if (c.lane == 0) {
            c.w_arcs += total;
            c.w_verts += min(vpw, fhi - base);
        }
    }
    // back: hub arcs in 32-arc chunks over all warps of the group
    for (int k = blo; k < bhi; ++k) {
        int v = back_at(c, Q, k);
        int b = ldro(&c.row[v]), e1 = ldro(&c.row[v + 1]);
        int nch = (e1 - b + 31) >> 5;
        for (int ch = gw; ch < nch; ch += gW) {
            int e = b + ch * 32 + c.lane;
            bool ok = false;
            int w = 0;
            if (e < e1) {
                w = ldro(&c.col[e]);
                ok = cl(v, e, w, level);
            }
            append2(c, ok, w, Q, bank);
            if (c.lane == 0) c.w_arcs += min(32, e1 - (b + ch * 32));
        }
        if (c.lane == 0 && gw == 0) c.w_verts += 1;
    }
}

// One bottom-up level over a universe of candidates: uf(i), i < nuf, gives a
// vertex of at most HUB_T arcs and ub(k), k < nub, a hub, or -1 when the
// candidate is already visited.  par(w, e, x, level) tests whether arc
// e = w->x links w to the search; set(w, level) claims w and returns true
// (one lane calls it per candidate, so it may store without atomics).  Each
// lane first tests its own candidate's first BU_PRE arcs; the rest of a
// small candidate's arcs are scanned by 8-lane tiles (four per warp step),
// hubs by whole warps (one hub per warp); all stop at the first parent.
#define BU_PRE 4  // arcs a bottom-up candidate tests on its own lane before the tiles

template <class UF, class UB, class Par, class Set>
__device__ void bu_level(QCtx &c, int *Q, int bank, int level, int nuf, UF uf, int nub, UB ub, Par par,
                         Set set) {
    const int tile = c.lane >> 3, tb = tile << 3, tl = c.lane & 7;
    const unsigned tmask = 0xffu << tb;
    i64 arcs = 0;
    // Software-pipelined over the warp's steps: the next step's candidate
    // and its row bounds are loaded while this step's arcs are in flight,
    // so a step waits on about three memory latencies instead of five.
    const int stride = c.gW * 32;
    int w_nx = -1, b_nx = 0, e_nx = 0;
    {
        const int i = c.gw * 32 + c.lane;
        if (c.gw * 32 < nuf && i < nuf) w_nx = uf(i);
        if (w_nx >= 0) {
            b_nx = ldro(&c.row[w_nx]);
            e_nx = ldro(&c.row[w_nx + 1]);
        }
    }
    for (int base = c.gw * 32; base < nuf; base += stride) {
        const int w = w_nx, b = b_nx, e1 = e_nx;
        if (c.lane == 0) c.w_verts += min(32, nuf - base);
        // lane pass: every lane tests its own candidate's first BU_PRE arcs
        // (independent loads, 32 candidates at once); only candidates with
        // more arcs and no parent among those go on to the 8-lane tiles
        int xs[BU_PRE];
#pragma unroll
        for (int k = 0; k < BU_PRE; ++k) xs[k] = (w >= 0 && b + k < e1) ? ldro(&c.col[b + k]) : 0;
        {
            const int i = base + stride + c.lane;
            w_nx = (base + stride < nuf && i < nuf) ? uf(i) : -1;
            if (w_nx >= 0) {
                b_nx = ldro(&c.row[w_nx]);
                e_nx = ldro(&c.row[w_nx + 1]);
            }
        }
        bool claimed1 = false, more = false;
        if (w >= 0) {
            bool hit = false;
#pragma unroll
            for (int k = 0; k < BU_PRE; ++k) {
                const int e = b + k;
                if (e < e1) hit |= par(w, e, xs[k], level);
            }
            arcs += min(BU_PRE, e1 - b);
            if (hit) claimed1 = set(w, level);
            else more = e1 - b > BU_PRE;
        }
        append2(c, claimed1, w, Q, bank);
        unsigned todo = __ballot_sync(MF_FULL, more);
        while (todo) {
            unsigned rest = todo;
            for (int k = 0; k < tile && rest; ++k) rest &= rest - 1;
            int src = rest ? __ffs(rest) - 1 : -1;
            int wt = __shfl_sync(MF_FULL, w, src < 0 ? 0 : src);
            for (int k = 0; k < 4 && todo; ++k) todo &= todo - 1;
            bool claimed = false;
            if (src >= 0) {
                int b = ldro(&c.row[wt]) + BU_PRE, e1 = ldro(&c.row[wt + 1]);
                bool found = false;
                for (int eb = b; eb < e1 && !found; eb += 8) {
                    int e = eb + tl;
                    bool hit = e < e1 && par(wt, e, ldro(&c.col[e]), level);
                    found = __any_sync(tmask, hit);
                    if (tl == 0) arcs += min(8, e1 - eb);
                }
                if (found && tl == 0) claimed = set(wt, level);
            }
            __syncwarp();
            append2(c, claimed, wt, Q, bank);
        }
    }
    for (int k = c.gw; k < nub; k += c.gW) {
        int w = 0;
        if (c.lane == 0) w = ub(k);
        w = __shfl_sync(MF_FULL, w, 0);
        bool claimed = false;
        if (w >= 0) {
            int b = ldro(&c.row[w]), e1 = ldro(&c.row[w + 1]);
            unsigned hm = 0;
            for (int eb = b; eb < e1 && !hm; eb += 32) {
                int e = eb + c.lane;
                hm = __ballot_sync(MF_FULL, e < e1 && par(w, e, ldro(&c.col[e]), level));
                if (c.lane == 0) arcs += min(32, e1 - eb);
            }
            if (hm && c.lane == 0) claimed = set(w, level);
        }
        append2(c, claimed, w, Q, bank);
    }
    arcs = warp_sum_i64(arcs);
    if (c.lane == 0) c.w_arcs += arcs;
}

struct NoLevelHook {
    __device__ void operator()(int, int, int, int, int, int, int) const {}
};

#define SOLO_MAX 96         // a hub-free top-down frontier at most this large runs solo
#define SOLO_LEVELS 1024    // levels per solo episode at most
#define CNT_SOLO 32         // cnt[32..38]: state published by a solo episode
static_assert(CNT_SOLO >= CNT_BACK + NBANKS && CNT_SOLO > CNT_HUBCH && CNT_SOLO + 8 <= CNT_ACT && CNT_FOUND < CNT_WORDS,
              "solo state must not overlap the other control words");

// Direction-optimizing BFS: a level runs bottom-up when the frontier holds
// more than a 1/bu_factor share of the unvisited universe (nu - visited)
// and at least 1/64 of the universe, top-down otherwise.  Both directions append
// the newly visited vertices to Q, so the next level can run either way,
// and visited = the queue's length.
// Small top-down frontiers run "solo": the group's first CTA expands them
// level after level with block barriers (up to SOLO_LEVELS, while the
// frontier stays top-down, hub-free and at most SOLO_MAX), then publishes the level
// state; the other CTAs wait at one group barrier instead of one per level
// (deep, narrow searches: grids, chains).  nuf = nub = 0: top-down only.
// on_level(level, plo, phi, pblo, pbhi, tid, nthreads) runs at the start of
// each level on the threads doing it; [plo, phi) and back [pblo, pbhi) are
// the previous level's frontier.
template <class Claim, class UF, class UB, class Par, class Set, class Hook = NoLevelHook>
__device__ bool bfs_dir(QCtx &c, int *Q, int bank, int fhi, int bhi, Claim cl, int nuf, UF uf, int nub,
                        UB ub, Par par, Set set, Hook on_level = Hook{}, int *levels_out = nullptr,
                        int stop_at = -1, bool *stopped_out = nullptr, bool arcs_rule = false,
                        int max_levels = INT_MAX) {
    // stop_at >= 0: the search ends after the first level by which the
    // control word cnt[CNT_FOUND] (raised by cl / set) has reached stop_at.
    // arcs_rule: cl / set add the arcs of every vertex they claim to the
    // thread's w_farcs; the level's total (cnt[CNT_FARCS], snapshotted at the
    // level barrier) is the next frontier's arc count, and a frontier with
    // more than bu_arcs arcs per unvisited vertex also goes bottom-up (a few
    // hub vertices can carry more arcs than the whole unvisited universe
    // would cost to test)
    // max_levels: at most this many levels are expanded (a local relabel's
    // depth bound)
    int flo = 0, blo = 0, pflo = 0, pblo = 0, level = 0, nbu = 0, nsolo = 0;
    bool stopped = stop_at == 0;
    long long ffarcs = 0;  // arcs of the current frontier (0: unknown)
    int farcs_prev = 0;
    const long long nu = (long long)nuf + nub;
    const int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
    while (!stopped && (flo < fhi || blo < bhi) && level < max_levels) {
        const long long visited = (long long)fhi + bhi;
        const long long fsize = (long long)(fhi - flo) + (bhi - blo);
        // bottom-up sweeps the whole universe, so the frontier must also be a
        // sizeable share of it (a small frontier near the end of a deep
        // search is cheaper to expand than nu candidates are to check)
        const bool bottom_up = nu > visited && ((fsize * c.bu_factor > nu - visited && fsize * 64 > nu) ||
                                                (arcs_rule && ffarcs > (long long)c.bu_arcs * (nu - visited)));
        if (!bottom_up && c.G > 1 && fsize <= SOLO_MAX && bhi == blo) {
            if (c.crank == 0) {
                const int wpc = blockDim.x >> 5;
                for (int k = 0; k < SOLO_LEVELS; ++k) {
                    MF_TRACE(11, level);
                    on_level(level, pflo, flo, pblo, blo, threadIdx.x, blockDim.x);
                    td_level(c, Q, bank, flo, fhi, blo, bhi, level, cl, c.warp, wpc);
                    if (arcs_rule) {
                        const i64 x = warp_sum_i64(c.w_farcs);
                        c.w_farcs = 0;
                        if (c.lane == 0 && x) atomicAdd(&c.st.cnt[CNT_FARCS], (int)x);
                    }
                    __syncthreads();
                    const int ft = ldcg(&c.st.cnt[bank]), bt = ldcg(&c.st.cnt[CNT_BACK + bank]);
                    __syncthreads();
                    pflo = flo;
                    pblo = blo;
                    flo = fhi;
                    fhi = ft;
                    blo = bhi;
                    bhi = bt;
                    ++level;
                    // only this CTA claims during a solo episode, and its
                    // claims are complete at the block barrier above
                    bool done = stop_at > 0 && ldcg(&c.st.cnt[CNT_FOUND]) >= stop_at;
                    __syncthreads();
                    if (done) {
                        stopped = true;
                        break;
                    }
                    const long long fs = (long long)(fhi - flo) + (bhi - blo);
                    const long long vis = (long long)fhi + bhi;
                    if (level >= max_levels || fs == 0 || fs > SOLO_MAX || bhi != blo || (nu > vis && fs * c.bu_factor > nu - vis && fs * 64 > nu))
                        break;
                }
                if (threadIdx.x == 0) {
                    int *o = c.st.cnt + CNT_SOLO;
                    o[0] = flo;
                    o[1] = fhi;
                    o[2] = blo;
                    o[3] = bhi;
                    o[4] = level;
                    o[5] = pflo;
                    o[6] = pblo;
                    o[7] = stopped ? 1 : 0;
                }
            }
            if (!c.sync()) return false;
            const int *o = c.st.cnt + CNT_SOLO;
            nsolo += ldcg(&o[4]) - level;
            flo = ldcg(&o[0]);
            fhi = ldcg(&o[1]);
            blo = ldcg(&o[2]);
            bhi = ldcg(&o[3]);
            level = ldcg(&o[4]);
            pflo = ldcg(&o[5]);
            pblo = ldcg(&o[6]);
            stopped = ldcg(&o[7]) != 0;
            ffarcs = 0;  // solo frontiers are small; the vertex rule decides
            farcs_prev = ldcg(&c.st.cnt[CNT_FARCS]);  // stable: nobody claims until the next level
            continue;
        }
        MF_TRACE(10, level);
        on_level(level, pflo, flo, pblo, blo, gt, gT);
        if (bottom_up) {
            bu_level(c, Q, bank, level, nuf, uf, nub, ub, par, set);
            ++nbu;
        } else
            td_level(c, Q, bank, flo, fhi, blo, bhi, level, cl, c.gw, c.gW);
        int ft = 0, bt = 0;
        if (arcs_rule) {
            const i64 x = warp_sum_i64(c.w_farcs);
            c.w_farcs = 0;
            if (c.lane == 0 && x) atomicAdd(&c.st.cnt[CNT_FARCS], (int)x);
        }
        if (stop_at > 0 || arcs_rule) {
            int found = 0, farcs = 0;
            if (!c.sync_tails4(bank, ft, bt, CNT_FOUND, found, CNT_FARCS, farcs)) return false;
            if (stop_at > 0) stopped = found >= stop_at;
            ffarcs = (long long)farcs - farcs_prev;
            farcs_prev = farcs;
        } else if (!c.sync_tails(bank, ft, bt)) {
            return false;
        }
        pflo = flo;
        pblo = blo;
        flo = fhi;
        fhi = ft;
        blo = bhi;
        bhi = bt;
        ++level;
    }
    if (levels_out) *levels_out = level;
    if (stopped_out) *stopped_out = stopped;
    if (c.leader) {
        i64 *tot = c.st.acc + ACC_TOT;
        tot[T_LEVELS] += level;
        tot[T_BU] += nbu;
        tot[T_SOLO] += nsolo;
    }
    return true;
}

// The giants selected by sel(v) (uniform over the group), each with its
// arcs spread over all the group's threads: pv(v, b, e1) once per giant by
// the group's thread 0, pa(v, e) per arc.
template <class Sel, class PerV, class PerArc>
__device__ void for_giants(QCtx &c, Sel sel, PerV pv, PerArc pa) {
    const int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
    for (int k = 0; k < c.ngiant; ++k) {
        const int v = ldro(&c.giants[k]);
        if (!sel(v)) continue;
        const int b = ldro(&c.row[v]), e1 = ldro(&c.row[v + 1]);
        if (gt == 0) pv(v, b, e1);
        for (int e = b + gt; e < e1; e += gT) pa(v, e);
    }
}

struct NoCand {
    __device__ int operator()(int) const { return -1; }
};
struct NoPar {
    __device__ bool operator()(int, int, int, int) const { return false; }
};
struct NoSet {
    __device__ bool operator()(int, int) const { return false; }
};

template <class Claim>
__device__ bool bfs_levels(QCtx &c, int *Q, int bank, int fhi, int bhi, Claim cl) {
    return bfs_dir(c, Q, bank, fhi, bhi, cl, 0, NoCand{}, 0, NoCand{}, NoPar{}, NoSet{});
}

// ---------------------------------------------------------------------------
// Reachability over arcs with capacity, forward (dir 0: x -> w) or backward
// (dir 1: w -> x), from x.  Vertices whose stamp st[] is below S are
// unvisited; reached ones get S and are listed in Q (bank).  Bottom-up
// levels need the graph's hub list; without it the search is top-down.
__device__ bool reach_all(QCtx &c, int x, int dir, unsigned *st, unsigned S, int *Q, int bank) {
    if (c.leader) {
        st[x] = S;
        append1(c, x, Q, bank);
    }
    int f0 = 0, b0 = 0;
    if (!c.sync_tails(bank, f0, b0)) return false;
    const i64 *cap = c.cap;
    const int *rev = c.rev;
    auto td = [&](int v, int e, int w, int) -> bool {
        i64 ce = ldcap(&cap[dir ? ldro(&rev[e]) : e]);
        unsigned mw = ldcg(&st[w]);
        if (ce <= 0 || mw >= S) return false;
        return atomicMax(&st[w], S) < S;
    };
    const int *hubs = c.gr->hubs;
    const int nuf = hubs ? c.n : 0, nub = hubs ? c.gr->nhub : 0;
    auto uf = [&](int i) -> int { return (c.deg(i) <= HUB_T && ldcg(&st[i]) < S) ? i : -1; };
    auto ub = [&](int k) -> int {
        int w = ldro(&hubs[k]);
        return ldcg(&st[w]) < S ? w : -1;
    };
    auto par = [&](int w, int e, int y, int) -> bool {
        return ldcg(&st[y]) >= S && ldcap(&cap[dir ? e : ldro(&rev[e])]) > 0;
    };
    auto set = [&](int w, int) -> bool {
        st[w] = S;
        return true;
    };
    return bfs_dir(c, Q, bank, f0, b0, td, nuf, uf, nub, ub, par, set);
}

// Reachability from x in direction dir restricted to the vertices stamped
// S by an earlier search (listed in U: front nuf entries, back nub), which
// move to stamp M and are listed in vlist (bank vb).
__device__ bool reach_within(QCtx &c, int x, int dir, unsigned S, unsigned M, const int *U, int nuf, int nub,
                             int vb) {
    unsigned *mark = c.st.mark;
    if (c.leader) {
        mark[x] = M;
        append1(c, x, c.st.vlist, vb);
    }
    int f0 = 0, b0 = 0;
    if (!c.sync_tails(vb, f0, b0)) return false;
    const i64 *cap = c.cap;
    const int *rev = c.rev;
    auto td = [&](int v, int e, int w, int) -> bool {
        unsigned mw = ldcg(&mark[w]);
        i64 ce = ldcap(&cap[dir ? ldro(&rev[e]) : e]);
        if (mw != S || ce <= 0) return false;
        return atomicCAS(&mark[w], S, M) == S;
    };
    auto uf = [&](int i) -> int {
        int w = ldcg(&U[i]);
        return ldcg(&mark[w]) == S ? w : -1;
    };
    auto ub = [&](int k) -> int {
        int w = back_at(c, U, k);
        return ldcg(&mark[w]) == S ? w : -1;
    };
    auto par = [&](int w, int e, int y, int) -> bool {
        return ldcg(&mark[y]) == M && ldcap(&cap[dir ? e : ldro(&rev[e])]) > 0;
    };
    auto set = [&](int w, int) -> bool {
        mark[w] = M;
        return true;
    };
    if (!bfs_dir(c, c.st.vlist, vb, f0, b0, td, nuf, uf, nub, ub, par, set)) return false;
    c.vf = ldcg(&c.st.cnt[vb]);
    return true;
}

// ---------------------------------------------------------------------------
// Prune.  Stamps: S (first search), M = S+1 (kept), U (undirected, mode 0).
// Leaves the kept vertices in vlist (front c.vf entries, back nv - c.vf) and
// returns nv (0 if t is not reachable from s, in which case the flow is 0).
// Mode 1 keeps fwd(s) & bwd(t): a full search from one end, then a search
// from the other end inside the first one's set.  It starts from s, or from
// t when fb (the pivot closures) says t is outside F: then bwd(t) cannot
// meet F and the first search stays small, while fwd(s) may cover F.
__device__ bool prune(QCtx &c, int s, int t, int mode, unsigned S, unsigned M, int &nv, bool &t_reach,
                      const unsigned char *fb) {
    MF_TRACE(20, s);
    unsigned *mark = c.st.mark;
    int bank = c.take_bank();
    int vb = c.take_bank();
    if (mode == 1) {
        bool tfirst = fb && !(ldro_u8(&fb[t]) & KC_F);
        int a = tfirst ? t : s, b = tfirst ? s : t, dir1 = tfirst ? 1 : 0;
        if (!reach_all(c, a, dir1, mark, S, c.st.qa, bank)) return false;
        int nff = ldcg(&c.st.cnt[bank]), nfb = ldcg(&c.st.cnt[CNT_BACK + bank]);
        t_reach = ldcg(&mark[b]) >= S;
        if (!t_reach) {
            nv = 0;
            c.vf = 0;
            return true;
        }
        if (!reach_within(c, b, 1 - dir1, S, M, c.st.qa, nff, nfb, vb)) return false;
        nv = c.vf + ldcg(&c.st.cnt[CNT_BACK + vb]);
        return true;
    }
    // mode 0: forward reach of s
    if (!reach_all(c, s, 0, mark, S, c.st.qa, bank)) return false;
    int nff = ldcg(&c.st.cnt[bank]), nfb = ldcg(&c.st.cnt[CNT_BACK + bank]);
    t_reach = ldcg(&mark[t]) >= S;
    const int *hubs = c.gr->hubs;
    const int nuf = hubs ? c.n : 0, nub = hubs ? c.gr->nhub : 0;
    // mode 0: undirected component of t (all arcs) with qmark stamp U = M
    // (qmark stamps come from the same clock, so M is unused there), then
    // kept = forward-reached & undirected-reached, plus s and t.
    int ub = c.take_bank();
    unsigned *qm = c.st.qmark;
    if (c.leader) {
        qm[t] = M;
        append1(c, t, c.st.qb, ub);
    }
    int f0 = 0, b0 = 0;
    if (!c.sync_tails(ub, f0, b0)) return false;
    auto und = [&](int v, int e, int w, int) -> bool {
        if (ldcg(&qm[w]) >= M) return false;
        return atomicMax(&qm[w], M) < M;
    };
    auto und_uf = [&](int i) -> int { return (c.deg(i) <= HUB_T && ldcg(&qm[i]) < M) ? i : -1; };
    auto und_ub = [&](int k) -> int {
        int w = ldro(&hubs[k]);
        return ldcg(&qm[w]) < M ? w : -1;
    };
    auto und_par = [&](int w, int e, int x, int) -> bool { return ldcg(&qm[x]) >= M; };
    auto und_set = [&](int w, int) -> bool {
        qm[w] = M;
        return true;
    };
    if (!bfs_dir(c, c.st.qb, ub, f0, b0, und, nuf, und_uf, nub, und_ub, und_par, und_set)) return false;
    // intersect: sweep the forward list (both parts); s is in it
    int nf = nff + nfb;
    for (int base = c.gw * 32; base < nf; base += c.gW * 32) {
        int i = base + c.lane;
        bool keep = false;
        int v = 0;
        if (i < nf) {
            v = ldcg(i < nff ? &c.st.qa[i] : &c.st.qa[c.n - 1 - (i - nff)]);
            keep = (ldcg(&qm[v]) == M) || v == s;
            if (keep) mark[v] = M;
        }
        append2(c, keep, v, c.st.vlist, vb);
    }
    if (!c.sync()) return false;
    if (c.leader && !t_reach) {
        // t is always kept (RA:1443-1444) even when s cannot reach it
        append1(c, t, c.st.vlist, vb);
        mark[t] = M;
    }
    if (!c.sync()) return false;
    c.vf = ldcg(&c.st.cnt[vb]);
    nv = c.vf + ldcg(&c.st.cnt[CNT_BACK + vb]);
    return true;
}

// ---------------------------------------------------------------------------
// Kept set of a query with s in B and t in F that is not inside the cached
// component: the component plus the extras
//   X = vertices reachable from s without entering F (mark stamp S),
//   Y = vertices reaching t without entering B (qmark stamp S),
//   extras = (X & B) | (Y & F) | (X & Y).
// (A path from s can only leave F's complement for good, and a path into t
// only leave B's, so fwd(s) = F | X and bwd(t) = B | Y.)  Lists the image
// then the extras in vlist with mark = M, ex = h = 0; the caller copies the
// image's residuals and then fixes the extras' arcs (fix_extra_arcs).
__device__ bool prune_ext(QCtx &c, int s, int t, unsigned S, unsigned M, int &nv) {
    const DGraph &g = *c.gr;
    const unsigned char *fb = g.kc_fb;
    unsigned *mark = c.st.mark, *qm = c.st.qmark;
    const i64 *cap = c.cap;
    const int *rev = c.rev;
    int xb = c.take_bank(), yb = c.take_bank(), vb = c.take_bank();
    if (c.leader) {
        if (!(ldro_u8(&fb[s]) & KC_F)) {
            mark[s] = S;
            append1(c, s, c.st.qa, xb);
        }
        if (!(ldro_u8(&fb[t]) & KC_B)) {
            qm[t] = S;
            append1(c, t, c.st.qb, yb);
        }
        c.st.cnt[vb] = g.kc_f;  // the extras follow the image
        c.st.cnt[CNT_BACK + vb] = g.kc_b;
        c.st.acc[ACC_TOT + T_MASKARCS] = g.kc_arcs;
    }
    int f0 = 0, b0 = 0;
    if (!c.sync_tails(xb, f0, b0)) return false;
    auto xs = [&](int v, int e, int w, int) -> bool {
        i64 ce = ldcap(&cap[e]);
        unsigned mw = ldcg(&mark[w]);
        if (ce <= 0 || mw >= S || (ldro_u8(&fb[w]) & KC_F)) return false;
        return atomicMax(&mark[w], S) < S;
    };
    if (!bfs_levels(c, c.st.qa, xb, f0, b0, xs)) return false;
    // The Y seed count must come from a barrier snapshot: once a CTA starts
    // the Y search it appends to the same counter, and a plain read by a
    // slower CTA would see a different frontier (and level count).
    int yf0 = 0, yb0 = 0;
    if (!c.sync_tails(yb, yf0, yb0)) return false;
    auto ys = [&](int v, int e, int w, int) -> bool {
        i64 cr = ldcap(&cap[ldro(&rev[e])]);
        unsigned qw = ldcg(&qm[w]);
        if (cr <= 0 || qw >= S || (ldro_u8(&fb[w]) & KC_B)) return false;
        return atomicMax(&qm[w], S) < S;
    };
    if (!bfs_levels(c, c.st.qb, yb, yf0, yb0, ys)) return false;
    const int nxf = ldcg(&c.st.cnt[xb]), nx = nxf + ldcg(&c.st.cnt[CNT_BACK + xb]);
    const int nyf = ldcg(&c.st.cnt[yb]), ny = nyf + ldcg(&c.st.cnt[CNT_BACK + yb]);
    // image of the component
    const int nimg = g.kc_f + g.kc_b;
    int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
    for (int i = gt; i < nimg; i += gT) {
        int pos = i < g.kc_f ? i : c.n - 1 - (i - g.kc_f);
        int v = ldro(&g.kc_img[pos]);
        c.st.vlist[pos] = v;
        mark[v] = M;
        c.st.ex[v] = 0;
        c.st.h[v] = 0;
    }
    // extras
    i64 xarcs = 0;
    for (int base = c.gw * 32; base < nx + ny; base += c.gW * 32) {
        int i = base + c.lane;
        bool add = false;
        int v = 0;
        if (i < nx) {
            v = i < nxf ? ldcg(&c.st.qa[i]) : back_at(c, c.st.qa, i - nxf);
            add = (ldro_u8(&fb[v]) & KC_B) || ldcg(&qm[v]) == S;
        } else if (i < nx + ny) {
            int j = i - nx;
            v = j < nyf ? ldcg(&c.st.qb[j]) : back_at(c, c.st.qb, j - nyf);
            add = (ldro_u8(&fb[v]) & KC_F) != 0;
        }
        if (add) {
            mark[v] = M;
            c.st.ex[v] = 0;
            c.st.h[v] = 0;
            xarcs += c.deg(v);
        }
        append2(c, add, v, c.st.vlist, vb);
    }
    xarcs = warp_sum_i64(xarcs);
    if (c.lane == 0 && xarcs) atomic_add_i64(&c.st.acc[ACC_TOT + T_MASKARCS], xarcs);
    int nf = 0, nb = 0;
    if (!c.sync_tails(vb, nf, nb)) return false;
    c.vf = nf;
    nv = nf + nb;
    return true;
}

// Initial residuals on the arcs of the extras (vlist front entries from
// kc_f, back entries from kc_b): an arc between two kept vertices starts at
// its capacity, an arc from an extra to a dropped vertex at 0.  The image's
// residuals must be in place (they hold 0 on arcs into the extras).
__device__ bool fix_extra_arcs(QCtx &c, unsigned M, int nv) {
    const DGraph &g = *c.gr;
    const int xf = c.vf - g.kc_f;             // front extras
    const int nb = (nv - c.vf) - g.kc_b;      // back extras
    for (int i = c.gw; i < xf + nb; i += c.gW) {
        int v = i < xf ? ldcg(&c.st.vlist[g.kc_f + i]) : back_at(c, c.st.vlist, g.kc_b + (i - xf));
        int b = ldro(&c.row[v]), e1 = ldro(&c.row[v + 1]);
        if (c.lane == 0) c.w_verts += 1;
        if (c.giant(b, e1)) continue;
        for (int e = b + c.lane; e < e1; e += 32) {
            int w = ldro(&c.col[e]);
            bool kw = ldcg(&c.st.mark[w]) >= M;
            c.st.res[e] = kw ? ldcap(&c.cap[e]) : 0;
            if (kw) {
                int r = ldro(&c.rev[e]);
                c.st.res[r] = ldcap(&c.cap[r]);
            }
        }
    }
    // giant extras: kept and outside the cached component
    for_giants(
        c, [&](int v) { return ldcg(&c.st.mark[v]) >= M && !ldro_u8(&g.kc_in[v]); }, [&](int, int, int) {},
        [&](int, int e) {
            int w = ldro(&c.col[e]);
            bool kw = ldcg(&c.st.mark[w]) >= M;
            c.st.res[e] = kw ? ldcap(&c.cap[e]) : 0;
            if (kw) {
                int r = ldro(&c.rev[e]);
                c.st.res[r] = ldcap(&c.cap[r]);
            }
        });
    return c.sync();
}

// Per-query capacity overrides: the query's own capacity on each override
// arc whose ends are both kept (the residual was just initialised from the
// graph's capacity, which bounds the override from above, so the kept set
// computed with the graph's capacities covers the query's).
__device__ bool apply_overrides(QCtx &c, const KParams &p, int q, unsigned M) {
    const long long nov = p.ov_n;
    const i64 *caps = p.ov_cap + (long long)q * nov;
    int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
    for (long long j = gt; j < nov; j += gT) {
        const int e = ldro(&p.ov_arc[j]);
        const int w = ldro(&c.col[e]), a = ldro(&c.col[ldro(&c.rev[e])]);
        if (ldcg(&c.st.mark[w]) >= M && ldcg(&c.st.mark[a]) >= M) c.st.res[e] = ldro(&caps[j]);
    }
    return c.sync();
}

// ---------------------------------------------------------------------------
// Fresh residual state over the kept vertices: excess 0; res[e] = cap[e]
// when the head is kept, else 0 (the arc is outside the induced subgraph).
// count_mask: add the kept vertices' arcs to the query's mask-arc total.
__device__ bool init_state(QCtx &c, int nv, unsigned M, bool count_mask = true) {
    MF_TRACE(30, nv);
    i64 mask_arcs = 0;
    if ((i64)nv * 2 > c.n) {
        // Most vertices kept: a thread per kept vertex for its resets, then
        // one coalesced sweep over every arc of the graph (four per thread;
        // arcs whose tail was dropped are never read, so their value does
        // not matter).  A warp per vertex would walk ~10-arc lists with
        // dependent loads.
        const int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
        for (int i = gt; i < nv; i += gT) {
            int v = c.vat(i);
            c.st.ex[v] = 0;
            c.st.h[v] = 0;
            mask_arcs += c.deg(v);
            c.w_verts += 1;
        }
        const i64 A = ldro(&c.row[c.n]);
        // 16-byte vectors only on 16-byte aligned arrays (a caller-held CSR
        // need not be)
        const bool vec = ((reinterpret_cast<uintptr_t>(c.col) | reinterpret_cast<uintptr_t>(c.cap) |
                           reinterpret_cast<uintptr_t>(c.st.res)) & 15) == 0;
        const i64 nq4 = vec ? (A >> 2) : 0;
        const int4 *col4 = reinterpret_cast<const int4 *>(c.col);
        const longlong2 *cap2 = reinterpret_cast<const longlong2 *>(c.cap);
        longlong2 *res2 = reinterpret_cast<longlong2 *>(c.st.res);
        const unsigned *mark = c.st.mark;
        i64 swept = 0;
        for (i64 k = gt; k < nq4; k += gT) {
            const int4 w = __ldg(&col4[k]);
            const longlong2 ca = ldcap2(&cap2[2 * k]), cb = ldcap2(&cap2[2 * k + 1]);
            longlong2 ra, rb;
            ra.x = ldcg(&mark[w.x]) >= M ? ca.x : 0;
            ra.y = ldcg(&mark[w.y]) >= M ? ca.y : 0;
            rb.x = ldcg(&mark[w.z]) >= M ? cb.x : 0;
            rb.y = ldcg(&mark[w.w]) >= M ? cb.y : 0;
            res2[2 * k] = ra;
            res2[2 * k + 1] = rb;
            swept += 4;
        }
        for (i64 e = 4 * nq4 + gt; e < A; e += gT) {
            c.st.res[e] = ldcg(&mark[ldro(&c.col[e])]) >= M ? ldcap(&c.cap[e]) : 0;
            ++swept;
        }
        c.w_arcs += swept;
        mask_arcs = warp_sum_i64(mask_arcs);
        if (count_mask && c.lane == 0 && mask_arcs) atomic_add_i64(&c.st.acc[ACC_TOT + T_MASKARCS], mask_arcs);
        return c.sync();
    }
    for (int i = c.gw; i < nv; i += c.gW) {
        int v = c.vat(i);
        int b = ldro(&c.row[v]), e1 = ldro(&c.row[v + 1]);
        if (c.lane == 0) {
            c.st.ex[v] = 0;
            c.st.h[v] = 0;
        }
        mask_arcs += e1 - b;
        if (c.lane == 0) {
            c.w_arcs += e1 - b;
            c.w_verts += 1;
        }
        if (c.giant(b, e1)) continue;
        for (int e = b + c.lane; e < e1; e += 32) {
            int w = ldro(&c.col[e]);
            c.st.res[e] = (ldcg(&c.st.mark[w]) >= M) ? ldcap(&c.cap[e]) : 0;
        }
    }
    if (count_mask && c.lane == 0 && mask_arcs) atomic_add_i64(&c.st.acc[ACC_TOT + T_MASKARCS], mask_arcs);
    for_giants(
        c, [&](int v) { return ldcg(&c.st.mark[v]) >= M; }, [&](int, int, int) {},
        [&](int, int e) { c.st.res[e] = (ldcg(&c.st.mark[ldro(&c.col[e])]) >= M) ? ldcap(&c.cap[e]) : 0; });
    return c.sync();
}

// Saturate every residual arc out of s (RA:173-200; parallel over arcs).
__device__ bool preflow(QCtx &c, int s) {
    MF_TRACE(31, s);
    int b = ldro(&c.row[s]), e1 = ldro(&c.row[s + 1]);
    int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
    for (int e = b + gt; e < e1; e += gT) {
        i64 d = ldcg(&c.st.res[e]);
        if (d > 0) {
            c.st.res[e] = 0;
            atomic_add_i64(&c.st.res[ldro(&c.rev[e])], d);
            atomic_add_i64(&c.st.ex[ldro(&c.col[e])], d);
        }
    }
    return c.sync();
}

// ---------------------------------------------------------------------------
// BFS of the global relabel (direction-optimizing, exact levels) over the
// slot's bitmaps: `vis` (visited, pre-set for dropped vertices and the
// blocked vertex) and three frontier maps used in rotation (level L reads
// map L % 3, fills map (L+1) % 3 and takes the previous frontier's bits out
// of map (L-1) % 3, which level L+1 fills next).  The bitmaps
// (n/8 bytes each) stay in L2 while the per-vertex arrays do not, so the
// visited and frontier tests per examined arc cost no DRAM sector.
// Top-down: frontier vertex v claims an unvisited w with residual w->v
// (atomicOr on the visited word).  Bottom-up: an unvisited kept vertex w
// takes level + 1 when one of its residual arcs reaches the frontier map.
// Claims write the height and the next frontier bit.
// Q: the search queue (front / back parts of list bank `bank`).  raise_only:
// a reached vertex takes max(its height, its distance) (local relabels).
__device__ bool relabel_bfs(QCtx &c, int *Q, int nv, int bank, int fhi, int bhi, int &depth, int stop_at,
                            bool &stopped, int max_levels = INT_MAX, bool raise_only = false) {
    const int W = bitmap_words(c.n);
    unsigned *vis = c.st.bits + W, *F = c.st.bits + 2 * W;
    const int *rev = c.rev;
    i64 *res = c.st.res;
    int *h = c.st.h;
    const int *vl = c.st.vlist;
    auto fmap = [&](int level) -> unsigned * { return F + (size_t)(level % 3) * W; };
    // with stop_at >= 0, every labelled vertex holding excess is counted in
    // cnt[CNT_FOUND] (the search ends once all active vertices are labelled)
    const i64 *ex = c.st.ex;
    int *found = c.st.cnt + CNT_FOUND;
    const bool count = stop_at > 0;
    const bool arcs_rule = c.bu_arcs > 0;
    auto relab = [&](int v, int e, int w, int level) -> bool {
        const unsigned bit = 1u << (w & 31);
        unsigned vw = ldcg(&vis[w >> 5]);
        i64 rr = ldcg(&res[ldro(&rev[e])]);
        if ((vw & bit) || rr <= 0) return false;
        if (atomicOr(&vis[w >> 5], bit) & bit) return false;
        h[w] = raise_only ? max(ldcg(&h[w]), level + 1) : level + 1;
        atomicOr(&fmap(level + 1)[w >> 5], bit);
        if (count && ldcg(&ex[w]) > 0) atomicAdd(found, 1);
        if (arcs_rule) c.w_farcs += c.deg(w);
        return true;
    };
    auto unvisited = [&](int w) -> bool { return !((ldcg(&vis[w >> 5]) >> (w & 31)) & 1u); };
    auto uf = [&](int i) -> int {
        int w = ldcg(&vl[i]);
        return unvisited(w) ? w : -1;
    };
    auto ub = [&](int k) -> int {
        int w = back_at(c, vl, k);
        return unvisited(w) ? w : -1;
    };
    auto par = [&](int w, int e, int x, int level) -> bool {
        // both loads issued together (the frontier word is in L2)
        const i64 r = ldcg(&res[e]);
        const unsigned fw = ldcg(&fmap(level)[x >> 5]);
        return r > 0 && ((fw >> (x & 31)) & 1u);
    };
    auto set = [&](int w, int level) -> bool {
        const unsigned bit = 1u << (w & 31);
        h[w] = raise_only ? max(ldcg(&h[w]), level + 1) : level + 1;
        atomicOr(&vis[w >> 5], bit);
        atomicOr(&fmap(level + 1)[w >> 5], bit);
        if (count && ldcg(&ex[w]) > 0) atomicAdd(found, 1);
        if (arcs_rule) c.w_farcs += c.deg(w);
        return true;
    };
    // at level L the previous frontier's bits leave map (L - 1) % 3, which
    // level L + 1 fills again (cost: the frontier's size, not n)
    auto clear_prev = [&](int level, int plo, int phi, int pblo, int pbhi, int tid, int nth) {
        if (level == 0) return;
        unsigned *z = fmap(level - 1);
        for (int i = plo + tid; i < phi; i += nth) {
            int v = ldcg(&Q[i]);
            atomicAnd(&z[v >> 5], ~(1u << (v & 31)));
        }
        for (int k = pblo + tid; k < pbhi; k += nth) {
            int v = back_at(c, Q, k);
            atomicAnd(&z[v >> 5], ~(1u << (v & 31)));
        }
    };
    c.w_farcs = 0;
    return bfs_dir(c, Q, bank, fhi, bhi, relab, c.vf, uf, nv - c.vf, ub, par, set, clear_prev, &depth,
                   stop_at, &stopped, arcs_rule, max_levels);
}

// Kept-vertex bitmap of the query (bit v: mark[v] >= M), read by every
// global relabel to pre-set the visited map.
__device__ bool build_kept_bits(QCtx &c, unsigned M) {
    MF_TRACE(60, c.n);
    const int W = bitmap_words(c.n);
    for (int wd = c.gw; wd < W; wd += c.gW) {
        int v = wd * 32 + c.lane;
        unsigned word = __ballot_sync(MF_FULL, v < c.n && ldcg(&c.st.mark[v]) >= M);
        if (c.lane == 0) c.st.bits[wd] = word;
    }
    return c.sync();
}

// ---------------------------------------------------------------------------
// Exact global relabel.  Seeds at height 0: the phase sink (if any) and, in
// phases A and B, every deficit vertex (RA:224-231 seeds the sink and
// negative-excess vertices).  Backward BFS over residual arcs through kept
// vertices; the blocked vertex is never labeled.  Unreached kept vertices
// keep height n, and the active list (excess > 0, height < n, not
// the phase sink or blocked vertex) is compacted into L (front / back).
// Returns counts in naf / nab (active front / back) and nd (deficits).
// Dead vertices (height n + 1).  In phase A, a vertex that a complete
// search did not reach cannot reach the sink again: every vertex it can
// reach was unreached too, so sits at height >= n, where no push can enter
// it (a push needs a vertex one level higher) and RM leaves it alone; its
// residual reach therefore never grows.  keep_dead: dead marks from earlier
// relabels of this phase stand (else every kept vertex starts at n);
// mark_dead: the previous relabel's search was complete and its visited
// bitmap is intact, so the kept vertices it left unvisited become dead.
// Dead vertices are pre-marked visited (no search touches them) and are not
// counted among the active vertices an early stop waits for.  complete
// (out): this search was not stopped early.
__device__ bool global_relabel(QCtx &c, int nv, unsigned M, int sinkv, int blockv, int srcv,
                               bool deficit_seeds, int *L, int lbk, int &naf, int &nab, int &nd,
                               i64 *&ab, int &depth, bool early_stop, bool keep_dead = false,
                               bool mark_dead = false, bool *complete = nullptr) {
    MF_TRACE(40, nv);
    int qbk = c.take_bank();
    const int n = c.n;
    // bitmaps: visited = not kept, plus the blocked vertex; frontier maps empty
    const int W = bitmap_words(n);
    unsigned *kept = c.st.bits, *vis = kept + W, *F0 = kept + 2 * W;
    {
        int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
        for (int wd = gt; wd < W; wd += gT) {
            const unsigned kw = ldcg(&kept[wd]);
            unsigned x = ~kw;
            if (blockv >= 0 && wd == (blockv >> 5)) x |= 1u << (blockv & 31);
            // the third frontier map (first written at level 1) carries the
            // kept vertices the previous complete search left unvisited to
            // the seeds pass below
            F0[2 * W + wd] = mark_dead ? (kw & ~ldcg(&vis[wd])) : 0u;
            vis[wd] = x;
            F0[wd] = 0;
            F0[W + wd] = 0;
        }
        if (c.leader) {
            c.st.cnt[CNT_ACT] = 0;
            c.st.cnt[CNT_FOUND] = 0;
            c.st.cnt[CNT_FARCS] = 0;
        }
    }
    if (!c.sync()) return false;
    MF_TRACE(42, nv);
    // seeds (and, for an early stop, the count of active vertices: the
    // vertices the search labels and that hold excess)
    int nact = 0;
    for (int base = c.gw * 32; base < nv; base += c.gW * 32) {
        int i = base + c.lane;
        bool seed = false, act = false;
        int v = 0;
        if (i < nv) {
            v = c.vat(i);
            const i64 ev = ldcg(&c.st.ex[v]);
            if (v == sinkv) seed = true;
            else if (deficit_seeds && v != blockv && v != srcv && ev < 0) seed = true;
            bool dead = false;
            if (keep_dead && !seed && v != blockv)
                dead = ldcg(&c.st.h[v]) > n || (mark_dead && ((ldcg(&F0[2 * W + (v >> 5)]) >> (v & 31)) & 1u));
            act = !seed && !dead && v != blockv && ev > 0;
            if (seed) {
                atomicOr(&vis[v >> 5], 1u << (v & 31));
                atomicOr(&F0[v >> 5], 1u << (v & 31));
            } else if (dead) {
                atomicOr(&vis[v >> 5], 1u << (v & 31));
            }
            // every other kept vertex starts the search at height n (unreached)
            c.st.h[v] = seed ? 0 : (dead ? n + 1 : n);
        }
        nact += __popc(__ballot_sync(MF_FULL, act));
        append2(c, seed, v, c.st.qa, qbk);
    }
    if (early_stop && c.lane == 0 && nact) atomicAdd(&c.st.cnt[CNT_ACT], nact);
    int f0 = 0, b0 = 0;
    if (!c.sync_tails(qbk, f0, b0)) return false;
    if (mark_dead) {
        // the third frontier map is written from level 1 on (a solo episode
        // may reach it without a group barrier): clear it and wait
        int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
        for (int wd = gt; wd < W; wd += gT) F0[2 * W + wd] = 0;
        if (!c.sync()) return false;
    }
    MF_TRACE(43, f0 + b0);
    // Early stop: once every active vertex holds its exact height the
    // search ends; vertices it did not reach keep height n, which no push
    // can reach (a push needs a vertex one level higher), until the next
    // relabel.  A search that cannot reach some active vertex runs to the
    // end as before, so the relabel that ends a phase stays exact.
    const int stop_at = early_stop ? ldcg(&c.st.cnt[CNT_ACT]) : -1;
    bool stopped = false;
    if (!relabel_bfs(c, c.st.qa, nv, qbk, f0, b0, depth, stop_at, stopped)) return false;
    if (complete) *complete = !stopped;
    int *h = c.st.h;

    // Active list in decreasing height: the search queue (every reached
    // vertex, in level order) read backwards, so each round's warps take
    // the highest-labelled vertices first.  Active vertices are reached
    // ones; with deficit seeds every deficit is a seed and so in the queue
    // too, and one pass over the queue also yields the counts.  Without
    // them (a deficit may be unreached) the counts take a pass over the
    // kept vertices.
    MF_TRACE(41, 0);
    ab = c.take_abank();
    i64 l_sum = 0, l_def = 0;
    if (!deficit_seeds) {
        for (int i = c.gw * 32 + c.lane; i < nv; i += c.gW * 32) {
            const int v = c.vat(i);
            if (ldcg(&c.st.ex[v]) < 0 && v != srcv && v != blockv) ++l_def;
        }
    }
    {
        const int *Q = c.st.qa;
        const int qf = ldcg(&c.st.cnt[qbk]), qn = qf + ldcg(&c.st.cnt[CNT_BACK + qbk]);
        for (int base = c.gw * 32; base < qn; base += c.gW * 32) {
            const int i = base + c.lane;
            bool act = false;
            int v = 0;
            if (i < qn) {
                v = i < qf ? ldcg(&Q[qf - 1 - i]) : back_at(c, Q, qn - 1 - i);
                const i64 ev = ldcg(&c.st.ex[v]);
                act = ev > 0 && ldcg(&h[v]) < n && v != sinkv && v != blockv;
                if (act) l_sum += ev;
                if (deficit_seeds && ev < 0 && v != srcv && v != blockv) ++l_def;
            }
            append2(c, act, v, L, lbk);
        }
    }
    l_sum = warp_sum_i64(l_sum);
    l_def = warp_sum_i64(l_def);
    if (c.lane == 0) {
        if (l_sum) atomic_add_i64(&ab[A_SUMEX], l_sum);
        if (l_def) atomic_add_i64(&ab[A_NDEF], l_def);
    }
    if (!c.sync_tails(lbk, naf, nab)) return false;
    nd = (int)ldcg(&ab[A_NDEF]);
    return true;
}

// ---------------------------------------------------------------------------
// Local relabel (RA:236-279 init_local_frontier_in_band, RA:519-556
// compute_active_height_range / compute_region_active, driver RA:1583-1720).
// Between global relabels, when the active vertices' heights span at most
// LR_BAND levels: a backward search over the kept vertices of the regions
// that hold an active vertex (the next worklist N) whose height is below n
// (RA's band: its margin of n covers every height below n).  Seeds at
// height 0: the phase sink and, in phases A and B, the deficit vertices of
// that universe.  At most band + 3 levels are expanded (RA:1683 runs
// levels 0 .. band + 2).  A vertex the search reaches takes the larger of
// its height and its distance; one it does not reach, the seeds and the
// vertices outside the universe keep theirs.  RA's version sets the distance
// even where it is lower; here heights never fall between global relabels.
// A raised height may exceed a neighbour's outside the universe by more than
// one, which is what RM treats as an invalid arc: with both on, RM moved
// that flow back each time and an R-MAT 2^14 query with relabels every 64
// rounds ran into the launch time limit (with RA's lowering rule too), so
// RM is off while local relabels are on.  Exactness does not rest on these
// labels: only an exact global relabel ends a solve.  N is
// unchanged; the search queue is Q, a list buffer other than N (the
// worklist the next round fills).  The search overwrites the visited and
// frontier bitmaps, so the next global relabel takes no dead marks from
// them.
#define LR_BAND 128
__device__ bool local_relabel(QCtx &c, int nv, int sinkv, int blockv, int srcv, bool deficit_seeds, const int *N,
                              int nNf, int nNb, int *Q, int band, int &depth) {
    MF_TRACE(48, band);
    {
        const int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
        for (int i = gt; i < nNf + nNb; i += gT) {
            const int v = i < nNf ? ldcg(&N[i]) : back_at(c, N, i - nNf);
            c.st.ract[ldro(&c.rof[v])] = 1;
        }
    }
    const int qbk = c.take_bank();
    if (c.leader) c.st.cnt[CNT_FARCS] = 0;
    if (!c.sync()) return false;
    // visited = everything outside the universe, plus the seeds; the seeds
    // also form the first frontier
    const int n = c.n, W = bitmap_words(n);
    unsigned *kept = c.st.bits, *vis = kept + W, *F0 = kept + 2 * W;
    for (int wd = c.gw; wd < W; wd += c.gW) {
        const unsigned kw = ldcg(&kept[wd]);
        const int v = wd * 32 + c.lane;  // below n wherever its kept bit is set
        bool in = false, seed = false;
        if ((kw >> c.lane) & 1u) {
            in = v != blockv && ldcg(&c.st.h[v]) < n && ldcg(&c.st.ract[ldro(&c.rof[v])]) != 0;
            if (in)
                seed = v == sinkv || (deficit_seeds && v != srcv && ldcg(&c.st.ex[v]) < 0);
        }
        const unsigned inw = __ballot_sync(MF_FULL, in), sw = __ballot_sync(MF_FULL, seed);
        if (c.lane == 0) {
            vis[wd] = ~inw | sw;
            F0[wd] = sw;
            F0[W + wd] = 0;
            F0[2 * W + wd] = 0;
        }
        append2(c, seed, v, Q, qbk);
    }
    int f0 = 0, b0 = 0;
    if (!c.sync_tails(qbk, f0, b0)) return false;
    if (f0 + b0 == 0) return true;
    bool stopped = false;
    return relabel_bfs(c, Q, nv, qbk, f0, b0, depth, -1, stopped, band + 3, true);
}

// ---------------------------------------------------------------------------
// Push d along arc e = v->w; returns true when w turns active (its excess
// crosses from <= 0 to > 0) and should join the next worklist.
__device__ __forceinline__ bool push_arc(QCtx &c, int e, int w, i64 d, int sinkv, int blockv) {
    atomic_add_i64(&c.st.res[e], -d);
    atomic_add_i64(&c.st.res[ldro(&c.rev[e])], d);
    i64 old = atomic_add_i64(&c.st.ex[w], d);
    return old <= 0 && old + d > 0 && w != sinkv && w != blockv;
}

// Claim w for the next worklist (stamp de-dup) — true if this caller adds it.
__device__ __forceinline__ bool enlist(QCtx &c, int w, unsigned rstamp) {
    return atomicMax(&c.st.qmark[w], rstamp) < rstamp;
}

// Cooperative discharge of one vertex by a tile of TW lanes (TW = 8 or 32;
// the tile is lanes [tb, tb+TW) of the warp, mask its lane mask) for up to
// K cycles.  Each cycle scans v's arcs TW at a time: lanes read residual +
// head height, a ballot finds downhill residual arcs, a 64-bit inclusive
// shuffle scan splits the remaining excess over them in arc order, and every
// lane pushes its share with native 64-bit atomics.  If excess remains after
// all arcs, v is relabeled to 1 + the lowest height over arcs that still
// have residual (n when none).  Newly active heads and v itself (if still
// active) are appended to N.
//
// The caller passes v's arc range [b, e1), height hv and excess ev, the
// same values on every lane of the tile (read by one lane and broadcast):
// they steer tile-wide branches, and under independent thread scheduling
// per-lane loads could disagree (another warp may raise ex[v] meanwhile)
// and split the tile across its shuffles.  An excess read early is a lower
// bound (only this tile lowers ex[v]); the height is exact (only the owner
// relabels v during rounds).
template <int TW>
__device__ void discharge_tile(QCtx &c, int v, int b, int e1, int hv, i64 ev, int K, int sinkv, int blockv,
                               int *N, int nbk, unsigned rstamp, i64 *ab, unsigned mask, int tb) {
    const int n = c.n;
    const int tl = c.lane - tb;  // lane within the tile
    MF_TRACE(50, v);
    i64 pushes = 0, arcs = 0;
    for (int cyc = 0; cyc < K; ++cyc) {
        if (ev <= 0 || hv >= n) break;
        i64 rem = ev;
        int minh = MF_INF_H;
        // residual and head of the lane's arc are loaded one step ahead (a
        // residual read early is never above the current one: only this
        // tile lowers residuals out of v)
        i64 r_nx = 0;
        int w_nx = 0;
        if (b + tl < e1) {
            r_nx = ldcg(&c.st.res[b + tl]);
            w_nx = ldro(&c.col[b + tl]);
        }
        for (int base = b; base < e1; base += TW) {
            int e = base + tl;
            i64 r = r_nx;
            int w = w_nx, hw = MF_INF_H;
            if (e + TW < e1) {
                r_nx = ldcg(&c.st.res[e + TW]);
                w_nx = ldro(&c.col[e + TW]);
            } else {
                r_nx = 0;  // the lane has no arc in the next step
            }
            if (r > 0) hw = ldcg(&c.st.h[w]);
            bool adm = r > 0 && hw < hv;
            unsigned am = __ballot_sync(mask, adm);
            i64 d = 0;
            bool act = false;
            if (am) {
                i64 x = adm ? r : 0;
                i64 incl = x;
#pragma unroll
                for (int o = 1; o < TW; o <<= 1) {
                    i64 y = __shfl_up_sync(mask, incl, o, TW);
                    if (tl >= o) incl += y;
                }
                i64 excl = incl - x;
                if (adm && rem > excl) d = min(r, rem - excl);
                if (d > 0) act = push_arc(c, e, w, d, sinkv, blockv);
                i64 tot = __shfl_sync(mask, incl, TW - 1, TW);
                rem -= min(tot, rem);
                pushes += __popc(__ballot_sync(mask, d > 0));
            }
            if (r - d > 0) minh = min(minh, hw);
            bool add = act && enlist(c, w, rstamp);
            append2(c, add, w, N, nbk, mask);
            arcs += min(TW, e1 - base);
            if (rem == 0) break;
        }
        i64 pushed = ev - rem;
        if (tl == 0 && pushed) atomic_add_i64(&c.st.ex[v], -pushed);
        if (rem > 0) {
            int mh = __reduce_min_sync(mask, minh);
            hv = (mh >= n - 1) ? n : mh + 1;
            if (tl == 0) c.st.h[v] = hv;
        }
        __syncwarp(mask);
        if (tl == 0) ev = ldcg(&c.st.ex[v]);
        ev = __shfl_sync(mask, ev, 0, TW);
    }
    MF_TRACE(51, v);
    bool again = (tl == 0) && ev > 0 && hv < n && enlist(c, v, rstamp);
    append2(c, again, v, N, nbk, mask);
    if (tl == 0) {
        c.w_arcs += arcs;
        c.w_verts += 1;
        c.w_push += pushes;
        if (arcs) atomic_add_i64(&ab[A_WORK], arcs);
    }
}


// Discharge of the front part L[0, nf): each warp takes 32 entries.
// Vertices with at most SMALL_T arcs go to 8-lane tiles, four at a time (a
// tile reads 8 consecutive arcs per step); the others get the whole warp,
// with cycles capped so that one vertex scans at most about K x 32 arcs per
// round.  hot != NULL restricts the pass to vertices of hot regions.
__device__ void discharge_front(QCtx &c, const int *L, int nf, int K, int sinkv, int blockv,
                                int *N, int nbk, unsigned rstamp, i64 *ab, const int *hot) {
    // Software-pipelined: each lane loads the next step's entry, and then
    // its arc range, height and excess, while this step's tiles work.
    const int stride = c.gW * 32;
    auto entry = [&](int base) -> int {
        const int i = base + c.lane;
        int v = -1;
        if (base < nf && i < nf) {
            v = ldcg(&L[i]);
            if (!MF_OK_IDX(v, c.n, 12)) v = -1;
            else if (hot && !ldcg(&hot[ldro(&c.rof[v])])) v = -1;
        }
        return v;
    };
    int v_nx = entry(c.gw * 32);
    int b_nx = 0, e_nx = 0, h_nx = 0;
    i64 x_nx = 0;
    if (v_nx >= 0) {
        b_nx = ldro(&c.row[v_nx]);
        e_nx = ldro(&c.row[v_nx + 1]);
        h_nx = ldcg(&c.st.h[v_nx]);
        x_nx = ldcg(&c.st.ex[v_nx]);
    }
    for (int base = c.gw * 32; base < nf; base += stride) {
        const int v = v_nx, vb = b_nx, ve = e_nx, vh = h_nx;
        const i64 vx = x_nx;
        const int d = v >= 0 ? ve - vb : 0;
        v_nx = entry(base + stride);
        bool small = v >= 0 && d <= SMALL_T;
        unsigned sm = __ballot_sync(MF_FULL, small);
        unsigned med = __ballot_sync(MF_FULL, v >= 0 && !small);
        if (v_nx >= 0) {
            b_nx = ldro(&c.row[v_nx]);
            e_nx = ldro(&c.row[v_nx + 1]);
            h_nx = ldcg(&c.st.h[v_nx]);
            x_nx = ldcg(&c.st.ex[v_nx]);
        }
        // small vertices: 8-lane tiles, four per step
        const int tile = c.lane >> 3, tb = tile << 3;
        const unsigned tmask = 0xffu << tb;
        while (sm) {
            // the k-th set bit of sm for k = tile
            unsigned rest = sm;
            for (int k = 0; k < tile && rest; ++k) rest &= rest - 1;
            const int src = rest ? __ffs(rest) - 1 : -1, sl = src < 0 ? 0 : src;
            const int vt = __shfl_sync(MF_FULL, v, sl), bt = __shfl_sync(MF_FULL, vb, sl);
            const int et = __shfl_sync(MF_FULL, ve, sl), ht = __shfl_sync(MF_FULL, vh, sl);
            const i64 xt = __shfl_sync(MF_FULL, vx, sl);
            for (int k = 0; k < 4 && sm; ++k) sm &= sm - 1;
            if (src >= 0) discharge_tile<8>(c, vt, bt, et, ht, xt, K, sinkv, blockv, N, nbk, rstamp, ab, tmask, tb);
            __syncwarp();
        }
        // medium vertices: one warp each
        while (med) {
            int o = __ffs(med) - 1;
            med &= med - 1;
            const int vo = __shfl_sync(MF_FULL, v, o), bo = __shfl_sync(MF_FULL, vb, o);
            const int eo = __shfl_sync(MF_FULL, ve, o), ho = __shfl_sync(MF_FULL, vh, o);
            const i64 xo = __shfl_sync(MF_FULL, vx, o);
            int dv = eo - bo;
            int Kv = max(1, min(K, (K * 32) / max(dv, 1)));
            discharge_tile<32>(c, vo, bo, eo, ho, xo, Kv, sinkv, blockv, N, nbk, rstamp, ab, MF_FULL, 0);
        }
    }
}

// Hubs of L's back part, one cycle per round, spread over all warps of the
// group.  Set-up (before a group barrier): per hub, budget = its excess,
// minh = INF, done = 0, hv = its height; the first CTA then lays the hubs'
// 32-arc chunks out in one index space (exclusive prefix of the chunk
// counts) and every warp takes an equal contiguous range of it.  Per chunk a
// warp sums the downhill residual of its chunk, claims that much
// from the hub's budget with one atomicAdd (getting the whole amount, the
// rest, or nothing), spreads the claim over the chunk's downhill arcs in arc
// order, and folds the lowest height over arcs left with residual into
// minh.  The warp that finishes a hub's last chunk relabels it when budget
// is left (then every downhill arc was saturated, so minh >= its height) and
// re-lists it if it is still active.
__shared__ int s_hscan[MAX_WARPS];
__shared__ int s_htot;

__device__ bool hub_setup(QCtx &c, const int *L, int nb, const int *hot) {
    int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
    for (int k = gt; k < nb; k += gT) {
        int v = back_at(c, L, k);
        HubWork hw;
        hw.budget = ldcg(&c.st.ex[v]);
        hw.minh = MF_INF_H;
        hw.done = 0;
        hw.hv = ldcg(&c.st.h[v]);
        bool skip = hw.budget <= 0 || hw.hv >= c.n || (hot && !ldcg(&hot[ldro(&c.rof[v])]));
        hw.nch = skip ? 0 : (c.deg(v) + 31) >> 5;
        hw.cstart = 0;
        if (MF_OK_IDX(k, c.st.nhub, 95)) c.st.hubw[k] = hw;
    }
    if (!c.sync()) return false;
    // exclusive prefix of the chunk counts (first CTA of the group)
    if (c.crank == 0) {
        const int nw = blockDim.x >> 5;
        int carry = 0;
        for (int base = 0; base < nb; base += blockDim.x) {
            int k = base + threadIdx.x;
            bool in = k < nb && k < c.st.nhub;
            int x = in ? ldcg(&c.st.hubw[k].nch) : 0;
            int incl = warp_incl_scan_int(x);
            if (c.lane == 31) s_hscan[c.warp] = incl;  // warp totals
            __syncthreads();
            if (c.warp == 0) {
                int y = c.lane < nw ? s_hscan[c.lane] : 0;
                int yi = warp_incl_scan_int(y);
                if (c.lane < nw) s_hscan[c.lane] = yi - y;  // warp offsets
                if (c.lane == 31) s_htot = yi;              // tile total
            }
            __syncthreads();
            if (in) c.st.hubw[k].cstart = carry + s_hscan[c.warp] + incl - x;
            carry += s_htot;
            __syncthreads();
        }
        if (threadIdx.x == 0) c.st.cnt[CNT_HUBCH] = carry;
    }
    return c.sync();
}

__device__ void discharge_hubs(QCtx &c, const int *L, int nb, int sinkv, int blockv, int *N, int nbk,
                               unsigned rstamp, i64 *ab) {
    const int n = c.n;
    // this warp's arc examinations (statistics) and the arcs of the chunks it
    // covered, scanned or skipped (the relabel trigger's work measure: a
    // skipped chunk stands for work the pass did not need to repeat)
    i64 arcs = 0, work = 0;
    nb = min(nb, c.st.nhub);
    const int T = ldcg(&c.st.cnt[CNT_HUBCH]);
    // this warp's contiguous share of the (hub, chunk) index space
    const int j0 = (int)((long long)T * c.gw / c.gW), j1 = (int)((long long)T * (c.gw + 1) / c.gW);
    if (j0 < j1 && nb > 0) {
        // the hub holding chunk j0: the last k with cstart <= j0 (it has chunks)
        int lo = 0, hi = nb - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (ldcg(&c.st.hubw[mid].cstart) <= j0) lo = mid;
            else hi = mid - 1;
        }
        int k = lo;
        int cs = ldcg(&c.st.hubw[k].cstart), nch = ldcg(&c.st.hubw[k].nch);
        int j = j0;
        while (j < j1) {
            while (j >= cs + nch && k + 1 < nb) {
                ++k;
                cs = ldcg(&c.st.hubw[k].cstart);
                nch = ldcg(&c.st.hubw[k].nch);
            }
            if (j >= cs + nch) break;
            // this warp's run of hub k's chunks, [j, jend): the excess taken,
            // the lowest height left and the chunks done are flushed once
            // per run rather than once per chunk
            const int jbeg = j, jend = min(j1, cs + nch);
            HubWork *hw = &c.st.hubw[k];
            const int v = back_at(c, L, k);
            const int hv = ldcg(&hw->hv);
            const int b = ldro(&c.row[v]), e1 = ldro(&c.row[v + 1]);
            i64 take_sum = 0;
            int run_minh = MF_INF_H;
            // the lane's residual and head are loaded one chunk ahead (a
            // residual read early is never above the current one: only this
            // warp lowers the residuals of its run's arcs)
            i64 r_nx = 0;
            int w_nx = 0;
            {
                const int e = b + (j - cs) * 32 + c.lane;
                if (e < e1) {
                    r_nx = ldcg(&c.st.res[e]);
                    w_nx = ldro(&c.col[e]);
                }
            }
            for (; j < jend; ++j) {
                const int cb = b + (j - cs) * 32;
                const int e = cb + c.lane;
                const i64 r = r_nx;
                const int w = w_nx;
                // budget, head heights and the next chunk's arcs in flight together
                i64 bud = 0;
                if (c.lane == 0) bud = ldcg(&hw->budget);
                int hwt = MF_INF_H;
                if (r > 0) hwt = ldcg(&c.st.h[w]);
                if (j + 1 < jend && e + 32 < e1) {
                    r_nx = ldcg(&c.st.res[e + 32]);
                    w_nx = ldro(&c.col[e + 32]);
                } else {
                    r_nx = 0;  // no arc for this lane in the next chunk
                }
                // Once the hub's budget is spent the pass cannot end in a
                // relabel (budget only falls), so the rest of the run serves
                // nothing: its chunks are only counted as done.
                bud = __shfl_sync(MF_FULL, bud, 0);
                if (bud <= 0) {
                    if (c.lane == 0) work += min(e1, b + (jend - cs) * 32) - cb;
                    j = jend;
                    break;
                }
                bool adm = r > 0 && hwt < hv;
                i64 x = adm ? r : 0;
                i64 incl = warp_incl_scan_i64(x);
                i64 tot = __shfl_sync(MF_FULL, incl, 31);
                i64 take = 0;
                if (tot > 0) {
                    if (c.lane == 0) {
                        i64 old = atomic_add_i64(&hw->budget, -tot);
                        take = old >= tot ? tot : (old > 0 ? old : 0);
                    }
                    take = __shfl_sync(MF_FULL, take, 0);
                }
                i64 dd = 0;
                bool act = false;
                if (adm && take > incl - x) dd = min(r, take - (incl - x));
                if (dd > 0) act = push_arc(c, e, w, dd, sinkv, blockv);
                if (act) act = enlist(c, w, rstamp);
                append2(c, act, w, N, nbk);
                if (r - dd > 0) run_minh = min(run_minh, hwt);
                if (c.lane == 0) {
                    const int chunk_arcs = min(32, e1 - cb);
                    take_sum += take;
                    arcs += chunk_arcs;
                    work += chunk_arcs;
                    c.w_push += take ? 1 : 0;
                }
            }
            const int mh = __reduce_min_sync(MF_FULL, run_minh);
            if (c.lane == 0) {
                if (take_sum) atomic_add_i64(&c.st.ex[v], -take_sum);
                if (mh != MF_INF_H) atomicMin(&hw->minh, mh);
                const int nrun = jend - jbeg;
                __threadfence();
                if (atomicAdd(&hw->done, nrun) + nrun == nch) {
                    // last run of this hub: relabel if excess was left over
                    __threadfence();
                    i64 left = atomic_add_i64(&hw->budget, 0);
                    int hnew = hv;
                    atomic_add_i64(&c.st.acc[ACC_TOT + T_HPASS], 1);
                    if (left > 0) {
                        int m = atomicAdd(&hw->minh, 0);
                        hnew = (m >= n - 1) ? n : m + 1;
                        c.st.h[v] = hnew;
                        atomic_add_i64(&c.st.acc[ACC_TOT + T_HREL], 1);
                    }
                    i64 ev = ldcg(&c.st.ex[v]);
                    if (ev > 0 && hnew < n && enlist(c, v, rstamp)) append1(c, v, N, nbk);
                    c.w_verts += 1;
                }
            }
        }
    }
    if (c.lane == 0 && work) {
        c.w_arcs += arcs;
        atomic_add_i64(&ab[A_WORK], work);
        if (arcs) atomic_add_i64(&c.st.acc[ACC_TOT + T_HARCS], arcs);
    }
}

// Path push (RA:773-955): follow exactly-one-lower residual arcs from v for
// up to max_path hops, pushing the whole excess along; vertices on the path
// are claimed with a per-round ownership stamp so that only one warp ever
// lowers a vertex's excess.  Relabels in place when stuck (bounded retries).
__device__ void path_push_vertex(QCtx &c, int v, int max_path, int sinkv, int blockv, int *N,
                                 int nbk, unsigned rstamp, unsigned pstamp, i64 *ab) {
    const int n = c.n;
    MF_TRACE(60, v);
    bool own = false;
    if (c.lane == 0) own = atomicMax(&c.st.claim[v], pstamp) < pstamp;
    own = __shfl_sync(MF_FULL, own, 0);
    if (!own) return;
    int cur = v;
    int hops = 0, steps = 0;
    i64 arcs = 0, pushes = 0;
    while (hops < max_path && steps < 2 * max_path + 8) {
        ++steps;
        i64 ec = 0;
        int hc = 0;
        if (c.lane == 0) {
            ec = ldcg(&c.st.ex[cur]);
            hc = ldcg(&c.st.h[cur]);
        }
        ec = __shfl_sync(MF_FULL, ec, 0);
        hc = __shfl_sync(MF_FULL, hc, 0);
        if (ec <= 0 || cur == sinkv || hc >= n) break;
        int b = ldro(&c.row[cur]), e1 = ldro(&c.row[cur + 1]);
        int best_e = INT_MAX, minh = MF_INF_H;
        for (int base = b; base < e1; base += 32) {
            int e = base + c.lane;
            if (e < e1) {
                i64 r = ldcg(&c.st.res[e]);
                if (r > 0) {
                    int hw = ldcg(&c.st.h[ldro(&c.col[e])]);
                    minh = min(minh, hw);
                    if (hw == hc - 1) best_e = min(best_e, e);
                }
            }
            arcs += min(32, e1 - base);
        }
        best_e = __reduce_min_sync(MF_FULL, best_e);
        minh = __reduce_min_sync(MF_FULL, minh);
        if (best_e != INT_MAX) {
            int nxt = 0;
            bool cont = false;
            if (c.lane == 0) {
                int w = ldro(&c.col[best_e]);
                i64 r = ldcg(&c.st.res[best_e]);
                i64 d = min(ec, r);
                bool act = false;
                if (d > 0) {
                    act = push_arc(c, best_e, w, d, sinkv, blockv);
                    atomic_add_i64(&c.st.ex[cur], -d);
                    ++pushes;
                }
                if (ec - d > 0 && enlist(c, cur, rstamp)) append1(c, cur, N, nbk);
                if (w != sinkv && w != blockv && atomicMax(&c.st.claim[w], pstamp) < pstamp) {
                    cont = true;
                    nxt = w;
                } else if (act && enlist(c, w, rstamp)) {
                    append1(c, w, N, nbk);
                }
            }
            cont = __shfl_sync(MF_FULL, cont, 0);
            nxt = __shfl_sync(MF_FULL, nxt, 0);
            ++hops;
            if (!cont) {
                cur = -1;
                break;
            }
            cur = nxt;
        } else {
            int nh = (minh >= n - 1) ? n : minh + 1;
            if (c.lane == 0) c.st.h[cur] = nh;
            if (nh >= n) break;
        }
    }
    if (c.lane == 0 && cur >= 0) {
        i64 ec = ldcg(&c.st.ex[cur]);
        if (ec > 0 && ldcg(&c.st.h[cur]) < n && cur != sinkv && enlist(c, cur, rstamp))
            append1(c, cur, N, nbk);
    }
    if (c.lane == 0) {
        c.w_arcs += arcs;
        c.w_verts += hops + 1;
        c.w_push += pushes;
        if (arcs) atomic_add_i64(&ab[A_WORK], arcs);
    }
}

// Hot-region selection (RA:1902-1946): per-region counts of the worklist,
// top-K regions with a non-zero count become hot.  CTA 0 of the group
// bitonic-sorts (count desc, region asc) in shared memory.
__device__ bool select_hot(QCtx &c, const int *N, int nNf, int nNb, int hot_k) {
    MF_TRACE(70, nNf);
    const int R = c.R;
    int *hot = c.st.hot;
    int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
    for (int i = gt; i < nNf + nNb; i += gT) {
        int v = i < nNf ? ldcg(&N[i]) : back_at(c, N, i - nNf);
        atomicAdd(&hot[ldro(&c.rof[v])], 1);
    }
    if (!c.sync()) return false;
    if (c.crank == 0) {
        __shared__ long long keys[1024];
        int P = 1;
        while (P < R) P <<= 1;
        for (int i = threadIdx.x; i < P; i += blockDim.x) {
            long long k = LLONG_MAX;
            if (i < R) k = ((long long)(INT_MAX - ldcg(&hot[i])) << 16) | i;
            keys[i] = k;
        }
        __syncthreads();
        for (int k = 2; k <= P; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = threadIdx.x; i < P; i += blockDim.x) {
                    int ixj = i ^ j;
                    if (ixj > i) {
                        long long a = keys[i], b2 = keys[ixj];
                        bool up = ((i & k) == 0);
                        if ((a > b2) == up) {
                            keys[i] = b2;
                            keys[ixj] = a;
                        }
                    }
                }
                __syncthreads();
            }
        for (int i = threadIdx.x; i < R; i += blockDim.x) {
            long long k = keys[i];
            int r = (int)(k & 0xffff);
            int cntv = INT_MAX - (int)(k >> 16);
            keys[i] = ((long long)r << 1) | ((i < hot_k && cntv > 0) ? 1 : 0);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < R; i += blockDim.x) {
            long long k = keys[i];
            hot[(int)(k >> 1)] = (int)(k & 1);
        }
    }
    return c.sync();
}

// RM (RA:605-657): for kept vertices in active regions with height in the
// band, every arc v->w to a kept w with h(w) > h(v)+1, excess(w) <= 0 and
// residual on w->v has that residual moved from w to v (saturating the steep
// arc w->v).  Residuals updated atomically; w may go negative (a deficit).
__device__ bool rm_pass(QCtx &c, int nv, unsigned M, int hlo, int hhi, int s, int t, int *N,
                        int nbk, unsigned rstamp, i64 *ab) {
    const int n = c.n;
    MF_TRACE(80, nv);
    i64 fixed = 0;
    for (int i = c.gw; i < nv; i += c.gW) {
        int v = c.vat(i);
        if (v == s || v == t) continue;
        if (!ldcg(&c.st.ract[ldro(&c.rof[v])])) continue;
        int hv = 0;
        if (c.lane == 0) hv = ldcg(&c.st.h[v]);
        hv = __shfl_sync(MF_FULL, hv, 0);
        if (hv < hlo || hv > hhi || hv >= n) continue;
        int b = ldro(&c.row[v]), e1 = ldro(&c.row[v + 1]);
        i64 gained = 0;
        for (int base = b; base < e1; base += 32) {
            int e = base + c.lane;
            i64 d = 0;
            if (e < e1) {
                int w = ldro(&c.col[e]);
                // heads at height n (not reached by the last relabel's
                // search) are left alone: nothing can push into them
                const int hw = ldcg(&c.st.mark[w]) >= M ? ldcg(&c.st.h[w]) : 0;
                if (hw > hv + 1 && hw < n && ldcg(&c.st.ex[w]) <= 0) {
                    int re = ldro(&c.rev[e]);
                    if (ldcg(&c.st.res[re]) > 0) {
                        d = (i64)atomicExch(reinterpret_cast<u64 *>(&c.st.res[re]), 0ull);
                        if (d > 0) {
                            atomic_add_i64(&c.st.res[e], d);
                            atomic_add_i64(&c.st.ex[w], -d);
                        }
                    }
                }
            }
            gained += d;
            fixed += (d > 0);
        }
        gained = warp_sum_i64(gained);
        bool add = false;
        if (c.lane == 0 && gained > 0) {
            atomic_add_i64(&c.st.ex[v], gained);
            add = enlist(c, v, rstamp);
        }
        append2(c, add, v, N, nbk);
        if (c.lane == 0) {
            c.w_arcs += e1 - b;
            c.w_verts += 1;
        }
    }
    fixed = warp_sum_i64(fixed);
    if (c.lane == 0 && fixed) atomic_add_i64(&ab[A_FIXED], fixed);
    return c.sync();
}

// ---------------------------------------------------------------------------
// The push-relabel driver (RA:1450-2115, device-resident): relabel -> rounds
// of discharge (+ hot sweep, path push, RM, stagnation control) -> relabel
// ... until a relabel finds nothing to do.  start_phase PH_A: maximum preflow
// for (s,t); PH_C: return excess to s.
// dead_in: the dead-mark state a warm start inherits (0: none; 1: heights
// above n are dead marks; 2: also the visited bitmap of a complete search,
// see repair); dead_out (may be NULL): the state this call leaves, for the
// next warm start.
__device__ bool run_phases(QCtx &c, const KOpts &o, int s, int t, int nv, unsigned M,
                           int start_phase, QOut &qo, int &status, int dead_in = 0, int *dead_out = nullptr) {
    const int n = c.n;
    int phase = start_phase;
    int K = o.K;
    int gr_freq = o.gr_freq;
    const int gr_base = o.gr_freq;
    int rm_freq = o.rm_freq;
    int stag = 0, calm = 0;
    i64 last_sum = LLONG_MAX;
    int pp_stable = 0, p_count = 64, pp_iter = 0;
    i64 round = 0;
    i64 mask_arcs = ldcg(&c.st.acc[ACC_TOT + T_MASKARCS]);
    int gr_depth = 0;  // levels of the last global relabel's search
    // dead marks (see global_relabel): phase A only, from the second relabel
    // of the phase on; new ones only after a complete search
    int dead_phase = (dead_in > 0 && start_phase == PH_A && o.gr_stop) ? PH_A : -1;  // phase of the last relabel
    bool last_complete = dead_phase == PH_A && dead_in == 2;
    if (dead_out) *dead_out = 0;
    for (;;) {
        int sinkv = (phase == PH_A) ? t : (phase == PH_B ? -1 : s);
        int blockv = (phase == PH_C) ? t : s;
        bool defseeds = (phase != PH_C);
        int naf = 0, nab = 0, nd = 0;
        i64 *ab = nullptr;
        int *L = c.st.qb, *N = c.st.qa;
        int lbk = c.take_bank();
        u64 t0 = globaltimer_ns();
        i64 a0 = c.w_arcs;
        const bool keep_dead = o.gr_stop && phase == PH_A && dead_phase == PH_A;
        if (!global_relabel(c, nv, M, sinkv, blockv, s, defseeds, L, lbk, naf, nab, nd, ab, gr_depth, o.gr_stop,
                            keep_dead, keep_dead && last_complete, &last_complete))
            return false;
        dead_phase = phase;
        c.tm_relabel += globaltimer_ns() - t0;
        if (c.leader) {
            u64 t1 = globaltimer_ns();
            c.st.acc[ACC_GR_DUR] = (i64)(t1 - t0);
            c.st.acc[ACC_GR_END] = (i64)t1;
        }
        if (c.lane == 0 && c.w_arcs > a0) atomic_add_i64(&c.st.acc[ACC_TOT + T_RARCS], c.w_arcs - a0);
        qo.relabels++;
        if (naf + nab == 0) {
            if (phase == PH_A) {
                if (nd == 0) {
                    if (dead_out && o.gr_stop) *dead_out = last_complete ? 2 : 1;
                    return true;
                }
                phase = PH_B;
                qo.deficit_phases++;
                continue;
            }
            if (phase == PH_B) {
                if (nd == 0) {
                    phase = PH_A;
                    continue;
                }
                status = MFD_INEXACT;
                return true;
            }
            if (nd != 0) status = MFD_INEXACT;
            return true;  // PH_C done
        }
        i64 work_since = 0;
        int rounds_since = 0;
        bool force_gr = false;
        u64 tr0 = globaltimer_ns();
        while (naf + nab > 0) {
            if (round >= o.iter_max) {
                status = MFD_ITER_LIMIT;
                return true;
            }
            // launch time limit: the leader raises the error word; every CTA
            // then leaves at its next group barrier
            if (c.leader && c.time_limit && globaltimer_ns() - c.t_start > c.time_limit)
                atomicCAS(c.err, 0, MFD_TIMEOUT);
            // ---- one discharge round over L -> N
            MF_TRACE(45, (int)round);
            int na = naf + nab;
            unsigned rstamp = ++c.clock;
            int nbk = c.take_bank();
            i64 *rb = c.take_abank();
            if (na > 0 && na <= o.pp_switch) ++pp_stable;
            else {
                pp_stable = 0;
                p_count = 64;
            }
            bool use_pp = o.use_pp && na > 0 && na <= o.pp_switch &&
                          (o.force_pp || pp_stable >= p_count);
            // round-start counts over L (RA:1738-1763): active-high, sum of excess, band
            i64 l_sum = 0, l_high = 0;
            int l_hmin = INT_MAX, l_hmax = -1;
            for (int i = c.gw * 32 + c.lane; i < na; i += c.gW * 32) {
                int v = i < naf ? ldcg(&L[i]) : back_at(c, L, i - naf);
                i64 ev = ldcg(&c.st.ex[v]);
                int hv = ldcg(&c.st.h[v]);
                if (ev > 0 && hv < n) {
                    l_sum += ev;
                    l_high += (hv > o.h_cut);
                    l_hmin = min(l_hmin, hv);
                    l_hmax = max(l_hmax, hv);
                }
            }
            l_sum = warp_sum_i64(l_sum);
            l_high = warp_sum_i64(l_high);
            l_hmin = __reduce_min_sync(MF_FULL, l_hmin);
            l_hmax = __reduce_max_sync(MF_FULL, l_hmax);
            if (c.lane == 0) {
                if (l_sum) atomic_add_i64(&rb[A_SUMEX], l_sum);
                if (l_high) atomic_add_i64(&rb[A_HIGH], l_high);
                if (l_hmin != INT_MAX) atomicMin(reinterpret_cast<long long *>(&rb[A_HMIN]), (long long)l_hmin);
                if (l_hmax >= 0) atomicMax(reinterpret_cast<long long *>(&rb[A_HMAX]), (long long)l_hmax);
            }
            if (use_pp) {
                unsigned pstamp = ++c.clock;
                for (int i = c.gw; i < na; i += c.gW) {
                    int v = i < naf ? ldcg(&L[i]) : back_at(c, L, i - naf);
                    path_push_vertex(c, v, o.max_path, sinkv, blockv, N, nbk, rstamp, pstamp, rb);
                }
                pp_stable = 0;
                if (++pp_iter >= 4) {
                    pp_iter = 0;
                    p_count = 2;
                }
                qo.pp_rounds++;
            } else {
                if (nab > 0 && !hub_setup(c, L, nab, nullptr)) return false;
                discharge_front(c, L, naf, K, sinkv, blockv, N, nbk, rstamp, rb, nullptr);
                if (nab > 0) discharge_hubs(c, L, nab, sinkv, blockv, N, nbk, rstamp, rb);
            }
            // clear region scratch for this round's optional passes
            {
                int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
                for (int r = gt; r < c.R; r += gT) {
                    c.st.hot[r] = 0;
                    c.st.ract[r] = 0;
                }
            }
            MF_TRACE(46, (int)round);
            if (c.leader) rb[A_TIME] = (i64)globaltimer_ns();
            int nNf = 0, nNb = 0;
            if (!c.sync_tails(nbk, nNf, nNb)) return false;
            MF_TRACE(47, (int)round);
            i64 sum = ldcg(&rb[A_SUMEX]);
            i64 high = ldcg(&rb[A_HIGH]);
            int hmin = (int)ldcg(&rb[A_HMIN]), hmax = (int)ldcg(&rb[A_HMAX]);
            i64 work_round = ldcg(&rb[A_WORK]);
            work_since += work_round;
            ++round;
            ++rounds_since;
            qo.rounds = round;
            float frac_high = (na > 0) ? (float)high / (float)na : 0.0f;
            if (frac_high > 0.8f && (round % 2048) == 0) force_gr = true;
            // stagnation control (RA:1860-1891)
            bool hotspot = false;
            if (last_sum != LLONG_MAX) {
                if (sum >= last_sum) ++stag;
                else stag = 0;
            }
            last_sum = sum;
            if (stag >= o.stagnate && !use_pp) {
                hotspot = true;
                force_gr = true;
                stag = 0;
                gr_freq = min(2 * gr_base, gr_freq * 2);
                K = min(max(16, 2 * o.K), K * 2);
                calm = 0;
            } else if (++calm >= o.stagnate) {
                gr_freq = max(gr_base, gr_freq / 2);
                K = max(o.K, K / 2);
                calm = 0;
            }
            // hot-region extra sweep over the next worklist (RA:1899-1984)
            if (o.use_hot && !use_pp && !hotspot && nNf + nNb >= 64 && (round % 2) == 1 && c.R > 1) {
                if (!select_hot(c, N, nNf, nNb, o.hot_k)) return false;
                if (nNb > 0 && !hub_setup(c, N, nNb, c.st.hot)) return false;
                discharge_front(c, N, nNf, K, sinkv, blockv, N, nbk, rstamp, rb, c.st.hot);
                if (nNb > 0) discharge_hubs(c, N, nNb, sinkv, blockv, N, nbk, rstamp, rb);
                if (!c.sync_tails(nbk, nNf, nNb)) return false;
                work_since += ldcg(&rb[A_WORK]) - work_round;
                qo.hot_sweeps++;
            }
            // RM (RA:1991-2097)
            bool do_rm = o.use_rm && o.local_rl == 0 && start_phase != PH_C && nNf + nNb > 0 &&
                         (round % rm_freq) == 0 &&
                         (o.force_rm || frac_high >= 0.5f);
            if (do_rm) {
                int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
                for (int i = gt; i < nNf + nNb; i += gT) {
                    int v = i < nNf ? ldcg(&N[i]) : back_at(c, N, i - nNf);
                    c.st.ract[ldro(&c.rof[v])] = 1;
                }
                if (!c.sync()) return false;
                int hlo = max(0, (hmin == INT_MAX ? 0 : hmin) - 4);
                int hhi = min(n - 1, (hmax < 0 ? n - 1 : hmax) + 4);
                if (!rm_pass(c, nv, M, hlo, hhi, s, t, N, nbk, rstamp, rb)) return false;
                nNf = ldcg(&c.st.cnt[nbk]);
                nNb = ldcg(&c.st.cnt[CNT_BACK + nbk]);
                i64 fixed = ldcg(&rb[A_FIXED]);
                qo.rm_fixed += fixed;
                double frac_fix = (double)fixed / (double)max((i64)1, mask_arcs);
                if (frac_fix < 1e-5) rm_freq = min(rm_freq * 2, 256);
                else rm_freq = max(o.rm_freq, rm_freq / 2);
                if (fixed) force_gr = true;  // deficits are relabel seeds
            }
            // next round
            int *tmp = L;
            L = N;
            N = tmp;
            naf = nNf;
            nab = nNb;
            // relabel when forced (stagnation, deficits), after alpha x kept
            // arcs of scanning, or after gr_freq rounds.  After a deep relabel
            // (more than DEEP_LEVELS levels: long thin residual paths, where
            // each level is a barrier and the rounds that move excess along
            // the path are quick) none of these fires before the rounds have
            // taken as long as that relabel, or the solve would spend far
            // more time searching than pushing; the relabel that ends a phase
            // (no active vertex left) is never held.  gr_freq = 1 asks for a
            // relabel after every round.  The times are the leader's,
            // published before barriers, so every thread decides alike.
            const i64 since_gr = ldcg(&rb[A_TIME]) - ldcg(&c.st.acc[ACC_GR_END]);
            const bool deep_hold = o.gr_freq > 1 && gr_depth > DEEP_LEVELS &&
                                   since_gr < ldcg(&c.st.acc[ACC_GR_DUR]);
            bool gr_due = !deep_hold &&
                          (force_gr || rounds_since >= gr_freq ||
                           (o.gr_alpha > 0.0 && (double)work_since >= o.gr_alpha * (double)mask_arcs));
            if (gr_due) break;
            // local relabel between global ones (RA:1583-1720), every
            // local_rl-th round, when this round's active heights spanned at
            // most LR_BAND levels
            if (o.local_rl > 0 && naf + nab > 0 && (rounds_since % o.local_rl) == 0 && hmax >= hmin &&
                hmax - hmin < LR_BAND) {
                const u64 tl0 = globaltimer_ns();
                const i64 la0 = c.w_arcs;
                int ldepth = 0;
                if (!local_relabel(c, nv, sinkv, blockv, s, defseeds, L, naf, nab, N, hmax - hmin + 1, ldepth))
                    return false;
                last_complete = false;
                qo.local_relabels++;
                const u64 dl = globaltimer_ns() - tl0;
                c.tm_relabel += dl;
                tr0 += dl;  // rounds time excludes it
                if (c.lane == 0 && c.w_arcs > la0) atomic_add_i64(&c.st.acc[ACC_TOT + T_RARCS], c.w_arcs - la0);
            }
        }
        c.tm_rounds += globaltimer_ns() - tr0;
        // relabel (either nothing is active -> exact termination check, or due)
    }
}

// ---------------------------------------------------------------------------
// Certificate (after phase C): zero excess off {s,t}; residuals >= 0 and
// pairwise conserved on kept arcs; T = vertices reaching t in the full-graph
// residual (kept arcs: res; other arcs: cap); s not in T; capacity of
// (V\T -> T) == flow.  Uses qmark as the full-graph BFS stamp.
__device__ bool certify(QCtx &c, int s, int t, int nv, unsigned M, i64 flow, QOut &qo, int &status) {
    i64 *ab = c.take_abank();
    i64 bad = 0;
    auto arc_ok = [&](int e) -> int {
        int w = ldro(&c.col[e]);
        i64 r = ldcg(&c.st.res[e]);
        int nb = r < 0;
        if (ldcg(&c.st.mark[w]) >= M) {
            int re = ldro(&c.rev[e]);
            if (r + ldcg(&c.st.res[re]) != ldcap(&c.cap[e]) + ldcap(&c.cap[re])) ++nb;
        }
        return nb;
    };
    for (int i = c.gw; i < nv; i += c.gW) {
        int v = c.vat(i);
        if (c.lane == 0 && v != s && v != t && ldcg(&c.st.ex[v]) != 0) ++bad;
        int b = ldro(&c.row[v]), e1 = ldro(&c.row[v + 1]);
        if (c.giant(b, e1)) continue;
        for (int e = b + c.lane; e < e1; e += 32) bad += arc_ok(e);
    }
    for_giants(
        c, [&](int v) { return ldcg(&c.st.mark[v]) >= M; }, [&](int, int, int) {},
        [&](int, int e) { bad += arc_ok(e); });
    bad = warp_sum_i64(bad);
    if (c.lane == 0 && bad) atomic_add_i64(&ab[A_BAD], bad);
    // full-graph backward BFS from t
    unsigned Z = ++c.clock;
    int bk = c.take_bank();
    if (c.leader) {
        c.st.qmark[t] = Z;
        append1(c, t, c.st.qa, bk);
    }
    int f0 = 0, b0 = 0;
    if (!c.sync_tails(bk, f0, b0)) return false;
    unsigned *qm = c.st.qmark, *mark = c.st.mark;
    const int *rev = c.rev;
    const i64 *cap = c.cap;
    i64 *res = c.st.res;
    auto cut_bfs = [&](int v, int e, int w, int) -> bool {
        if (ldcg(&qm[w]) == Z) return false;
        int re = ldro(&rev[e]);  // arc w->v
        bool kept = ldcg(&mark[w]) >= M && ldcg(&mark[v]) >= M;
        i64 r = kept ? ldcg(&res[re]) : ldcap(&cap[re]);
        if (r <= 0) return false;
        return atomicMax(&qm[w], Z) < Z;
    };
    if (!bfs_levels(c, c.st.qa, bk, f0, b0, cut_bfs)) return false;
    // cut capacity over all vertices
    i64 cut = 0;
    auto cut_arc = [&](int e) -> i64 {
        i64 cp = ldcap(&cap[e]);
        return (cp > 0 && ldcg(&qm[ldro(&c.col[e])]) == Z) ? cp : 0;
    };
    for (int v = c.gw; v < c.n; v += c.gW) {
        if (ldcg(&qm[v]) == Z) continue;
        int b = ldro(&c.row[v]), e1 = ldro(&c.row[v + 1]);
        if (c.giant(b, e1)) continue;
        for (int e = b + c.lane; e < e1; e += 32) cut += cut_arc(e);
    }
    for_giants(
        c, [&](int v) { return ldcg(&qm[v]) != Z; }, [&](int, int, int) {}, [&](int, int e) { cut += cut_arc(e); });
    cut = warp_sum_i64(cut);
    if (c.lane == 0 && cut) atomic_add_i64(&ab[A_CUT], cut);
    if (!c.sync()) return false;
    i64 total_bad = ldcg(&ab[A_BAD]);
    i64 cutv = ldcg(&ab[A_CUT]);
    bool s_in_t = ldcg(&qm[s]) == Z;
    qo.cut = cutv;
    if (total_bad != 0 || s_in_t || cutv != flow) status = MFD_CERTIFY;
    return true;
}

// Full-graph residuals for host-side certification: kept arcs res, others cap.
__device__ bool write_full_residual(QCtx &c, unsigned M, i64 *out) {
    for (int v = c.gw; v < c.n; v += c.gW) {
        bool kv = ldcg(&c.st.mark[v]) >= M;
        int b = ldro(&c.row[v]), e1 = ldro(&c.row[v + 1]);
        if (c.giant(b, e1)) continue;
        for (int e = b + c.lane; e < e1; e += 32) {
            int w = ldro(&c.col[e]);
            bool kept = kv && ldcg(&c.st.mark[w]) >= M;
            out[e] = kept ? ldcg(&c.st.res[e]) : ldcap(&c.cap[e]);
        }
    }
    for_giants(
        c, [&](int) { return true; }, [&](int, int, int) {},
        [&](int v, int e) {
            bool kept = ldcg(&c.st.mark[v]) >= M && ldcg(&c.st.mark[ldro(&c.col[e])]) >= M;
            out[e] = kept ? ldcg(&c.st.res[e]) : ldcap(&c.cap[e]);
        });
    return c.sync();
}

// ---------------------------------------------------------------------------
// Warm start after capacity updates (mode KM_REPAIR).  The slot keeps the
// previous solve's residual, excess and kept set (meta: M_old, nv_old,
// vf_old).  1. old kept vertices get claim stamp O; 2. re-prune on the new
// capacities; new kept = old kept U new prune; 3. vertices new to the kept
// set get fresh state and their arc pairs with kept vertices are reopened;
// 4. each updated arc inside the kept set adjusts its residual, cancelling
// flow above the new capacity (tail gains excess, head loses it); 5. s
// re-saturates.
__device__ bool repair_deltas(QCtx &c, const KParams &p, unsigned Mn, unsigned O);

// dead_in (out): the dead-mark state the repaired solve may start from.
// The previous solve left meta[7] (see run_phases): its dead vertices (and,
// with 2, the kept vertices its last, complete search did not reach) could
// reach neither the sink nor a deficit.  A vertex's residual reach grows
// only through an arc whose residual goes from 0 to positive, and a new
// deficit appears only where flow is cancelled; when no update of the batch
// on the kept arcs does either, those vertices still reach neither (the
// repair's preflow only opens arcs into the source, which phase A never
// crosses), so the marks carry over and the first relabel need not search
// for them.  Otherwise, and after a re-prune, the solve starts clean.
__device__ bool repair(QCtx &c, const KParams &p, int s, int t, unsigned &M, int &nv, bool &t_reach,
                       int &dead_in) {
    dead_in = 0;
    int *meta = c.st.meta;
    int vf_old = ldcg(&meta[4]);
    int nv_old = ldcg(&meta[1]);
    c.vf = vf_old;
    unsigned O = ++c.clock;
    for (int i = c.crank * blockDim.x + threadIdx.x; i < nv_old; i += c.G * blockDim.x)
        c.st.claim[c.vat(i)] = O;
    if (!c.sync()) return false;
    unsigned S = ++c.clock;
    unsigned Mn = ++c.clock;
    unsigned *mark = c.st.mark, *claim = c.st.claim;
    const i64 *cap = c.cap;
    const int *rev = c.rev;
    // The kept set fwd(s) & bwd(t) follows arcs with capacity > 0, so it can
    // only grow through an arc whose capacity went from 0 to positive.  With
    // no such update the old kept set is a superset of the new one, which
    // gives the same maximum flow (every s-t path lies inside the new set):
    // it is kept as it is and both searches are skipped.
    int gt0 = c.crank * blockDim.x + threadIdx.x, gT0 = c.G * blockDim.x;
    if (c.leader) c.st.cnt[CNT_FLAG] = 0;
    if (!c.sync()) return false;
    for (int i = gt0; i < p.nupd; i += gT0)
        if (p.upd[i].old_cap <= 0 && p.upd[i].new_cap > 0) atomicOr(&c.st.cnt[CNT_FLAG], 1);
    if (!c.sync()) return false;
    const bool grows = ldcg(&c.st.cnt[CNT_FLAG]) != 0;
    if (!grows) {
        for (int i = gt0; i < nv_old; i += gT0) mark[c.vat(i)] = Mn;
        t_reach = ldcg(&meta[5]) != 0;
        nv = nv_old;
        if (c.leader) c.st.acc[ACC_TOT + T_MASKARCS] = ldcg(&meta[6]);
        if (c.leader) c.st.cnt[CNT_OPENED] = 0;
        if (!c.sync()) return false;
        if (!repair_deltas(c, p, Mn, O)) return false;
        if (ldcg(&c.st.cnt[CNT_OPENED]) == 0) dead_in = ldcg(&meta[7]);
        M = Mn;
        if (!t_reach) return true;
        return preflow(c, s);
    }
    // the kept set under the new capacities, fwd(s) & bwd(t), by two
    // direction-optimizing searches (a top-down-only pair examined every
    // arc of fwd(s) twice: ~270 M arcs for a hub query on R-MAT 2^22)
    int bank = c.take_bank();
    if (!reach_all(c, s, 0, mark, S, c.st.qa, bank)) return false;
    const int nff = ldcg(&c.st.cnt[bank]), nfb = ldcg(&c.st.cnt[CNT_BACK + bank]);
    t_reach = ldcg(&mark[t]) >= S;
    int nb = c.take_bank();
    int addb = c.take_bank();
    int nbf = 0, nbb = 0;
    if (t_reach) {
        if (c.leader) {
            mark[t] = Mn;
            append1(c, t, c.st.qb, nb);
        }
        int f0 = 0, b0 = 0;
        if (!c.sync_tails(nb, f0, b0)) return false;
        auto bwd = [&](int v, int e, int w, int) -> bool {
            if (ldcg(&mark[w]) != S) return false;
            if (ldcap(&cap[ldro(&rev[e])]) <= 0) return false;
            return atomicCAS(&mark[w], S, Mn) == S;
        };
        // bottom-up candidates: the forward-reached vertices not reached yet
        auto uf = [&](int i) -> int {
            const int w = ldcg(&c.st.qa[i]);
            return ldcg(&mark[w]) == S ? w : -1;
        };
        auto ub = [&](int k) -> int {
            const int w = back_at(c, c.st.qa, k);
            return ldcg(&mark[w]) == S ? w : -1;
        };
        auto par = [&](int w, int e, int y, int) -> bool {
            return ldcg(&mark[y]) == Mn && ldcap(&cap[e]) > 0;  // arc w -> y, y reaches t
        };
        auto set = [&](int w, int) -> bool {
            mark[w] = Mn;
            return true;
        };
        if (!bfs_dir(c, c.st.qb, nb, f0, b0, bwd, nff, uf, nfb, ub, par, set)) return false;
        nbf = ldcg(&c.st.cnt[nb]);
        nbb = ldcg(&c.st.cnt[CNT_BACK + nb]);
    }
    // vertices new to the kept set (bwd-reached, not old) go to the front of
    // vlist after the old front part; the old back part stays where it is
    if (c.leader) c.st.cnt[addb] = vf_old;
    if (!c.sync()) return false;
    int nnew_bfs = nbf + nbb;
    for (int base = c.gw * 32; base < nnew_bfs; base += c.gW * 32) {
        int i = base + c.lane;
        bool add = false;
        int v = 0;
        if (i < nnew_bfs) {
            v = ldcg(i < nbf ? &c.st.qb[i] : &c.st.qb[c.n - 1 - (i - nbf)]);
            add = ldcg(&claim[v]) != O;
        }
        warp_append(add, v, c.st.vlist, &c.st.cnt[addb], c.n);
    }
    if (!c.sync()) return false;
    int vf_new = ldcg(&c.st.cnt[addb]);
    int nadd = vf_new - vf_old;
    c.vf = vf_new;
    nv = nv_old + nadd;
    // every kept vertex (old and new) gets the current mask stamp
    for (int i = c.crank * blockDim.x + threadIdx.x; i < nv; i += c.G * blockDim.x) mark[c.vat(i)] = Mn;
    if (!c.sync()) return false;
    // fresh state for new vertices; reopen their arc pairs
    i64 add_arcs = 0;
    auto open_arc = [&](int e) {
        int w = ldro(&c.col[e]);
        if (ldcg(&mark[w]) == Mn) {
            c.st.res[e] = ldcap(&cap[e]);
            if (ldcg(&claim[w]) == O) {
                int re = ldro(&rev[e]);
                c.st.res[re] = ldcap(&cap[re]);
            }
        } else {
            c.st.res[e] = 0;
        }
    };
    for (int i = vf_old + c.gw; i < vf_new; i += c.gW) {
        int v = ldcg(&c.st.vlist[i]);
        int b = ldro(&c.row[v]), e1 = ldro(&c.row[v + 1]);
        if (c.lane == 0) {
            c.st.ex[v] = 0;
            c.st.h[v] = 0;
        }
        add_arcs += e1 - b;
        if (c.giant(b, e1)) continue;
        for (int e = b + c.lane; e < e1; e += 32) open_arc(e);
    }
    // new giants: kept now (Mn) and not among the old kept vertices (O)
    for_giants(
        c, [&](int v) { return ldcg(&mark[v]) == Mn && ldcg(&claim[v]) != O; }, [&](int, int, int) {},
        [&](int, int e) { open_arc(e); });
    if (c.leader) atomic_add_i64(&c.st.acc[ACC_TOT + T_MASKARCS], ldcg(&meta[6]));
    if (c.lane == 0 && add_arcs) atomic_add_i64(&c.st.acc[ACC_TOT + T_MASKARCS], add_arcs);
    if (!c.sync()) return false;
    if (!repair_deltas(c, p, Mn, O)) return false;
    M = Mn;
    if (!t_reach) return true;
    return preflow(c, s);
}

// Capacity deltas on kept arcs (forward arcs of changed edges) whose ends
// were both kept before (claim O) and are kept now (mark Mn): a rise adds
// residual; a fall below the arc's flow cancels the excess flow, leaving
// the surplus as excess at the tail and a deficit at the head.
__device__ bool repair_deltas(QCtx &c, const KParams &p, unsigned Mn, unsigned O) {
    unsigned *mark = c.st.mark, *claim = c.st.claim;
    const int *rev = c.rev;
    int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
    for (int i = gt; i < p.nupd; i += gT) {
        ArcUpdate u = p.upd[i];
        int e = u.arc;
        int re = ldro(&rev[e]);
        int w = ldro(&c.col[e]);
        int x = ldro(&c.col[re]);  // tail of e
        if (ldcg(&mark[w]) != Mn || ldcg(&mark[x]) != Mn) continue;
        // arc e (x->w) carries flow f = old_cap - res[e] on its pair
        // (its partner is a zero-capacity reverse arc).  Arcs that were
        // opened in step 3 already hold the new capacity.
        if (ldcg(&claim[x]) != O || ldcg(&claim[w]) != O) continue;
        i64 r = ldcg(&c.st.res[e]);
        i64 f = u.old_cap - r;
        if (f <= u.new_cap) {
            atomic_add_i64(&c.st.res[e], u.new_cap - u.old_cap);
            if (r <= 0 && u.new_cap > u.old_cap) atomicOr(&c.st.cnt[CNT_OPENED], 1);  // x -> w opened
        } else {
            atomicOr(&c.st.cnt[CNT_OPENED], 1);  // flow cancelled: a deficit at w
            i64 over = f - u.new_cap;
            atomic_add_i64(&c.st.res[e], -r);
            atomic_add_i64(&c.st.res[re], -over);
            atomic_add_i64(&c.st.ex[x], over);
            atomic_add_i64(&c.st.ex[w], -over);
        }
    }
    return c.sync();
}

// ---------------------------------------------------------------------------
__device__ void solve_query(QCtx &c, const KParams &p, int q, int s, int t) {
    MF_TRACE(2, q);
    QOut qo = {};
    int status = MFD_OK;
    const KOpts &o = p.o;
    if (c.leader) {
        for (int i = 0; i < NBANKS; ++i) {
            c.st.cnt[i] = 0;
            c.st.cnt[CNT_BACK + i] = 0;
        }
        for (int i = 0; i < 4 * ACC_BANK; ++i) c.st.acc[i] = 0;
        for (int b = 0; b < 4; ++b) {
            c.st.acc[b * ACC_BANK + A_HMIN] = INT_MAX;
            c.st.acc[b * ACC_BANK + A_HMAX] = -1;
        }
        for (int i = 0; i < 16; ++i) c.st.acc[ACC_TOT + i] = 0;
    }
    c.seq = 0;
    c.aseq = 0;
    c.vf = 0;
    c.tm_relabel = c.tm_rounds = 0;
    if (!c.sync()) return;
    unsigned M = 0;
    int nv = 0;
    bool t_reach = false;
    int dead_in = 0, dead_out = 0;  // dead-mark state carried between warm starts (run_phases)
    if (p.mode == KM_REPAIR) {
        if (!repair(c, p, s, t, M, nv, t_reach, dead_in)) return;
    } else {
        unsigned S = ++c.clock;
        M = ++c.clock;
        const DGraph &g = *c.gr;
        // kc_case 1: s and t in the cached component; 2: s in B, t in F
        const bool use_kc = p.mode != KM_KEPTSET && o.prune_mode == 1 && o.use_cache && g.kc_in && !c.no_cache;
        int kc_case = 0;
        if (use_kc) {
            if (ldro_u8(&g.kc_in[s]) && ldro_u8(&g.kc_in[t])) kc_case = 1;
            else if (g.kc_fb && (ldro_u8(&g.kc_fb[s]) & KC_B) && (ldro_u8(&g.kc_fb[t]) & KC_F)) kc_case = 2;
        }
        if (kc_case == 1) {
            // s and t lie in the cached component: it is the kept set
            nv = g.kc_f + g.kc_b;
            c.vf = g.kc_f;
            t_reach = true;
            int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
            for (int i = gt; i < nv; i += gT) {
                int pos = i < g.kc_f ? i : c.n - 1 - (i - g.kc_f);
                int v = ldro(&g.kc_img[pos]);
                c.st.vlist[pos] = v;
                c.st.mark[v] = M;
                c.st.ex[v] = 0;
                c.st.h[v] = 0;
            }
            if (c.leader) c.st.acc[ACC_TOT + T_MASKARCS] = g.kc_arcs;
            if (!c.sync()) return;
        } else if (kc_case == 2) {
            if (!prune_ext(c, s, t, S, M, nv)) return;
            t_reach = true;
        } else if (o.prune_mode == 2) {
            // no prune: every vertex is kept.  The kept set only has to
            // contain fwd(s) & bwd(t); where the terminals touch most of the
            // graph (segmentation grids) the two searches cost more than the
            // few extra vertices, which no push reaches or no relabel labels
            int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
            for (int v = gt; v < c.n; v += gT) {
                c.st.vlist[v] = v;
                c.st.mark[v] = M;
            }
            nv = c.n;
            c.vf = c.n;
            t_reach = true;
            if (!c.sync()) return;
        } else if (!prune(c, s, t, o.prune_mode, S, M, nv, t_reach, use_kc ? g.kc_fb : nullptr)) {
            return;
        }
        if (p.mode == KM_KEPTSET) {
            KcOut *ko = (KcOut *)p.dbg;
            int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
            for (int i = gt; i < nv; i += gT) {
                int pos = i < c.vf ? i : c.n - 1 - (i - c.vf);
                int v = ldcg(&c.st.vlist[pos]);
                ko->img[pos] = v;
                ko->in[v] = 1;
            }
            // closures of the pivot: F = forward-reached (stamp S or M),
            // B = a backward search on qmark
            int bb = c.take_bank();
            if (!reach_all(c, s, 1, c.st.qmark, S, c.st.qb, bb)) return;
            for (int v = gt; v < c.n; v += gT)
                ko->fb[v] = (ldcg(&c.st.mark[v]) >= S ? KC_F : 0) | (ldcg(&c.st.qmark[v]) == S ? KC_B : 0);
            if (c.leader) {
                qo.mask_n = nv;
                qo.kept_front = c.vf;
                p.out[q] = qo;
            }
            c.sync();
            return;
        }
        if (p.mode == KM_PRUNE) {
            unsigned char *mk = (unsigned char *)p.dbg;
            int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
            for (int v = gt; v < c.n; v += gT)
                mk[v] = (ldcg(&c.st.mark[v]) == M || v == s || v == t) ? 1 : 0;
            if (c.leader) {
                qo.mask_n = (o.prune_mode == 1 && !t_reach) ? 2 : nv;
                p.out[q] = qo;
            }
            c.sync();
            return;
        }
        if (t_reach && nv > 0) {
            const int nimg = g.kc_f + g.kc_b;
            if (kc_case == 2 && nv - nimg > nimg) {
                // the extras outnumber the cached component: a fresh init
                // costs less than the image copy plus the extras' fix-up
                // (their arcs are already in the mask-arc total)
                if (!init_state(c, nv, M, false)) return;
            } else if (kc_case) {
                // initial residuals of the component, copied whole (16-byte
                // vectors); ex/h were set with the kept list above
                const longlong2 *src = reinterpret_cast<const longlong2 *>(g.kc_res);
                longlong2 *dst = reinterpret_cast<longlong2 *>(c.st.res);
                i64 A = ldro(&c.row[c.n]);
                i64 nvec = A >> 1;
                int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
                // four independent loads in flight per thread (the arrays
                // may alias as far as the compiler knows, so a plain loop
                // waits out one load latency per vector)
                i64 k = gt;
                for (; k + 3 * (i64)gT < nvec; k += 4 * (i64)gT) {
                    const longlong2 x0 = __ldg(&src[k]), x1 = __ldg(&src[k + gT]);
                    const longlong2 x2 = __ldg(&src[k + 2 * (i64)gT]), x3 = __ldg(&src[k + 3 * (i64)gT]);
                    dst[k] = x0;
                    dst[k + gT] = x1;
                    dst[k + 2 * (i64)gT] = x2;
                    dst[k + 3 * (i64)gT] = x3;
                }
                for (; k < nvec; k += gT) dst[k] = __ldg(&src[k]);
                if (gt == 0 && (A & 1)) c.st.res[A - 1] = ldro(&g.kc_res[A - 1]);
                if (c.lane == 0 && c.gw == 0) c.w_verts += nv;
                if (!c.sync()) return;
                if (kc_case == 2 && !fix_extra_arcs(c, M, nv)) return;
            } else if (o.prune_mode == 2 && nv == c.n) {
                // every vertex kept: the initial residuals are the
                // capacities, copied whole like the cached image (no per-arc
                // test of the head)
                const i64 A = ldro(&c.row[c.n]);
                int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
                for (int v = gt; v < c.n; v += gT) {
                    c.st.ex[v] = 0;
                    c.st.h[v] = 0;
                }
                const bool vec = ((reinterpret_cast<uintptr_t>(c.cap) | reinterpret_cast<uintptr_t>(c.st.res)) & 15) == 0;
                const i64 nvec = vec ? (A >> 1) : 0;
                const longlong2 *src = reinterpret_cast<const longlong2 *>(c.cap);
                longlong2 *dst = reinterpret_cast<longlong2 *>(c.st.res);
                i64 k = gt;
                for (; k + 3 * (i64)gT < nvec; k += 4 * (i64)gT) {
                    const longlong2 x0 = ldcap2(&src[k]), x1 = ldcap2(&src[k + gT]);
                    const longlong2 x2 = ldcap2(&src[k + 2 * (i64)gT]), x3 = ldcap2(&src[k + 3 * (i64)gT]);
                    dst[k] = x0;
                    dst[k + gT] = x1;
                    dst[k + 2 * (i64)gT] = x2;
                    dst[k + 3 * (i64)gT] = x3;
                }
                for (; k < nvec; k += gT) dst[k] = ldcap2(&src[k]);
                for (i64 e = 2 * nvec + gt; e < A; e += gT) c.st.res[e] = ldcap(&c.cap[e]);
                if (c.leader) c.st.acc[ACC_TOT + T_MASKARCS] = A;
                if (c.lane == 0 && c.gw == 0) c.w_verts += nv;
                if (!c.sync()) return;
            } else if (!init_state(c, nv, M)) {
                return;
            }
            if (p.ov_arc && !apply_overrides(c, p, q, M)) return;
            if (!preflow(c, s)) return;
        }
    }
    i64 flow = 0;
    u64 t_pruned = globaltimer_ns();
    if (t_reach && nv > 0) {
        if (!build_kept_bits(c, M)) return;
        if (p.mode == KM_HEIGHTS) {
            int naf = 0, nab = 0, nd = 0;
            i64 *ab = nullptr;
            int lbk = c.take_bank();
            int depth = 0;
            if (!global_relabel(c, nv, M, t, s, s, true, c.st.qb, lbk, naf, nab, nd, ab, depth, false)) return;
            int *hd = (int *)p.dbg;
            int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
            for (int v = gt; v < c.n; v += gT)
                hd[v] = (ldcg(&c.st.mark[v]) >= M) ? ldcg(&c.st.h[v]) : c.n;
            if (!c.sync()) return;
        } else {
            if (!run_phases(c, o, s, t, nv, M, PH_A, qo, status, dead_in, &dead_out)) return;
            flow = ldcg(&c.st.ex[t]);
            if (p.mode == KM_CERTIFY && status == MFD_OK) {
                dead_out = 0;
                if (!run_phases(c, o, s, t, nv, M, PH_C, qo, status)) return;
                if (status == MFD_OK && !certify(c, s, t, nv, M, flow, qo, status)) return;
            }
        }
    } else if (p.mode == KM_HEIGHTS) {
        int *hd = (int *)p.dbg;
        int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
        for (int v = gt; v < c.n; v += gT) hd[v] = c.n;
        if (!c.sync()) return;
    }
    if (p.mode == KM_RESIDUAL) {
        if (t_reach && nv > 0) {
            if (!write_full_residual(c, M, (i64 *)p.dbg)) return;
        } else {
            i64 *out = (i64 *)p.dbg;
            int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
            for (i64 e = gt; e < (i64)ldro(&c.row[c.n]); e += gT) out[e] = ldcap(&c.cap[e]);
            if (!c.sync()) return;
        }
    }
    MF_TRACE(90, q);
    c.flush_warp_counts();
    if (!c.sync()) return;
    if (c.leader) {
        i64 *tot = c.st.acc + ACC_TOT;
        qo.flow = flow;
        qo.status = status;
        qo.mask_n = nv;
        qo.mask_arcs = tot[T_MASKARCS];
        qo.arcs_ex = tot[T_ARCS];
        qo.verts_ex = tot[T_VERTS];
        qo.pushes = tot[T_PUSH];
        qo.t_begin = c.q_begin;
        qo.t_done = globaltimer_ns();
        qo.t_prune = t_pruned - c.q_begin;
        qo.t_relabel = c.tm_relabel;
        qo.t_rounds = c.tm_rounds;
        qo.arcs_relabel = tot[T_RARCS];
        qo.arcs_hubs = tot[T_HARCS];
        qo.hub_passes = tot[T_HPASS];
        qo.hub_relabels = tot[T_HREL];
        qo.levels = tot[T_LEVELS];
        qo.levels_bottom_up = tot[T_BU];
        qo.levels_solo = tot[T_SOLO];
        p.out[q] = qo;
        c.st.meta[0] = (int)M;
        c.st.meta[1] = nv;
        c.st.meta[2] = s;
        c.st.meta[3] = t;
        c.st.meta[4] = c.vf;
        c.st.meta[5] = t_reach ? 1 : 0;
        c.st.meta[6] = (int)min(tot[T_MASKARCS], (i64)INT_MAX);
        c.st.meta[7] = status == MFD_OK ? dead_out : 0;
    }
    c.sync();
}

// Points the context at graph gi (its CSR, giants, kept-set cache).
__device__ __forceinline__ void bind_graph(QCtx &c, const KParams &p, int gi) {
    const DGraph &g = p.graphs[gi];
    c.n = g.n;
    c.R = g.R;
    c.row = g.row;
    c.col = g.col;
    c.rev = g.rev;
    c.rof = g.region_of;
    c.cap = g.cap;
    c.gr = &p.graphs[gi];
    c.giants = g.giants;
    c.ngiant = g.giants ? g.ngiant : 0;
}

#ifdef MF_SERVE_TU
// ---------------------------------------------------------------------------
// Serving loop (KParams::ring_tail != NULL).  Each group owns the slot the
// host published for it in slot_tab (a group still without one is parked
// until the host admits another slot, or until no group is serving), then
// claims requests in ticket order from a shared 64-bit counter.
//
// Ordering.  A query on graph g waits until the update batches submitted
// before it on g are applied (GState::epoch); an update batch waits until
// every query submitted before it on g has finished (GState::done_q) and the
// batches before it are applied.  Every wait is for a smaller ticket, and
// tickets are claimed in order, so the smallest unfinished ticket never
// waits: no wait can close a cycle.  Every wait is also bounded in time.
//
// A group that leaves while holding a claimed ticket not yet submitted gives
// it back (compare-and-swap of the counter from k+1 to k, possible once the
// groups that claimed after it have given theirs back), so a relaunch
// resumes at the first unclaimed ticket and no ticket is lost or run twice.

// Zero everything in the slot but the residuals (stamps, clock, lists,
// control words, bitmaps): a new slot's memory is uninitialized, and a slot
// whose stamp clock nears 2^31 is reset the same way.
__device__ bool srv_clear_slot(QCtx &c, const DSlot &sl, int n) {
    char *b = reinterpret_cast<char *>(sl.ex);
    char *e = reinterpret_cast<char *>(sl.bits + 5 * (size_t)bitmap_words(n));
    // the slot layout aligns every array to 256 bytes, so rounding the end up
    // to 16 bytes stays inside the slot
    const size_t words = ((size_t)(e - b) + 15) >> 4;
    int4 *w = reinterpret_cast<int4 *>(b);
    const int gt = c.crank * blockDim.x + threadIdx.x, gT = c.G * blockDim.x;
    for (size_t k = gt; k < words; k += gT) w[k] = make_int4(0, 0, 0, 0);
    __threadfence();
    return c.sync();
}

// Leader: wait until *word >= want (a bounded wait; false on timeout or a
// raised error word).
__device__ bool srv_wait_ge(const KParams &p, const int *word, int want) {
    const u64 t0 = globaltimer_ns();
    unsigned spins = 0;
    while (*(volatile const int *)word < want) {
        if (*(volatile int *)p.err) return false;
        __nanosleep(1000);
        if ((++spins & 63u) == 0 && globaltimer_ns() - t0 > p.bar_limit_ns) {
            atomicCAS(p.err, 0, MFD_TIMEOUT);
            return false;
        }
    }
    __threadfence();
    return true;
}

// One capacity-update batch, a warp per entry: resolve u -> v to its first
// forward arc (the shorter of the two arc lists is scanned, as in the
// host-side resolution), then cap = max(a, cap + b).  Entries name distinct
// (u, v) pairs, so no two warps write one arc.
__device__ bool srv_apply_updates(QCtx &c, const KParams &p, int gi, long long off, int nu) {
    const DGraph &g = p.graphs[gi];
    i64 *cap = const_cast<i64 *>(g.cap);
    for (int i = c.gw; i < nu; i += c.gW) {
        const UpdEntry *up = p.srv_upd + off + i;
        const int x = *(volatile const int *)&up->u, y = *(volatile const int *)&up->v;
        const i64 ua = *(volatile const i64 *)&up->a, ub = *(volatile const i64 *)&up->b;
        if (x < 0 || y < 0 || x >= g.n || y >= g.n) continue;
        const bool by_head = ldro(&g.row[y + 1]) - ldro(&g.row[y]) < ldro(&g.row[x + 1]) - ldro(&g.row[x]);
        const int w = by_head ? y : x, other = by_head ? x : y;
        const int b = ldro(&g.row[w]), e1 = ldro(&g.row[w + 1]);
        int a = INT_MAX;
        for (int eb = b; eb < e1; eb += 32) {
            const int e = eb + c.lane;
            int cand = INT_MAX;
            if (e < e1 && ldro(&g.col[e]) == other && (ldro_u8(&g.fwd[e]) != 0) != by_head)
                cand = by_head ? ldro(&g.rev[e]) : e;
            const int m = __reduce_min_sync(MF_FULL, cand);
            if (m != INT_MAX) {
                a = m;
                break;
            }
        }
        if (a != INT_MAX && c.lane == 0) {
            const i64 cur = ldcap(&cap[a]);
            cap[a] = max(ua, cur + ub);
        }
    }
    __threadfence();
    return c.sync();
}

__device__ void serve_loop(QCtx &c, const KParams &p, int gid) {
    GroupCtl *gc = p.gctl + gid;
    c.bar = &gc->bar;
    const unsigned long long NONE = ~0ull;
    // ---- wait for a slot
    if (c.leader) {
        int r = 0;
        unsigned spins = 0;
        u64 idle_since = 0;  // first time no group was seen serving (0: one was)
        for (;;) {
            r = p.slot_ready[gid];
            if (r > 0) break;
            if (*p.ring_stop) {
                r = -1;
                break;
            }
            __nanosleep(4000);
            if ((++spins & 15u) == 0) {
                // nobody serving for a millisecond: the launch is ending
                if (ldcg(&p.srv->live) > 0) {
                    idle_since = 0;
                } else {
                    const u64 now = globaltimer_ns();
                    if (!idle_since) idle_since = now;
                    else if (now - idle_since > 1000000ull) {
                        r = -1;
                        break;
                    }
                }
            }
        }
        if (r > 0) {
            __threadfence_system();
            const volatile unsigned *src = reinterpret_cast<const volatile unsigned *>(&p.slot_tab[gid]);
            unsigned *dst = reinterpret_cast<unsigned *>(&gc->slot);
            for (int i = 0; i < (int)(sizeof(DSlot) / 4); ++i) dst[i] = src[i];
            atomicAdd(&p.srv->live, 1);
        }
        gc->w[0] = r;
        __threadfence();
    }
    if (!gsync(c.G, c.bar, c.err, c.lim)) return;
    const int ready = ldcg(&gc->w[0]);
    if (ready < 0) return;
    c.st = gc->slot;
    if (ready == 1) {
        if (!srv_clear_slot(c, c.st, p.slot_n)) return;
        if (c.leader) {
            __threadfence_system();
            p.slot_ready[gid] = 2;
        }
    }
    c.clock = ldcg(c.st.clock);
    c.no_cache = false;
    for (;;) {
        // ---- claim the next ticket (leader), broadcast through gctl
        if (c.leader) {
            unsigned long long q = NONE;
            if (!*p.ring_stop) {
                q = atomicAdd(&p.srv->next, 1ull);
                const u64 t0 = globaltimer_ns();
                unsigned spins = 0;
                for (;;) {
                    if (q < *p.ring_tail) break;
                    const bool leave = *p.ring_stop || globaltimer_ns() - t0 > p.idle_limit_ns;
                    // give the ticket back before leaving; if a later ticket
                    // is claimed, wait until its holder has given it back
                    if (leave && atomicCAS(&p.srv->next, q + 1, q) == q + 1) {
                        q = NONE;
                        break;
                    }
                    __nanosleep(2000);
                    if ((++spins & 1023u) == 0 && globaltimer_ns() - t0 > p.idle_limit_ns + p.bar_limit_ns) {
                        atomicCAS(p.err, 0, MFD_TIMEOUT);
                        q = NONE;
                        break;
                    }
                }
            }
            gc->q = q;
            if (q != NONE) {
                __threadfence_system();
                const int e = (int)(q % (unsigned long long)p.ring_cap);
                const volatile RingReq *rq = reinterpret_cast<const volatile RingReq *>(p.ring_req + e);
                gc->w[0] = rq->kind;
                gc->w[1] = rq->graph;
                gc->w[2] = rq->s;
                gc->w[3] = rq->t;
                gc->w[4] = rq->epoch;
                gc->w[5] = rq->upd_n;
                const long long off = rq->upd_off;
                const unsigned long long need = rq->need_done;
                p.ring_done[e] = 2;
                p.ring_t0[2 * e] = globaltimer_ns();
                // the update waits for the earlier queries on its graph and
                // batches; a query waits for the batches before it
                GState *gs = p.gstate + rq->graph;
                bool ok = true;
                if (gc->w[0] == RQ_UPDATE) {
                    ok = srv_wait_ge(p, &gs->epoch, gc->w[4]);
                    const u64 tw = globaltimer_ns();
                    unsigned sp = 0;
                    while (ok && *(volatile unsigned long long *)&gs->done_q < need) {
                        if (*(volatile int *)p.err) ok = false;
                        __nanosleep(1000);
                        if ((++sp & 63u) == 0 && globaltimer_ns() - tw > p.bar_limit_ns) {
                            atomicCAS(p.err, 0, MFD_TIMEOUT);
                            ok = false;
                        }
                    }
                    __threadfence();
                    *reinterpret_cast<long long *>(&gc->w[6]) = off;
                } else {
                    ok = srv_wait_ge(p, &gs->epoch, gc->w[4]);
                    gc->w[6] = ldcg(&gs->no_cache);
                }
                (void)ok;  // a failed wait has raised the error word
            }
            __threadfence();
        }
        if (!gsync(c.G, c.bar, c.err, c.lim)) return;
        const unsigned long long q = *(volatile unsigned long long *)&gc->q;
        if (q == NONE) break;
        const int e = (int)(q % (unsigned long long)p.ring_cap);
        const int kind = ldcg(&gc->w[0]), gi = ldcg(&gc->w[1]);
        if (kind == RQ_UPDATE) {
            const long long off = __ldcg(reinterpret_cast<const long long *>(&gc->w[6]));
            if (!srv_apply_updates(c, p, gi, off, ldcg(&gc->w[5]))) return;
            if (c.leader) {
                GState *gs = p.gstate + gi;
                gs->no_cache = 1;
                __threadfence();
                atomicExch(&gs->epoch, ldcg(&gc->w[4]) + 1);
                QOut z = {};
                z.t_begin = z.t_done = globaltimer_ns();
                p.out[e] = z;
            }
        } else {
            const int s = ldcg(&gc->w[2]), t = ldcg(&gc->w[3]);
            bind_graph(c, p, gi);
            c.no_cache = ldcg(&gc->w[6]) != 0;
            c.q_begin = globaltimer_ns();
            if (s < 0 || t < 0 || s >= c.n || t >= c.n || s == t) {
                if (c.leader) {
                    QOut z = {};
                    z.t_begin = z.t_done = c.q_begin;
                    p.out[e] = z;
                }
            } else {
                solve_query(c, p, e, s, t);
                if (c.leader) *c.st.clock = c.clock;
            }
            if (*(volatile int *)p.err) return;
            if (c.leader) {
                __threadfence();
                atomicAdd(&p.gstate[gi].done_q, 1ull);
            }
        }
        if (*(volatile int *)p.err) return;
        if (c.leader) {
            __threadfence_system();
            p.ring_t0[2 * e + 1] = globaltimer_ns();
            __threadfence_system();
            p.ring_done[e] = 1;
        }
        // stamps are compared against the slot's 32-bit clock: reset the
        // slot long before it could wrap
        if (c.clock > (1u << 30)) {
            if (!srv_clear_slot(c, c.st, p.slot_n)) return;
            c.clock = 0;
        }
        if (!gsync(c.G, c.bar, c.err, c.lim)) return;
    }
    if (c.leader) atomicSub(&p.srv->live, 1);
}

#endif  // MF_SERVE_TU

// Per-thread context of a launch: group geometry, limits, counters.
__device__ __forceinline__ int init_ctx(QCtx &c, const KParams &p) {
    c.G = p.G;
    c.crank = blockIdx.x % p.G;
    const int gid = blockIdx.x / p.G;
    c.wpc = blockDim.x >> 5;
    c.warp = threadIdx.x >> 5;
    c.gw = c.crank * c.wpc + c.warp;
    c.gW = p.G * c.wpc;
    c.lane = threadIdx.x & 31;
    c.err = p.err;
    c.lim = p.bar_limit_ns;
    c.bu_factor = p.o.bu_factor;
    c.bu_arcs = p.o.bu_arcs;
    c.w_farcs = 0;
    c.leader = (c.crank == 0 && threadIdx.x == 0);
    c.w_arcs = c.w_verts = c.w_push = 0;
    c.t_start = globaltimer_ns();
    c.time_limit = p.time_limit_ns;
    c.no_cache = false;
    return gid;
}

#ifndef MF_SERVE_TU
// Batched / single / session solves: groups take query indices from a
// device counter until nq are taken.  (Serving has its own kernel below, so
// each kernel inlines one copy of the solve.)
__global__ void __launch_bounds__(512, 2) mf_kernel(KParams p) {
    QCtx c;
    const int gid = init_ctx(c, p);
    MF_TRACE(1, gid);
    DSlot gslot = p.slots[gid];
    c.bar = gslot.bar;
    for (;;) {
        // take a query (group leader), broadcast through the group slot
        int *qcell = gslot.cnt + CNT_Q;
        if (c.leader) *qcell = atomicAdd(p.q_next, 1);
        if (!gsync(c.G, c.bar, c.err, c.lim)) return;
        int q = ldcg(qcell);
        if (q >= p.nq) break;
        const int s = p.q_s[q], t = p.q_t[q];
        const int gi = p.q_g ? p.q_g[q] : 0;
        const int si = p.q_slot ? p.q_slot[q] : gid;
        bind_graph(c, p, gi);
        c.st = p.slots[si];
        c.clock = ldcg(c.st.clock);
        c.q_begin = globaltimer_ns();
        if (s < 0 || t < 0 || s >= c.n || t >= c.n || (s == t && p.mode != KM_KEPTSET)) {
            if (c.leader) {
                QOut z = {};
                z.t_begin = z.t_done = c.q_begin;
                p.out[q] = z;
            }
        } else {
            solve_query(c, p, q, s, t);
            // every path through solve_query consumed stamps: persist the
            // clock so the slot's next query never reuses one
            if (c.leader) *c.st.clock = c.clock;
        }
        if (*(volatile int *)p.err) return;
        if (!gsync(c.G, c.bar, c.err, c.lim)) return;
    }
}

#else  // MF_SERVE_TU
// Serving (KParams::ring_tail != NULL): see serve_loop.
__global__ void __launch_bounds__(512, 2) mf_serve_kernel(KParams p) {
    QCtx c;
    const int gid = init_ctx(c, p);
    MF_TRACE(1, gid);
    serve_loop(c, p, gid);
}

cudaError_t serve_launch_impl(const KParams &p, int grid, int threads, cudaStream_t st, bool cooperative) {
    void *args[] = {(void *)&p};
    if (cooperative)
        return cudaLaunchCooperativeKernel((void *)mf_serve_kernel, dim3(grid), dim3(threads), args, 0, st);
    return cudaLaunchKernel((void *)mf_serve_kernel, dim3(grid), dim3(threads), args, 0, st);
}

int serve_occupancy_impl(int threads) {
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, mf_serve_kernel) != cudaSuccess || threads > fa.maxThreadsPerBlock) return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, mf_serve_kernel, threads, 0) != cudaSuccess) return 0;
    return nb;
}
#endif  // MF_SERVE_TU

#ifndef MF_SERVE_TU

#ifdef MF_CHECKS
static unsigned *h_chk_trace = nullptr;
static int *h_chk_bad = nullptr;
static int h_chk_warps = 0;
extern "C" int mf_chk_host_buffers(unsigned **trace, int **bad, int *nwarps) {
    *trace = h_chk_trace;
    *bad = h_chk_bad;
    *nwarps = h_chk_warps;
    return h_chk_trace ? 0 : 1;
}
static void mf_chk_install(int warps) {
    if (h_chk_trace && warps <= h_chk_warps) {
        memset(h_chk_trace, 0, sizeof(unsigned) * 4 * h_chk_warps);
        return;
    }
    cudaHostAlloc((void **)&h_chk_trace, sizeof(unsigned) * 4 * warps, cudaHostAllocMapped);
    cudaHostAlloc((void **)&h_chk_bad, sizeof(int) * 4, cudaHostAllocMapped);
    memset(h_chk_trace, 0, sizeof(unsigned) * 4 * warps);
    memset(h_chk_bad, 0, sizeof(int) * 4);
    h_chk_warps = warps;
    MfChk c;
    cudaHostGetDevicePointer((void **)&c.trace, h_chk_trace, 0);
    cudaHostGetDevicePointer((void **)&c.bad, h_chk_bad, 0);
    cudaMemcpyToSymbol(g_chk, &c, sizeof(c));
}
#endif

void mf_launch_kernel(const KParams &p, int grid, int threads, cudaStream_t st, bool cooperative,
                      cudaError_t *err) {
#ifdef MF_CHECKS
    mf_chk_install(grid * threads / 32);
#endif
    if (p.ring_tail) {
        *err = mf_launch_serve_kernel(p, grid, threads, st, cooperative);
        return;
    }
    void *args[] = {(void *)&p};
    if (cooperative)
        *err = cudaLaunchCooperativeKernel((void *)mf_kernel, dim3(grid), dim3(threads), args, 0, st);
    else
        *err = cudaLaunchKernel((void *)mf_kernel, dim3(grid), dim3(threads), args, 0, st);
}

// Co-resident CTAs per SM that both kernels allow (every launch size is
// derived from it).
int mf_kernel_max_blocks_per_sm(int threads) {
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, mf_kernel) != cudaSuccess || threads > fa.maxThreadsPerBlock) return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, mf_kernel, threads, 0) != cudaSuccess) return 0;
    const int ns = mf_serve_kernel_max_blocks_per_sm(threads);
    return nb < ns ? nb : ns;
}
#endif  // MF_SERVE_TU
