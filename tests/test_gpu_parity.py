"""GPU parity tests: the CUDA engine, called through its C ABI, against the
CPU oracle on the same seeded inputs.  Integer results are compared exactly
(max-flow values, masks, heights, CSR arrays, ids)."""
import glob
import os
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import mscresearch_b200 as mf  # noqa: E402
from oracle import oracle as O  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(d for d in glob.glob(os.path.join(GOLDEN, "*")) if os.path.isdir(d))


def oracle_flows(g, s, t):
    return [O.dinic(g, a, b) if (0 <= a < g.n and 0 <= b < g.n and a != b) else 0 for a, b in zip(s, t)]


@pytest.mark.parametrize("d", CASES, ids=[os.path.basename(x) for x in CASES])
def test_golden_plain_and_batch(d):
    exp = np.loadtxt(os.path.join(d, "expected.txt"), dtype=np.int64, ndmin=1)
    s, t = O.parse_queries(os.path.join(d, "test.txt"))
    R = 16 if "c1" in d else 128
    with mf.Graph.load(os.path.join(d, "graph.txt"), R=R) as g:
        for i, (a, b) in enumerate(zip(s, t)):
            f, st = g.solve(a, b)
            assert f == exp[i], (i, a, b)
            assert st.status == 0
        fb = g.solve_batch(s, t)
        assert list(fb) == list(exp)


@pytest.mark.parametrize("d", CASES, ids=[os.path.basename(x) for x in CASES])
def test_golden_cli_res_mt(d):
    exp = np.loadtxt(os.path.join(d, "expected.txt"), dtype=np.int64, ndmin=1)
    with tempfile.TemporaryDirectory() as out:
        for mode, extra, fname in (("static", (), "res_mt.txt"), ("static", ("--batch",), "res_mt.txt"),
                                   ("dynamic", (), "res_dynamic.txt")):
            rc, err = mf.run_cli(d, out, mode, extra, timeout=600)
            assert rc == 0, err[-2000:]
            res = np.loadtxt(os.path.join(out, fname), dtype=np.int64, ndmin=2)
            assert res.shape == (len(exp), 2)
            assert list(res[:, 0]) == list(exp)
            assert (res[:, 1] >= 0).all()


@pytest.mark.parametrize("R", [1, 16, 128, 300])
def test_partition_reorder_bit_exact(R):
    u, v, c = mf.gen_rmat(12, 30000, seed=11)
    n = 4096
    g = O.build_csr(n, u, v, c)
    part, score = O.partition(g, min(R, n))
    g2, new_id, old_id, rs = O.reorder(g, min(R, n), part)
    with mf.Graph.from_edges(n, u, v, c, R=R) as eg:
        ex = eg.export()
    assert np.array_equal(ex["score"].view(np.int64), score.view(np.int64))
    assert np.array_equal(ex["part"], part)
    assert np.array_equal(ex["new_id"], new_id)
    assert np.array_equal(ex["region_start"], rs)
    assert np.array_equal(ex["row"], g2.row)
    assert np.array_equal(ex["col"], g2.col)
    assert np.array_equal(ex["cap"], g2.cap)
    assert np.array_equal(ex["rev"], g2.rev)


def test_partition_uniform_large_bit_exact():
    # several chunks of the stable region placement and a non-power-of-2 n
    u, v, c = mf.gen_uniform(50000, 300000, 1, 100, seed=2)
    g = O.build_csr(50000, u, v, c)
    part, score = O.partition(g, 128)
    g2, new_id, _, rs = O.reorder(g, 128, part)
    with mf.Graph.from_edges(50000, u, v, c, R=128) as eg:
        ex = eg.export()
    assert np.array_equal(ex["part"], part)
    assert np.array_equal(ex["new_id"], new_id)
    assert np.array_equal(ex["col"], g2.col) and np.array_equal(ex["rev"], g2.rev)


@pytest.fixture(scope="module")
def rmat14():
    u, v, c = mf.gen_rmat(14, 1 << 18, seed=21)
    n = 1 << 14
    g = O.build_csr(n, u, v, c)
    s, t = mf.gen_queries_hub(n, u, v, 12, 12, seed=4)
    eg = mf.Graph.from_edges(n, u, v, c, R=64)
    yield n, u, v, c, g, s, t, eg
    eg.close()


@pytest.mark.parametrize("mode,cache", [(0, 1), (1, 1), (1, 0)])
def test_prune_masks_match_oracle(rmat14, mode, cache):
    n, u, v, c, g, s, t, eg = rmat14
    for a, b in list(zip(s, t))[:10] + [(0, 1), (5, 5)]:
        m = eg.prune_mask(a, b, mode, cache)
        if a == b:
            assert m.sum() == 0
            continue
        assert np.array_equal(m, O.prune_mask(g, a, b, mode)), (a, b)


def test_initial_heights_match_oracle_bfs(rmat14):
    n, u, v, c, g, s, t, eg = rmat14
    for a, b in list(zip(s, t))[:8]:
        h = eg.initial_heights(a, b)
        mk = O.prune_mask(g, a, b, 1)
        sub, o2s, s2o = O.induced_subgraph(g, mk)
        if mk[b] == 0 or sub.n == 0 or mk.sum() <= 2 and O.dinic(g, a, b) == 0:
            continue
        res = sub.cap.copy()
        sa = o2s[a]
        for e in range(sub.row[sa], sub.row[sa + 1]):
            res[sub.rev[e]] += res[e]
            res[e] = 0
        blocked = np.zeros(sub.n, np.uint8)
        blocked[sa] = 1
        d = O.bfs_heights(sub, res, o2s[b], blocked=blocked)
        exp = np.full(n, n, np.int32)
        for i in range(sub.n):
            exp[s2o[i]] = n if d[i] >= sub.n else d[i]
        assert np.array_equal(h, exp), (a, b)


def test_rmat_batch_plain_groups_match_dinic(rmat14):
    n, u, v, c, g, s, t, eg = rmat14
    exp = oracle_flows(g, s, t)
    assert [eg.solve(a, b)[0] for a, b in zip(s, t)] == exp
    for G in (1, 2, 4, 16):
        assert list(eg.solve_batch(s, t, mf.opts(group_ctas=G))) == exp, G


def test_residual_certified_by_oracle(rmat14):
    n, u, v, c, g, s, t, eg = rmat14
    ex = eg.export()
    gi = O.CSR(n, ex["row"], ex["col"], ex["cap"], ex["rev"])
    nid = ex["new_id"]
    for a, b in list(zip(s, t))[:8]:
        f, res, st = eg.solve_residual(a, b)
        rc, cut = O.certify(gi, nid[a], nid[b], res, f, require_flow=False)
        assert rc == 0 and cut == f, (a, b, rc, cut, f)


def test_device_certificate(rmat14):
    n, u, v, c, g, s, t, eg = rmat14
    for a, b in list(zip(s, t))[:8]:
        f, st = eg.certify(a, b)
        assert st.status == 0 and st.cut_capacity == f == O.dinic(g, a, b)


def test_batch_certify_option(rmat14):
    """opts.certify = 1 on a batched solve: every answer comes back certified
    on the device (zero-excess flow, s-t cut of equal capacity)."""
    n, u, v, c, g, s, t, eg = rmat14
    exp = oracle_flows(g, s, t)
    flows, sts = eg.solve_batch(s, t, mf.opts(certify=1), with_stats=True)
    assert list(flows) == exp
    for f, st in zip(flows, sts):
        assert st.status == 0 and st.cut_capacity == f


@pytest.mark.parametrize("kw", [
    dict(use_rm=1, force_rm=1, rm_freq=1),
    dict(use_path_push=1, force_path_push=1, path_push_switch=1 << 30),
    dict(use_hot_sweep=1, hot_regions=2, kernel_cycles=1),
    dict(use_rm=0, use_path_push=0, use_hot_sweep=0, gr_freq=1, gr_work_alpha=0.0),
    dict(kernel_cycles=64, gr_freq=100000, gr_work_alpha=0.0),
    dict(prune_mode=0),
    dict(prune_mode=2),
    dict(use_kept_cache=0),
    dict(kernel_cycles=32),
    dict(local_relabel=1),
    dict(local_relabel=1, gr_freq=64, gr_work_alpha=0.0, use_rm=1, force_rm=1, rm_freq=2),
    dict(local_relabel=3, kernel_cycles=2, use_hot_sweep=1, hot_regions=2),
], ids=["rm", "path_push", "hot", "relabel_every_round", "rare_relabel", "ref_prune", "no_prune", "no_kept_cache",
        "k32", "local_relabel", "local_relabel_rare_global", "local_relabel_every_3rd_hot"])
def test_heuristics_stay_exact(rmat14, kw):
    n, u, v, c, g, s, t, eg = rmat14
    exp = oracle_flows(g, s, t)
    o = mf.opts(**kw)
    assert list(eg.solve_batch(s, t, o)) == exp
    f, st = eg.certify(s[0], t[0], o)
    assert f == exp[0] and st.cut_capacity == f


def test_local_relabel_runs_and_stays_exact(rmat14):
    """opts.local_relabel = 1 with rare global relabels: the region-restricted,
    depth-bounded relabel of RA:1583-1720 runs between global ones (counted
    in the stats) and every answer still equals the oracle's Dinic."""
    n, u, v, c, g, s, t, eg = rmat14
    exp = oracle_flows(g, s, t)
    o = mf.opts(local_relabel=1, gr_freq=1000, gr_work_alpha=0.0)
    flows, sts = eg.solve_batch(s, t, o, with_stats=True)
    assert list(flows) == exp
    assert sum(st.local_relabels for st in sts) > 0
    off = eg.solve_batch(s, t, mf.opts(gr_freq=1000, gr_work_alpha=0.0), with_stats=True)[1]
    assert sum(st.local_relabels for st in off) == 0


def test_random_small_graphs_edge_cases():
    rng = np.random.default_rng(5)
    for trial in range(40):
        n = int(rng.integers(2, 60))
        m = int(rng.integers(0, 400))
        u = rng.integers(-2, n + 2, m)
        v = rng.integers(-2, n + 2, m)
        c = rng.integers(-5, 1000, m)
        g = O.build_csr(n, u, v, c)
        s = list(rng.integers(-1, n + 1, 6)) + [0, n - 1]
        t = list(rng.integers(-1, n + 1, 6)) + [0, 0]
        exp = oracle_flows(g, s, t)
        with mf.Graph.from_edges(n, u, v, c, R=int(rng.integers(1, 20))) as eg:
            assert list(eg.solve_batch(s, t)) == exp, trial
            assert [eg.solve(a, b)[0] for a, b in zip(s, t)] == exp, trial


def test_grid_segmentation():
    W, H = 64, 48
    u, v, c = mf.gen_grid(W, H, seed=9)
    n = W * H + 2
    g = O.build_csr(n, u, v, c)
    s = [W * H, W * H, 3]
    t = [W * H + 1, 100, W * H + 1]
    exp = oracle_flows(g, s, t)
    with mf.Graph.from_edges(n, u, v, c, R=32) as eg:
        assert list(eg.solve_batch(s, t)) == exp
        f, st = eg.certify(s[0], t[0])
        assert f == exp[0] and st.cut_capacity == f


def test_full_size_rmat20_properties():
    """R-MAT n=2^20, 2^24 draws (the headline graph): batched == plain and
    device-certified (zero-excess flow + equal-capacity cut) on a sample."""
    u, v, c = mf.gen_rmat(20, 1 << 24, seed=1)
    n = 1 << 20
    s, t = mf.gen_queries_hub(n, u, v, 6, 6, seed=2)
    with mf.Graph.from_edges(n, u, v, c, R=128) as eg:
        fb = eg.solve_batch(s, t)
        for i in (0, 1, 6):
            f, st = eg.solve(s[i], t[i])
            assert f == fb[i]
            fc, stc = eg.certify(s[i], t[i])
            assert fc == f and stc.cut_capacity == f and stc.status == 0


def test_full_size_grid_properties():
    """2048 x 2048 grid with super terminals (segmentation shape, 4.2 M
    vertices): the s->t flow is device-certified, and batched == plain for it
    and for pixel pairs (deep, ~3000-level searches)."""
    W = 2048
    u, v, c = mf.gen_grid(W, W, seed=9)
    n = W * W + 2
    S, T = W * W, W * W + 1
    rng = np.random.default_rng(3)
    s = [S] + list(rng.integers(0, W * W, 3))
    t = [T] + list(rng.integers(0, W * W, 3))
    with mf.Graph.from_edges(n, u, v, c, R=128) as eg:
        fb = eg.solve_batch(s, t)
        assert [eg.solve(a, b)[0] for a, b in zip(s, t)] == list(fb)
        fc, stc = eg.certify(S, T)
        assert fc == fb[0] and stc.cut_capacity == fc and stc.status == 0


def test_batch_override_terminal_sets():
    """Queries that vary the terminal set of one grid (per-query capacities
    on the terminal arcs) == the oracle on a graph built for each set."""
    W, H, nq = 24, 16, 5
    n, gu, gv, gc, tu, tv, caps = mf.gen_grid_terminal_sets(W, H, nq, seed=4)
    S, T = W * H, W * H + 1
    nbr = len(gu) - len(tu)
    exp = []
    for i in range(nq):
        keep = caps[i] > 0
        u = np.concatenate([gu[:nbr], tu[keep]])
        v = np.concatenate([gv[:nbr], tv[keep]])
        c = np.concatenate([gc[:nbr], caps[i][keep]])
        exp.append(O.dinic(O.build_csr(n, u, v, c), S, T))
    s, t = [S] * nq, [T] * nq
    with mf.Graph.from_edges(n, gu, gv, gc, R=16) as eg:
        assert list(eg.solve_batch_override(s, t, tu, tv, caps)) == exp
        # without the prune (every vertex kept)
        assert list(eg.solve_batch_override(s, t, tu, tv, caps, mf.opts(prune_mode=2))) == exp
        assert list(eg.solve_batch_override([T, T], [S, S], tu, tv, caps[:2], mf.opts(prune_mode=2))) == [0, 0]
        # all capacities at the graph's own values: the plain batch
        full = np.tile(gc[nbr:], (2, 1))
        assert list(eg.solve_batch_override([S, 7], [T, T], tu, tv, full)) == list(eg.solve_batch([S, 7], [T, T]))
        # a pixel pair inside the grid, and a query whose source arcs are all zero
        z = caps[:2].copy()
        z[1, :W * H] = 0
        f = eg.solve_batch_override([3, S], [100, T], tu, tv, z)
        g0 = O.build_csr(n, np.concatenate([gu[:nbr], tu[z[0] > 0]]), np.concatenate([gv[:nbr], tv[z[0] > 0]]),
                         np.concatenate([gc[:nbr], z[0][z[0] > 0]]))
        assert list(f) == [O.dinic(g0, 3, 100), 0]
        # one shared pair with no path (T cannot reach S): all zero
        assert list(eg.solve_batch_override([T, T], [S, S], tu, tv, caps[:2])) == [0, 0]
        # the graph's own cache is back in place after one-pair batches
        assert list(eg.solve_batch([S, 7, 3], [T, T, 100])) == oracle_flows(O.build_csr(n, gu, gv, gc), [S, 7, 3],
                                                                           [T, T, 100])
        # rejected: an arc the graph lacks, a capacity above the graph's, certify
        with pytest.raises(mf.MaxflowError):
            eg.solve_batch_override([S], [T], [0], [W * H - 1], [[1]])
        with pytest.raises(mf.MaxflowError):
            eg.solve_batch_override([S], [T], tu[:1], tv[:1], [[256]])
        with pytest.raises(mf.MaxflowError):
            eg.solve_batch_override([S], [T], tu[:1], tv[:1], [[1]], o=mf.opts(certify=1))


def _giant_graph(seed):
    """s -> two giants (> 4096 arcs each) -> 12000 leaves -> t, leaves also
    back to the giants and to each other (so the giants sit in a strongly
    connected component); random capacities."""
    rng = np.random.default_rng(seed)
    L = 12000
    s, g1, g2, t = 0, 1, 2, 3
    leaves = np.arange(4, 4 + L, dtype=np.int32)
    n = 4 + L
    u = [np.array([s, s], np.int32), np.full(L, g1, np.int32), np.full(L // 2, g2, np.int32), leaves,
         leaves[:L // 3], leaves[1:]]
    v = [np.array([g1, g2], np.int32), leaves, leaves[L // 2:], np.full(L, t, np.int32),
         np.full(L // 3, g1, np.int32), leaves[:-1]]
    u, v = np.concatenate(u), np.concatenate(v)
    c = rng.integers(1, 60, len(u)).astype(np.int64)
    c[:2] = rng.integers(50000, 200000, 2)
    return n, u, v, c, s, t, g1, g2


def test_giant_vertices_init_certify_residual():
    n, u, v, c, s, t, g1, g2 = _giant_graph(5)
    g = O.build_csr(n, u, v, c)
    qs = [s, g1, 10, g1, s]
    qt = [t, t, t, 500, 700]
    exp = oracle_flows(g, qs, qt)
    with mf.Graph.from_edges(n, u, v, c, R=8) as eg:
        for kc in (1, 0):
            o = mf.opts(use_kept_cache=kc)
            assert list(eg.solve_batch(qs, qt, o)) == exp, kc
            assert [eg.solve(a, b, o)[0] for a, b in zip(qs, qt)] == exp, kc
        ex = eg.export()
        gi = O.CSR(n, ex["row"], ex["col"], ex["cap"], ex["rev"])
        nid = ex["new_id"]
        for a, b, e in zip(qs, qt, exp):
            f, res, st = eg.solve_residual(a, b)
            rc, cut = O.certify(gi, nid[a], nid[b], res, f, require_flow=False)
            assert f == e and rc == 0 and cut == f, (a, b)
            fc, stc = eg.certify(a, b)
            assert fc == e and stc.cut_capacity == e and stc.status == 0, (a, b)


def test_giant_vertices_session_repair():
    """A giant leaves and re-enters a resident query's kept set through
    capacity updates; every answer equals a fresh solve of the updated graph."""
    n, u, v, c, s, t, g1, g2 = _giant_graph(6)
    g = O.build_csr(n, u, v, c)
    fwd = g.cap > 0
    with mf.Graph.from_edges(n, u, v, c, R=8) as eg:
        ss = mf.Session(eg, [s, g1], [t, t])
        assert list(ss.solve()) == oracle_flows(g, [s, g1], [t, t])
        for du in ([-int(c[0]), -int(c[1])], [7, 0], [0, 90000], [-3, 5]):
            uu = np.array([s, s], np.int32)
            vv = np.array([g1, g2], np.int32)
            d = np.array(du, np.int64)
            fr = ss.update(uu, vv, d)
            for a, b, dd in zip(uu, vv, d):
                es = [e for e in range(g.row[a], g.row[a + 1]) if g.col[e] == b and fwd[e]]
                g.cap[es[0]] = max(0, g.cap[es[0]] + dd)
            exp = oracle_flows(g, [s, g1], [t, t])
            assert list(fr) == exp, du
            assert list(eg.solve_batch([s, g1], [t, t])) == exp, du
        ss.close()
