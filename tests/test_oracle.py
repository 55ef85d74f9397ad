"""CPU tests of the oracle itself: golden vectors, two independent exact
solvers agreeing, certificates, and the reference's host-side semantics
(reader rules, prune masks, partition/reorder invariants)."""
import glob
import math
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(d for d in glob.glob(os.path.join(GOLDEN, "*")) if os.path.isdir(d))


def load_case(d):
    n, u, v, c = O.parse_graph(os.path.join(d, "graph.txt"))
    g = O.build_csr(n, u, v, c)
    s, t = O.parse_queries(os.path.join(d, "test.txt"))
    exp = np.loadtxt(os.path.join(d, "expected.txt"), dtype=np.int64, ndmin=1)
    return g, s, t, exp


@pytest.mark.parametrize("d", CASES, ids=[os.path.basename(x) for x in CASES])
def test_golden_dinic_and_push_relabel(d):
    g, s, t, exp = load_case(d)
    assert len(s) == len(exp)
    for a, b, e in zip(s, t, exp):
        valid = 0 <= a < g.n and 0 <= b < g.n and a != b
        f1 = O.dinic(g, a, b) if valid else 0
        f2 = O.push_relabel(g, a, b) if valid else 0
        assert f1 == e and f2 == e


@pytest.mark.parametrize("d", CASES, ids=[os.path.basename(x) for x in CASES])
def test_golden_reference_dynamic_outputs(d):
    """Pin: the oracle's flows equal the reference CUDA program's dynamic-mode
    answers (res_dynamic.txt; full graph + reach mask, RA:2232-2269), recorded
    on a B200 by make_golden.py --with-ref — every query, no exceptions."""
    p = os.path.join(d, "ref_res_dynamic.txt")
    if not os.path.exists(p):
        pytest.skip("no reference output recorded for this case")
    ref = np.loadtxt(p, dtype=np.int64, ndmin=2)[:, 0]
    _, _, _, exp = load_case(d)
    assert list(ref) == list(exp)


@pytest.mark.parametrize("d", CASES, ids=[os.path.basename(x) for x in CASES])
def test_golden_reference_outputs(d):
    """Pin: the oracle's flows equal the reference CUDA program's static-mode
    res_mt.txt except on the queries listed in ref_mismatch.txt, each a
    'fallback=full' query hit by the reference's stale-topology upload
    (RA:1303-1331; see that file and the reference's own log ref_log_static.txt)."""
    p = os.path.join(d, "ref_res_mt.txt")
    if not os.path.exists(p):
        pytest.skip("no reference output recorded for this case")
    ref = np.loadtxt(p, dtype=np.int64, ndmin=2)[:, 0]
    _, _, _, exp = load_case(d)
    log = os.path.join(d, "ref_log_static.txt")
    fallback = [("fallback=full" in l) for l in open(log) if l.startswith("[QueryPrune")] if os.path.exists(log) else []
    known = os.path.join(d, "ref_mismatch.txt")
    allowed = set()
    if os.path.exists(known):
        allowed = {int(l.split()[0]) for l in open(known) if l.strip() and not l.startswith("#")}
    for i, (r, e) in enumerate(zip(ref, exp)):
        if i in allowed:
            continue
        assert r == e, "query %d: reference %d vs oracle %d" % (i, r, e)
    # every listed mismatch is a fallback=full query (one prune line per
    # query when no query is invalid)
    if fallback and len(fallback) == len(exp):
        for i in allowed:
            assert fallback[i], i


def random_graph(rng, n, m, lo=-3, hi=40):
    u = rng.integers(-1, n + 1, m)
    v = rng.integers(-1, n + 1, m)
    c = rng.integers(lo, hi, m)
    return O.build_csr(n, u, v, c)


def test_random_solvers_agree_and_certify():
    rng = np.random.default_rng(7)
    for _ in range(200):
        n = int(rng.integers(2, 50))
        g = random_graph(rng, n, int(rng.integers(0, 200)))
        s, t = int(rng.integers(0, n)), int(rng.integers(0, n))
        f, res = O.dinic(g, s, t, want_res=True)
        assert O.push_relabel(g, s, t) == f
        if s != t:
            rc, cut = O.certify(g, s, t, res, f, require_flow=True)
            assert rc == 0 and cut == f


def test_certifier_rejects_wrong_answers():
    rng = np.random.default_rng(8)
    g = random_graph(rng, 30, 150, lo=1)
    f, res = O.dinic(g, 0, 29, want_res=True)
    assert O.certify(g, 0, 29, res, f + 1)[0] != 0
    bad = res.copy()
    bad[0] += 1
    assert O.certify(g, 0, 29, bad, f)[0] != 0


def test_reader_rules():
    # RA:1073-1075: out-of-range ids, self loops, cap <= 0 dropped
    g = O.build_csr(3, [0, 1, 2, 0, 5, -1, 1], [1, 1, 0, 2, 1, 0, 2], [4, 9, 3, 0, 2, 2, -1])
    assert g.arcs == 4
    assert list(g.row) == [0, 2, 3, 4]
    # row 0: forward 0->1 then reverse of 2->0
    assert list(g.col[:2]) == [1, 2] and list(g.cap[:2]) == [4, 0]
    for e in range(g.arcs):
        assert g.rev[g.rev[e]] == e


def test_parse_stops_at_first_bad_line(tmp_path):
    p = tmp_path / "graph.txt"
    p.write_text("4 5\n1 2 3\n2 3 4\n3 x 1\n3 4 5\n")
    n, u, v, c = O.parse_graph(str(p))
    assert n == 4 and len(u) == 2


def test_prune_masks():
    # 0->1->2->3 plus 4->3 (not reachable from 0) and 1->5 (dead end)
    g = O.build_csr(6, [0, 1, 2, 4, 1], [1, 2, 3, 3, 5], [1, 1, 1, 1, 1])
    m0 = O.prune_mask(g, 0, 3, 0)  # fwd(0) & undirected comp(3): includes 5
    m1 = O.prune_mask(g, 0, 3, 1)  # fwd(0) & bwd(3): excludes dead end 5
    assert list(m0) == [1, 1, 1, 1, 0, 1]
    assert list(m1) == [1, 1, 1, 1, 0, 0]
    # both preserve the flow on random graphs
    rng = np.random.default_rng(9)
    for _ in range(100):
        n = int(rng.integers(2, 40))
        g = random_graph(rng, n, int(rng.integers(0, 120)), lo=1)
        s, t = int(rng.integers(0, n)), int(rng.integers(0, n))
        if s == t:
            continue
        f = O.dinic(g, s, t)
        for mode in (0, 1):
            mk = O.prune_mask(g, s, t, mode)
            sub, o2s, _ = O.induced_subgraph(g, mk)
            assert O.dinic(sub, o2s[s], o2s[t]) == f


def test_det_log_accuracy():
    rng = np.random.default_rng(3)
    for x in list(rng.uniform(1, 1e15, 500)) + [1.0, 2.0, 1e300]:
        assert abs(O.det_log(x) - math.log(x)) <= 4e-16 * max(1.0, abs(math.log(x)))


def test_partition_reorder_invariants():
    rng = np.random.default_rng(4)
    g = random_graph(rng, 300, 2000, lo=1)
    R = 16
    part, score = O.partition(g, R)
    g2, new_id, old_id, rs = O.reorder(g, R, part)
    assert rs[0] == 0 and rs[R] == g.n and np.all(np.diff(rs) >= 0)
    assert np.array_equal(np.sort(new_id), np.arange(g.n))
    for x in range(g.n):
        r = part[x]
        assert rs[r] <= new_id[x] < rs[r + 1]
    # same multiset of arcs, rev involution, flows preserved
    for e in range(g2.arcs):
        assert g2.rev[g2.rev[e]] == e
        assert g2.cap[e] + g2.cap[g2.rev[e]] > 0
    for _ in range(10):
        s, t = rng.integers(0, g.n, 2)
        if s != t:
            assert O.dinic(g, s, t) == O.dinic(g2, new_id[s], new_id[t])
    # greedy packing keeps region loads within one max score of each other
    loads = np.zeros(R)
    for x in range(g.n):
        loads[part[x]] += score[x]
    assert loads.max() - loads.min() <= score.max() + 1e-9


def test_boundary_core_is_not_flow_preserving():
    """RA:2428-2475 keeps, inside each kept region, only vertices within 2
    intra-region hops of a boundary vertex (or in s's / t's region).  A path
    that dips deeper into a region is cut: the reference's core shrink can
    lower the max flow, so the engine applies only the exact prune."""
    # regions: A = {0 (s)}, B = {1..8} chain, C = {9 (t)}; only 1 and 8 are
    # boundary vertices; 4 and 5 are 3 hops deep -> dropped
    n = 10
    E = [(i, i + 1, 5) for i in range(9)]
    g = O.build_csr(n, [e[0] for e in E], [e[1] for e in E], [e[2] for e in E])
    region_of = [0] + [1] * 8 + [2]
    mk = O.boundary_core_mask(g, 3, region_of, 0, 9, hop_limit=2)
    assert list(mk) == [1, 1, 1, 1, 0, 0, 1, 1, 1, 1]
    sub, o2s, _ = O.induced_subgraph(g, mk)
    assert O.dinic(g, 0, 9) == 5
    assert O.dinic(sub, o2s[0], o2s[9]) == 0


def test_checker_generators_equal_engine_generators(tmp_path):
    """The reference arm of bench.py writes the reference program's inputs
    with the oracle's generators (so its process never loads the engine's
    library); they must produce exactly the engine's workload: the same
    R-MAT arrays, the same query mix, byte-identical graph.txt / test.txt."""
    import mscresearch_b200 as mf
    for scale, m, seed in ((10, 8192, 3), (14, 16 << 14, 1), (16, 300001, 77)):
        u1, v1, c1 = mf.gen_rmat(scale, m, 0.57, 0.19, 0.19, 1, 1000, seed)
        u2, v2, c2 = O.gen_rmat(scale, m, 0.57, 0.19, 0.19, 1, 1000, seed)
        assert np.array_equal(u1, u2) and np.array_equal(v1, v2) and np.array_equal(c1, c2)
        n = 1 << scale
        s1, t1 = mf.gen_queries_hub(n, u1, v1, 16, 16, seed + 5)
        s2, t2 = O.gen_queries_hub(n, u2, v2, 16, 16, seed + 5)
        assert np.array_equal(s1, s2) and np.array_equal(t1, t2)
        mf.write_graph_txt(str(tmp_path / "g1.txt"), n, u1, v1, c1)
        O.write_graph_txt(str(tmp_path / "g2.txt"), n, u2, v2, c2)
        assert (tmp_path / "g1.txt").read_bytes() == (tmp_path / "g2.txt").read_bytes()
        mf.write_test_txt(str(tmp_path / "t1.txt"), s1, t1)
        O.write_test_txt(str(tmp_path / "t2.txt"), s2, t2)
        assert (tmp_path / "t1.txt").read_bytes() == (tmp_path / "t2.txt").read_bytes()


@pytest.mark.parametrize("d", CASES, ids=[os.path.basename(x) for x in CASES])
def test_reference_mismatch_classifier_on_golden_logs(d):
    """bench.py's reference arm classifies each reference/oracle mismatch from
    the reference's own log.  On the recorded B200 runs every known mismatch
    (ref_mismatch.txt) must come out as 'stale-topology' (RA:1303-1331)."""
    import bench
    p = os.path.join(d, "ref_res_mt.txt")
    log = os.path.join(d, "ref_log_static.txt")
    if not (os.path.exists(p) and os.path.exists(log)):
        pytest.skip("no reference output recorded for this case")
    g, s, t, exp = load_case(d)
    ref = np.loadtxt(p, dtype=np.int64, ndmin=2)[:, 0]
    if not all(0 <= a < g.n and 0 <= b < g.n and a != b for a, b in zip(s, t)):
        pytest.skip("case has invalid queries (no log line for them)")
    bad = [i for i in range(len(exp)) if ref[i] != exp[i]]
    cls = bench.classify_reference_mismatches(open(log).read(), g.n, g.arcs, bad)
    assert all(c == "stale-topology" for c in cls.values()), cls


def test_partition_against_reference_libm_log():
    """The engine's partition (and the oracle's restatement it is pinned to)
    evaluates the score's logarithm with a fixed IEEE sequence so that host
    and device agree bit for bit; the reference uses libm std::log
    (RA:1147-1151).  The scores agree to a few ulp, and on the golden graphs
    and R-MAT 2^14 every vertex lands in the same region under both (ties in
    the score order broken by id in both; the reference's std::sort leaves
    their order unspecified).  Flows do not depend on the partition: the max
    flow is a property of the graph alone."""
    import mscresearch_b200 as mf
    graphs = []
    for d in CASES:
        g, _, _, _ = load_case(d)
        graphs.append((os.path.basename(d), g))
    u, v, c = mf.gen_rmat(14, 16 << 14, seed=4)
    graphs.append(("rmat14", O.build_csr(1 << 14, u, v, c)))
    for name, g in graphs:
        for R in (16, 128):
            if R > g.n:
                continue
            p1, s1 = O.partition(g, R)
            p2, s2 = O.partition_libm(g, R)
            rel = np.abs(s1 - s2) / np.maximum(1e-300, np.abs(s2))
            assert rel.max() < 1e-14, (name, R, rel.max())
            diff = int((p1 != p2).sum())
            print("partition %s R=%d: %d of %d vertices in another region (max score rel. diff %.1e)"
                  % (name, R, diff, g.n, rel.max()))
            assert diff == 0, (name, R, diff)


def _apply_to_residual(g, res, cap, e, delta):
    """One capacity change on forward arc e, as a repair applies it to the
    resident residual: returns (opened, cancelled)."""
    old = int(cap[e])
    new = max(0, old + int(delta))
    r = int(res[e])
    fl = old - r
    opened = cancelled = False
    if fl <= new:
        res[e] = r + (new - old)
        opened = r <= 0 and new > old
    else:
        res[e] = 0
        res[g.rev[e]] -= fl - new
        cancelled = True
    cap[e] = new
    return opened, cancelled


def test_unreachable_set_survives_batches_that_open_no_arc():
    """The argument behind carrying dead marks into a repair: after a max
    flow, the vertices that cannot reach t in the residual graph (s blocked)
    still cannot after a batch of capacity changes that opens no residual arc
    (0 to positive) and cancels no flow.  And the condition is needed: one
    opened arc out of that set can reconnect it."""
    rng = np.random.default_rng(17)
    checked = reconnected = 0
    for trial in range(60):
        n = int(rng.integers(30, 200))
        m = int(rng.integers(2 * n, 6 * n))
        u = rng.integers(0, n, m)
        v = rng.integers(0, n, m)
        c = rng.integers(1, 20, m)
        g = O.build_csr(n, u, v, c)
        s, t = 0, n - 1
        _, res = O.dinic(g, s, t, want_res=True)
        blocked = np.zeros(n, np.uint8)
        blocked[s] = 1
        U = O.bfs_heights(g, res, t, blocked=blocked) >= n
        U[s] = False
        cap = g.cap.copy()
        fwd = np.nonzero(g.cap > 0)[0]
        res2 = res.copy()
        opened = cancelled = False
        for e in rng.choice(fwd, size=min(len(fwd), int(rng.integers(1, 12))), replace=False):
            o, x = _apply_to_residual(g, res2, cap, e, int(rng.integers(-5, 6)))
            opened |= o
            cancelled |= x
        if not opened and not cancelled:
            d1 = O.bfs_heights(O.CSR(n, g.row, g.col, cap, g.rev), res2, t, blocked=blocked)
            assert (d1[U] >= n).all(), trial
            checked += 1
        # an arc x -> w from the set to a vertex that reaches t, saturated:
        # raising its capacity opens it and x reaches t again
        tails = np.repeat(np.arange(n), np.diff(g.row))
        cut = [e for e in fwd if U[tails[e]] and not U[g.col[e]] and g.col[e] != s and res[e] == 0]
        if cut:
            res3, cap3 = res.copy(), g.cap.copy()
            o, _ = _apply_to_residual(g, res3, cap3, cut[0], 3)
            assert o
            d2 = O.bfs_heights(O.CSR(n, g.row, g.col, cap3, g.rev), res3, t, blocked=blocked)
            assert d2[tails[cut[0]]] < n
            reconnected += 1
    assert checked >= 10 and reconnected >= 10, (checked, reconnected)
