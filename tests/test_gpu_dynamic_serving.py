"""GPU tests of the resident-session (dynamic capacity) path, the
continuous-batching server and the autotuner: every answer must equal a
fresh exact solve of the same graph state."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import mscresearch_b200 as mf  # noqa: E402
from oracle import oracle as O  # noqa: E402


def apply_updates_oracle(g, fwd, u, v, d):
    """Reference semantics of mf_update_caps on the oracle CSR (caller ids):
    first forward arc u->v, cap += delta clamped at 0, applied in order."""
    for a, b, x in zip(u, v, d):
        if not (0 <= a < g.n and 0 <= b < g.n) or a == b:
            continue
        for e in range(g.row[a], g.row[a + 1]):
            if g.col[e] == b and fwd[e]:
                g.cap[e] = max(0, g.cap[e] + x)
                break


def make_updates(rng, u, v, k, n):
    idx = rng.integers(0, len(u), k)
    uu, vv = u[idx].copy(), v[idx].copy()
    # a few pairs with no arc, a few repeated arcs
    uu[: k // 50] = rng.integers(0, n, k // 50)
    vv[: k // 50] = rng.integers(0, n, k // 50)
    if k >= 4:
        uu[-2:], vv[-2:] = uu[-4:-2], vv[-4:-2]
    d = rng.integers(1, 101, k) * np.where(rng.random(k) < 0.5, -1, 1)
    return uu, vv, d


@pytest.mark.parametrize("policy", ["repair", "default"])
@pytest.mark.parametrize("scale", [10, 14])
def test_session_incremental_equals_fresh(scale, policy, monkeypatch):
    """Resident answers after each update batch equal the oracle's; "repair"
    forces the incremental path for every batch size, "default" lets large
    batches re-solve from scratch."""
    if policy == "repair":
        monkeypatch.setenv("MF_REPAIR_MAX_UPDATES", "1000000000")
    else:
        monkeypatch.delenv("MF_REPAIR_MAX_UPDATES", raising=False)
    n = 1 << scale
    u, v, c = mf.gen_rmat(scale, 16 * n, seed=31 + scale)
    s, t = mf.gen_queries_hub(n, u, v, 6, 6, seed=8)
    g = O.build_csr(n, u, v, c)
    fwd = g.cap > 0
    rng = np.random.default_rng(scale)
    with mf.Graph.from_edges(n, u, v, c, R=32) as eg:
        ss = mf.Session(eg, s, t)
        f0 = ss.solve()
        assert list(f0) == [O.dinic(g, a, b) for a, b in zip(s, t)]
        for k in (10, 200, 3000):
            uu, vv, d = make_updates(rng, u, v, k, n)
            fr = ss.update(uu, vv, d)
            apply_updates_oracle(g, fwd, uu, vv, d)
            exp = [O.dinic(g, a, b) for a, b in zip(s, t)]
            assert list(fr) == exp, k
            # and a fresh static solve on the updated device graph agrees
            assert list(eg.solve_batch(s, t)) == exp
        ss.close()


@pytest.mark.parametrize("scale", [12, 15])
def test_session_many_small_batches_equal_oracle(scale):
    """Many small batches in a row (decreases and increases of 1..5): batches
    that open no residual arc and cancel no flow on a query's kept arcs let
    its repair keep the previous solve's dead marks; every answer after every
    batch equals the oracle's Dinic on the updated graph."""
    n = 1 << scale
    u, v, c = mf.gen_rmat(scale, 16 * n, seed=50 + scale)
    s, t = mf.gen_queries_hub(n, u, v, 8, 8, seed=9)
    g = O.build_csr(n, u, v, c)
    fwd = g.cap > 0
    rng = np.random.default_rng(100 + scale)
    with mf.Graph.from_edges(n, u, v, c, R=32) as eg:
        with mf.Session(eg, s, t) as ss:
            assert list(ss.solve()) == [O.dinic(g, a, b) for a, b in zip(s, t)]
            for b in range(16):
                k = int(rng.integers(1, 24))
                idx = rng.integers(0, len(u), k)
                sign = -1 if b % 3 == 0 else (1 if b % 3 == 1 else 0)
                mag = rng.integers(1, 6, k)
                d = mag * (sign if sign else np.where(rng.random(k) < 0.5, -1, 1))
                fr = ss.update(u[idx], v[idx], d)
                apply_updates_oracle(g, fwd, u[idx], v[idx], d)
                assert list(fr) == [O.dinic(g, a, b2) for a, b2 in zip(s, t)], b


def test_update_caps_hub_tail_parallel_arcs():
    """Updates on (hub, leaf) pairs are resolved through the leaf's shorter
    list; with parallel edges the first forward arc in input order must take
    the change (same rule as the oracle)."""
    n = 64
    u = list(range(1, 60)) + [7, 0, 0, 7, 3]
    v = [0] * 59 + [0, 7, 7, 3, 0]
    c = list(range(1, 60)) + [4, 5, 9, 2, 8]
    # vertex 0 gets 59 in-arcs + parallel out-arcs 0->7 (caps 5, 9); 7 and 3 are short lists
    u, v, c = np.array(u, np.int32), np.array(v, np.int32), np.array(c, np.int64)
    u = np.concatenate([u, np.zeros(40, np.int32)])
    v = np.concatenate([v, np.arange(20, 60, dtype=np.int32)])
    c = np.concatenate([c, np.full(40, 3, np.int64)])
    g = O.build_csr(n, u, v, c)
    fwd = g.cap > 0
    with mf.Graph.from_edges(n, u, v, c, R=4) as eg:
        uu = np.array([0, 7, 0, 3, 30], np.int32)
        vv = np.array([7, 0, 7, 0, 0], np.int32)
        d = np.array([100, -3, -50, 7, 2], np.int64)
        eg.update_caps(uu, vv, d)
        apply_updates_oracle(g, fwd, uu, vv, d)
        ex = eg.export()
        assert np.array_equal(np.sort(ex["cap"]), np.sort(g.cap))
        for a, b in [(0, 7), (7, 0), (30, 7), (3, 7)]:
            assert eg.solve(a, b)[0] == O.dinic(g, a, b), (a, b)


def test_update_caps_then_fresh_solve():
    n = 2000
    u, v, c = mf.gen_uniform(n, 12000, 1, 50, seed=2)
    g = O.build_csr(n, u, v, c)
    fwd = g.cap > 0
    rng = np.random.default_rng(1)
    with mf.Graph.from_edges(n, u, v, c, R=16) as eg:
        uu, vv, d = make_updates(rng, u, v, 500, n)
        skipped = eg.update_caps(uu, vv, d)
        apply_updates_oracle(g, fwd, uu, vv, d)
        assert skipped >= 1
        ex = eg.export()
        assert np.array_equal(np.sort(ex["cap"]), np.sort(g.cap))
        for a, b in [(0, 1), (5, 77), (1999, 3)]:
            assert eg.solve(a, b)[0] == O.dinic(g, a, b)


def test_server_results_equal_alone_and_in_the_mix():
    graphs, ocsr, queries = [], [], []
    for i, scale in enumerate((10, 12, 13)):
        n = 1 << scale
        u, v, c = mf.gen_rmat(scale, 16 * n, seed=40 + i)
        graphs.append(mf.Graph.from_edges(n, u, v, c, R=32))
        ocsr.append(O.build_csr(n, u, v, c))
        s, t = mf.gen_queries_hub(n, u, v, 8, 8, seed=50 + i)
        queries.append((s, t))
    # expected: each query alone (plain whole-GPU solve) and the oracle
    alone = {}
    for gi, (s, t) in enumerate(queries):
        for a, b in zip(s, t):
            alone[(gi, int(a), int(b))] = graphs[gi].solve(a, b)[0]
            assert alone[(gi, int(a), int(b))] == O.dinic(ocsr[gi], a, b)
    sv = mf.Server(graphs, mf.opts(group_ctas=2), max_slots=8)
    assert 1 <= sv.slots <= 8
    rng = np.random.default_rng(0)
    reqs = [(gi, int(a), int(b)) for gi, (s, t) in enumerate(queries) for a, b in zip(s, t)]
    order = rng.permutation(len(reqs))
    tickets = []
    for k, i in enumerate(order):
        gi, a, b = reqs[i]
        tickets.append((sv.submit(gi, a, b), reqs[i]))
        if k % 7 == 3:
            time.sleep(0.002)  # requests keep arriving while others run
    sv.drain()
    lat = []
    for tk, key in tickets:
        done, f, l, st = sv.poll(tk)
        assert done and st == 0
        assert f == alone[key], key
        lat.append(l)
    assert min(lat) >= 0
    # a second wave after the persistent kernel went idle
    time.sleep(0.5)
    gi, a, b = reqs[0]
    tk = sv.submit(gi, a, b)
    sv.drain()
    assert sv.poll(tk)[1] == alone[(gi, a, b)]
    sv.close()
    for g in graphs:
        g.close()


def test_server_interleaves_updates_and_queries():
    """Queries and capacity-update batches on two graphs go through one
    server in a random order, with pauses so some arrive while others run.
    Every answer equals the oracle's Dinic on its graph as left by exactly the
    update batches submitted before it; a ring of 64 entries is reused many
    times over; after the server is gone the graphs solve on the updated
    capacities (their kept-set caches dropped)."""
    import os
    rng = np.random.default_rng(21)
    graphs, ocsr, fwds, ends = [], [], [], []
    for i, scale in enumerate((11, 13)):
        n = 1 << scale
        u, v, c = mf.gen_rmat(scale, 16 * n, seed=60 + i)
        graphs.append(mf.Graph.from_edges(n, u, v, c, R=32))
        g = O.build_csr(n, u, v, c)
        ocsr.append(g)
        fwds.append(g.cap > 0)
        ends.append((u, v, n))
    old = os.environ.get("MF_SERVER_RING")
    os.environ["MF_SERVER_RING"] = "64"
    try:
        sv = mf.Server(graphs, mf.opts(group_ctas=2), max_slots=6)
    finally:
        if old is None:
            del os.environ["MF_SERVER_RING"]
        else:
            os.environ["MF_SERVER_RING"] = old
    expected, tickets = [], []
    nupd = 0
    for k in range(150):
        gi = int(rng.integers(0, 2))
        u, v, n = ends[gi]
        if rng.random() < 0.25:
            uu, vv, d = make_updates(rng, u, v, int(rng.integers(5, 300)), n)
            tickets.append(sv.update(gi, uu, vv, d))
            apply_updates_oracle(ocsr[gi], fwds[gi], uu, vv, d)
            expected.append(None)
            nupd += 1
        else:
            hub = rng.random() < 0.5
            deg = np.diff(ocsr[gi].row)
            if hub:
                top = np.argsort(-deg)[:max(2, n // 100)]
                a, b = int(rng.choice(top)), int(rng.choice(top))
            else:
                a, b = int(rng.integers(0, n)), int(rng.integers(0, n))
            tickets.append(sv.submit(gi, a, b))
            expected.append(O.dinic(ocsr[gi], a, b) if a != b else 0)
        if k % 5 == 2:
            time.sleep(0.003)
        # poll every answer before its ring entry (64) is reused
        if k % 16 == 15:
            sv.drain()
            for tk, ex in zip(tickets[-16:], expected[-16:]):
                done, f, lat, st = sv.poll(tk)
                assert done and st == 0
                if ex is not None:
                    assert f == ex, (tk, f, ex)
    sv.drain()
    for tk, ex in list(zip(tickets, expected))[-(150 % 16):]:
        done, f, lat, st = sv.poll(tk)
        assert done and st == 0
        if ex is not None:
            assert f == ex, (tk, f, ex)
    assert nupd >= 20 and 1 <= sv.slots <= 6
    # an expired ticket is reported as such
    with pytest.raises(mf.MaxflowError):
        sv.poll(tickets[0])
    sv.close()
    for gi, g in enumerate(graphs):
        n = ends[gi][2]
        for a, b in [(0, 1), (3, n - 1), (n // 2, 7)]:
            assert g.solve(a, b)[0] == O.dinic(ocsr[gi], a, b)
        g.close()


def test_server_admits_slots_as_requests_open():
    """The server starts with a few slots and admits more (from free HBM)
    while requests queue up; every answer stays exact."""
    n = 1 << 14
    u, v, c = mf.gen_rmat(14, 16 * n, seed=77)
    s, t = mf.gen_queries_hub(n, u, v, 48, 16, seed=78)
    g = O.build_csr(n, u, v, c)
    exp = [O.dinic(g, a, b) for a, b in zip(s, t)]
    with mf.Graph.from_edges(n, u, v, c, R=32) as eg:
        with mf.Server([eg], mf.opts(group_ctas=2)) as sv:
            first = sv.slots
            assert 1 <= first <= 4
            tks = [sv.submit(0, a, b) for a, b in zip(s, t)]
            sv.drain()
            assert [sv.poll(tk)[1] for tk in tks] == exp
            assert sv.slots > first


def test_autotune_consistent():
    n = 1 << 12
    u, v, c = mf.gen_rmat(12, 16 * n, seed=3)
    s, t = mf.gen_queries_hub(n, u, v, 6, 6, seed=1)
    g = O.build_csr(n, u, v, c)
    exp = [O.dinic(g, a, b) for a, b in zip(s, t)]
    with mf.Graph.from_edges(n, u, v, c, R=128) as eg:
        best, R = eg.autotune(s, t)
        assert R in (32, 64, 128, 256, 512)
        assert eg.info[2] == R
        assert list(eg.solve_batch(s, t, best)) == exp


def test_full_size_dynamic_properties():
    """R-MAT n = 2^22 with 2^26 draws (the dynamic-serving shape): after a
    batch of 10k seeded +-U[1,100] capacity changes the session's
    incrementally repaired answers equal fresh solves, and one is certified."""
    u, v, c = mf.gen_rmat(22, 1 << 26, seed=5)
    n = 1 << 22
    s, t = mf.gen_queries_hub(n, u, v, 4, 4, seed=6)
    rng = np.random.default_rng(7)
    with mf.Graph.from_edges(n, u, v, c, R=128) as eg:
        ss = mf.Session(eg, s, t)
        f0 = ss.solve()
        assert list(f0) == list(eg.solve_batch(s, t))
        idx = rng.integers(0, len(u), 10000)
        d = rng.integers(1, 101, 10000) * rng.choice([-1, 1], 10000)
        f1 = ss.update(u[idx], v[idx], d)
        assert list(f1) == list(eg.solve_batch(s, t))
        fc, stc = eg.certify(s[0], t[0])
        assert fc == f1[0] and stc.cut_capacity == fc and stc.status == 0
        ss.close()
