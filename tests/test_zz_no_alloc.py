"""The allocation-free entry point (mf_solve_csr_noalloc).

It exists for callers that must not allocate device memory where they need
a flow: code running inside a framework that owns the device memory pool,
services that reserve all memory at start-up and cannot let cudaMalloc
synchronize the device on the request path, plugins that are handed device
pointers and nothing else.  Such a caller brings its own graph in device
memory; the engine works in a fixed ~11 MB device array compiled into the
library.

Checked here through the C ABI: on graphs within the size limit it returns
exactly the flows of the allocating entry point (mf_solve), on two calls in a
row; on a CSR in the caller's own vertex order (the oracle's paired-arc
build, not the engine's region order) it returns the oracle's Dinic flows;
it rejects a graph above the limit, and a malformed CSR, with a clear error.
This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lib, mf, dev, n, arcs, a, b):
    flow = C.c_int64(-1)
    st = mf.MfStats()
    rc = lib.mf_solve_csr_noalloc(n, arcs, dev["row"].data_ptr(), dev["col"].data_ptr(), dev["rev"].data_ptr(),
                                  dev["cap"].data_ptr(), int(a), int(b), C.byref(mf.opts()), None,
                                  C.byref(flow), C.byref(st))
    return rc, flow.value


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    import mscresearch_b200 as mf
    from mscresearch_b200 import lib
    torch.cuda.set_device(0)
    n = 3000
    u, v, c = mf.gen_uniform(n, 20000, 1, 60, seed=17)
    with mf.Graph.from_edges(n, u, v, c, R=16) as g:
        ex = g.export()
        arcs = len(ex["col"])
        assert arcs <= 1 << 20
        dev = {k: torch.from_numpy(np.ascontiguousarray(ex[k])).cuda() for k in ("row", "col", "rev", "cap")}
        nid = ex["new_id"]
        rng = np.random.default_rng(5)
        queries = [(int(a), int(b)) for a, b in zip(rng.integers(0, n, 8), rng.integers(0, n, 8))] + [(3, 3)]
        expected = [g.solve(a, b)[0] for a, b in queries]
        for rep in range(2):
            got = []
            for a, b in queries:
                rc, f = _noalloc(lib, mf, dev, n, arcs, nid[a], nid[b])
                assert rc == 0, lib.mf_last_error_string()
                got.append(f)
            assert got == expected, (rep, got, expected)
    assert any(x > 0 for x in expected)


def test_noalloc_unaligned_caller_arrays():
    """A caller CSR whose arc arrays start off a 16-byte boundary (views one
    element into larger buffers): the residual init then reads scalars
    instead of 16-byte vectors, with the same flows."""
    import torch
    import mscresearch_b200 as mf
    from mscresearch_b200 import lib
    torch.cuda.set_device(0)
    n = 2000
    u, v, c = mf.gen_uniform(n, 16000, 1, 40, seed=23)
    with mf.Graph.from_edges(n, u, v, c, R=8) as g:
        ex = g.export()
        arcs = len(ex["col"])
        bufs = {}
        for k, dt in (("col", torch.int32), ("rev", torch.int32), ("cap", torch.int64)):
            b = torch.zeros(arcs + 1, dtype=dt, device="cuda")
            b[1:] = torch.from_numpy(np.ascontiguousarray(ex[k])).cuda()
            bufs[k] = b
        row = torch.from_numpy(np.ascontiguousarray(ex["row"])).cuda()
        assert (bufs["col"][1:].data_ptr() % 16) != 0 and (bufs["cap"][1:].data_ptr() % 16) != 0
        dev = {"row": row, "col": bufs["col"][1:], "rev": bufs["rev"][1:], "cap": bufs["cap"][1:]}
        nid = ex["new_id"]
        rng = np.random.default_rng(9)
        queries = [(int(a), int(b)) for a, b in zip(rng.integers(0, n, 6), rng.integers(0, n, 6))]
        expected = [g.solve(a, b)[0] for a, b in queries]
        got = []
        for a, b in queries:
            rc, f = _noalloc(lib, mf, dev, n, arcs, nid[a], nid[b])
            assert rc == 0, lib.mf_last_error_string()
            got.append(f)
        assert got == expected
    assert any(x > 0 for x in expected)


def test_noalloc_rejects_graphs_over_the_limit():
    import torch
    import mscresearch_b200 as mf
    from mscresearch_b200 import lib
    torch.cuda.set_device(0)
    dev = {k: torch.zeros(4, dtype=torch.int64 if k == "cap" else torch.int32, device="cuda")
           for k in ("row", "col", "rev", "cap")}
    rc, f = _noalloc(lib, mf, dev, 70000, 2, 0, 1)
    assert rc == 1 and f == 0
    assert b"allocation-free limit" in lib.mf_last_error_string()
    rc, f = _noalloc(lib, mf, dev, 10, (1 << 20) + 1, 0, 1)
    assert rc == 1 and b"allocation-free limit" in lib.mf_last_error_string()


def test_noalloc_caller_vertex_order_matches_dinic():
    """The caller's CSR in its own vertex order (the oracle's build of the
    edge list, no region reordering), checked against the oracle's Dinic on
    the same CSR, on two passes over the queries."""
    import torch
    import mscresearch_b200 as mf
    from mscresearch_b200 import lib
    from oracle import oracle as O
    torch.cuda.set_device(0)
    n = 4000
    u, v, c = mf.gen_rmat(12, 30000, lo=1, hi=500, seed=31)
    u, v = u % n, v % n
    g = O.build_csr(n, u, v, c)
    dev = {"row": torch.from_numpy(g.row.copy()).cuda(), "col": torch.from_numpy(g.col.copy()).cuda(),
           "rev": torch.from_numpy(g.rev.copy()).cuda(), "cap": torch.from_numpy(g.cap.copy()).cuda()}
    rng = np.random.default_rng(13)
    deg = np.diff(g.row)
    hubs = np.argsort(-deg)[:6]
    queries = [(int(a), int(b)) for a, b in zip(hubs[:3], hubs[3:])]
    queries += [(int(a), int(b)) for a, b in zip(rng.integers(0, n, 6), rng.integers(0, n, 6))]
    expected = [O.dinic(g, a, b) if a != b else 0 for a, b in queries]
    for rep in range(2):
        got = []
        for a, b in queries:
            rc, f = _noalloc(lib, mf, dev, n, g.arcs, a, b)
            assert rc == 0, lib.mf_last_error_string()
            got.append(f)
        assert got == expected, (rep, got, expected)
    assert any(x > 0 for x in expected)


def test_noalloc_rejects_malformed_csr():
    """Offsets that do not end at `arcs`, a head outside [0, n) and a reverse
    arc that does not pair back are each rejected with MF_ERR_ARG before any
    solve runs; a well-formed call on the same buffers still works after."""
    import torch
    import mscresearch_b200 as mf
    from mscresearch_b200 import lib
    from oracle import oracle as O
    torch.cuda.set_device(0)
    n = 500
    u, v, c = mf.gen_uniform(n, 3000, 1, 30, seed=41)
    g = O.build_csr(n, u, v, c)
    good = {"row": g.row, "col": g.col, "rev": g.rev, "cap": g.cap}

    def run(arrs, arcs):
        dev = {k: torch.from_numpy(np.ascontiguousarray(x)).cuda() for k, x in arrs.items()}
        return _noalloc(lib, mf, dev, n, arcs, 0, 1)

    # row[n] larger than arcs (the arc count is taken from the argument)
    row = g.row.copy()
    row[n] = g.arcs + 64
    rc, f = run(dict(good, row=row), g.arcs)
    assert rc == 1 and f == 0 and b"malformed CSR" in lib.mf_last_error_string()
    # arcs argument smaller than the offsets say
    rc, f = run(good, g.arcs - 2)
    assert rc == 1 and b"row offsets" in lib.mf_last_error_string()
    # a head outside [0, n)
    col = g.col.copy()
    col[7] = n + 3
    rc, f = run(dict(good, col=col), g.arcs)
    assert rc == 1 and b"head outside" in lib.mf_last_error_string()
    # a reverse index that points at an arc not paired back
    rev = g.rev.copy()
    rev[5] = rev[6]
    rc, f = run(dict(good, rev=rev), g.arcs)
    assert rc == 1 and b"not paired" in lib.mf_last_error_string()
    # negative capacity
    cap = g.cap.copy()
    cap[3] = -1
    rc, f = run(dict(good, cap=cap), g.arcs)
    assert rc == 1 and b"negative capacity" in lib.mf_last_error_string()
    rc, f = run(good, g.arcs)
    assert rc == 0 and f == O.dinic(g, 0, 1)
