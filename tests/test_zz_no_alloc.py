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
row, and it rejects a graph above the limit with a clear error.
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
