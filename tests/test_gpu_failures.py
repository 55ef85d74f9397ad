"""Failure paths of the engine, driven from the host.  None of these faults,
traps or hangs the GPU: the round cap and the launch time limit are
checked by the device code itself, which ends the solve with a status word
the host reads; admission is refused on the host before anything is
allocated; allocation failures are injected in the host's allocation wrapper
(no CUDA call is made for the failing allocation).

Reference guards these replace: ITER_MAX (RA:1476, 1893-1896) and
abort() after every launch (e.g. RA:2152-2157); the reference checks no
allocation.
"""
import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NOMEM, ITER_LIMIT, TIMEOUT = 3, 5, 6


def _rmat(scale=14, seed=11):
    import mscresearch_b200 as mf
    u, v, c = mf.gen_rmat(scale, 16 << scale, lo=1, hi=1000, seed=seed)
    n = 1 << scale
    s, t = mf.gen_queries_hub(n, u, v, 4, 4, seed=seed + 1)
    return n, u, v, c, s, t


def _dinic(n, u, v, c, s, t):
    from oracle import oracle as O
    g = O.build_csr(n, u, v, c)
    return [O.dinic(g, int(a), int(b)) for a, b in zip(s, t)]


def test_iteration_cap_returns_iter_limit_then_solves_exactly():
    """opts.iter_max = 1 on a hub query: the solve stops after its first round
    with MF_ERR_ITER_LIMIT; the same graph then solves exactly."""
    import torch
    import mscresearch_b200 as mf
    torch.cuda.set_device(0)
    n, u, v, c, s, t = _rmat()
    exp = _dinic(n, u, v, c, s[:2], t[:2])
    with mf.Graph.from_edges(n, u, v, c, R=32) as g:
        with pytest.raises(mf.MaxflowError) as ei:
            g.solve(s[0], t[0], mf.opts(iter_max=1))
        assert ei.value.code == ITER_LIMIT
        with pytest.raises(mf.MaxflowError) as ei:
            g.solve_batch(s[:2], t[:2], mf.opts(iter_max=1))
        assert ei.value.code == ITER_LIMIT
        assert [g.solve(a, b)[0] for a, b in zip(s[:2], t[:2])] == exp
        assert list(g.solve_batch(s[:2], t[:2])) == exp


def test_launch_time_limit_returns_timeout_then_solves_exactly():
    """MF_TIME_LIMIT_S=0.00001: the group leader finds the launch past its
    limit at its first round check and raises the status word; every CTA
    leaves at its next barrier and the host returns MF_ERR_TIMEOUT.  With the
    limit lifted the same graph solves exactly."""
    import torch
    import mscresearch_b200 as mf
    torch.cuda.set_device(0)
    n, u, v, c, s, t = _rmat(16, seed=5)
    exp = _dinic(n, u, v, c, s[:3], t[:3])
    with mf.Graph.from_edges(n, u, v, c, R=64) as g:
        g.solve(s[0], t[0])  # builds the kept-set cache outside the limit
        old = os.environ.get("MF_TIME_LIMIT_S")
        os.environ["MF_TIME_LIMIT_S"] = "0.00001"
        try:
            with pytest.raises(mf.MaxflowError) as ei:
                g.solve_batch(s, t)
            assert ei.value.code == TIMEOUT
        finally:
            if old is None:
                del os.environ["MF_TIME_LIMIT_S"]
            else:
                os.environ["MF_TIME_LIMIT_S"] = old
        assert list(g.solve_batch(s[:3], t[:3])) == exp
        assert [g.solve(a, b)[0] for a, b in zip(s[:3], t[:3])] == exp


def test_session_admission_refused_before_allocating():
    """A session whose resident queries need more HBM than is free is
    refused with MF_ERR_NOMEM and its message, with nothing allocated."""
    import torch
    import mscresearch_b200 as mf
    from mscresearch_b200 import lib
    torch.cuda.set_device(0)
    n, u, v, c, s, t = _rmat(16, seed=9)
    with mf.Graph.from_edges(n, u, v, c, R=64) as g:
        free, _ = torch.cuda.mem_get_info()
        arcs = g.info[1]
        per = 8 * arcs + 40 * n  # a lower bound of one resident query's slot
        nq = int(free / per) + 64
        live0, bytes0 = C.c_longlong(), C.c_longlong()
        lib.mf_debug_alloc_live(C.byref(live0), C.byref(bytes0), None)
        ss = np.resize(s, nq)
        tt = np.resize(t, nq)
        with pytest.raises(mf.MaxflowError) as ei:
            mf.Session(g, ss, tt)
        assert ei.value.code == NOMEM and "admission" in str(ei.value)
        live1, bytes1 = C.c_longlong(), C.c_longlong()
        lib.mf_debug_alloc_live(C.byref(live1), C.byref(bytes1), None)
        assert (live1.value, bytes1.value) == (live0.value, bytes0.value)
        # a session that fits still works on the same graph
        with mf.Session(g, s[:2], t[:2]) as small:
            assert list(small.solve()) == _dinic(n, u, v, c, s[:2], t[:2])


def test_injected_allocation_failures_leave_nothing_allocated():
    """Every allocation made while creating a graph and solving a batch on
    it is made to fail in turn (the k-th allocation of the sequence reports
    out-of-memory without allocating).  Each such run returns MF_ERR_NOMEM,
    and once the graph is destroyed the engine holds exactly what it held
    before.  A final clean run gives the oracle's flows."""
    import torch
    import mscresearch_b200 as mf
    from mscresearch_b200 import lib
    torch.cuda.set_device(0)
    n, u, v, c, s, t = _rmat(12, seed=3)
    exp = _dinic(n, u, v, c, s, t)

    def live():
        a, b, k = C.c_longlong(), C.c_longlong(), C.c_longlong()
        lib.mf_debug_alloc_live(C.byref(a), C.byref(b), C.byref(k))
        return a.value, b.value, k.value

    base = live()[:2]
    failures = 0
    for k in range(400):
        lib.mf_debug_alloc_fail_after(k)
        g = sess = None
        rc, got = 0, None
        try:
            g = mf.Graph.from_edges(n, u, v, c, R=16)
            got = list(g.solve_batch(s, t))
            sess = mf.Session(g, s[:2], t[:2])
            assert list(sess.solve()) == exp[:2]
        except mf.MaxflowError as e:
            rc = e.code
        finally:
            if sess is not None:
                sess.close()
            if g is not None:
                g.close()
        left = live()
        lib.mf_debug_alloc_fail_after(-1)
        assert left[:2] == base, (k, left, base)
        if left[2] >= 0:
            # the countdown outlived the whole sequence: every allocation
            # point has been failed once
            assert rc == 0 and got == exp
            break
        assert rc == NOMEM, (k, rc)
        failures += 1
    else:
        pytest.fail("allocation sequence longer than 400")
    assert failures >= 10
    with mf.Graph.from_edges(n, u, v, c, R=16) as g:
        assert list(g.solve_batch(s, t)) == exp
