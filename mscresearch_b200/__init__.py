"""B200-native exact max-flow engine (Python view of the C ABI).

The product is the C ABI in include/maxflow_b200.h, implemented by the
in-tree CUDA library mscresearch_b200/libmfb200.so (hand-written sm_100a
kernels + C++ host code).  This module is a thin ctypes layer over it for
tests, benchmarks and Python callers; it never computes a flow itself.

Drop-in surface of the reference program
(Region_Aware_PR_with_Pruning_BoundaryCore.cu): graph.txt / test.txt in,
res_mt.txt "flow time_ms" out, static | dynamic modes — see
``mscresearch_b200/bin/maxflow_b200`` and :func:`run_cli`.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from . import _capi
from ._capi import MfOpts, MfStats, lib

__all__ = [
    "Graph", "Session", "Server", "MaxflowError", "opts", "stats_dict",
    "gen_uniform", "gen_rmat", "gen_grid", "gen_queries_hub",
    "write_graph_txt", "write_test_txt", "read_graph_txt", "run_cli", "CLI_PATH",
]

CLI_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "bin", "maxflow_b200")

MF_OK = 0
ERR_NAMES = {1: "ARG", 2: "CUDA", 3: "NOMEM", 4: "IO", 5: "ITER_LIMIT", 6: "TIMEOUT",
             7: "INEXACT", 8: "CERTIFY"}


class MaxflowError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("MF_ERR_%s (%d): %s" % (ERR_NAMES.get(code, "?"), code, msg))
        self.code = code


def _check(rc):
    if rc != MF_OK:
        raise MaxflowError(rc, lib.mf_last_error_string().decode(errors="replace"))


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def opts(**kw):
    """mf_opts with the defaults of mf_opts_default, overridden by kw."""
    o = MfOpts()
    lib.mf_opts_default(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


def stats_dict(st):
    return {name: getattr(st, name) for name, _ in MfStats._fields_}


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def _i64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64))


class Graph:
    """A device-resident graph (region-ordered paired-arc CSR)."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle)

    @classmethod
    def from_edges(cls, n, u, v, cap, R=128):
        u, v, cap = _i32(u), _i32(v), _i64(cap)
        h = C.c_void_p()
        _check(lib.mf_graph_create_from_edges(int(n), len(u), _p(u, C.c_int32), _p(v, C.c_int32),
                                              _p(cap, C.c_int64), int(R), C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_device_edges(cls, n, m, d_u, d_v, d_cap, R=128):
        """Edges already on the device: d_u, d_v, d_cap are device addresses
        (e.g. torch int32/int32/int64 CUDA tensors' data_ptr())."""
        h = C.c_void_p()
        _check(lib.mf_graph_create_from_device_edges(int(n), int(m), C.c_void_p(d_u), C.c_void_p(d_v),
                                                     C.c_void_p(d_cap), int(R), C.byref(h)))
        return cls(h.value)

    @classmethod
    def load(cls, path, R=128):
        h = C.c_void_p()
        _check(lib.mf_graph_load_file(path.encode(), int(R), C.byref(h)))
        return cls(h.value)

    @classmethod
    def load_binary(cls, path):
        h = C.c_void_p()
        _check(lib.mf_graph_load_binary(path.encode(), C.byref(h)))
        return cls(h.value)

    def save(self, path):
        _check(lib.mf_graph_save(self._h, path.encode()))

    def close(self):
        if self._h:
            lib.mf_graph_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def info(self):
        n, arcs, R = C.c_int(), C.c_longlong(), C.c_int()
        _check(lib.mf_graph_info(self._h, C.byref(n), C.byref(arcs), C.byref(R)))
        return n.value, arcs.value, R.value

    def export(self):
        n, arcs, R = self.info
        row = np.zeros(n + 1, np.int32)
        col = np.zeros(max(arcs, 1), np.int32)
        cap = np.zeros(max(arcs, 1), np.int64)
        rev = np.zeros(max(arcs, 1), np.int32)
        nid = np.zeros(n, np.int32)
        rs = np.zeros(R + 1, np.int32)
        score = np.zeros(n, np.float64)
        part = np.zeros(n, np.int32)
        _check(lib.mf_graph_export(self._h, _p(row, C.c_int32), _p(col, C.c_int32), _p(cap, C.c_int64),
                                   _p(rev, C.c_int32), _p(nid, C.c_int32), _p(rs, C.c_int32),
                                   _p(score, C.c_double), _p(part, C.c_int32)))
        return dict(row=row, col=col[:arcs], cap=cap[:arcs], rev=rev[:arcs], new_id=nid,
                    region_start=rs, score=score, part=part)

    def repartition(self, R):
        _check(lib.mf_graph_repartition(self._h, int(R)))

    def scc(self):
        """Strongly connected components of the edges with capacity > 0,
        computed on the GPU (SCC_CONTRACT/scc_contract.cpp's partition).
        Returns (comp, ncomp, (cu, cv, cap)): each vertex's component
        (numbered by smallest vertex id) and the contracted graph's arcs in
        increasing (cu, cv)."""
        n = self.info[0]
        comp = np.zeros(max(n, 1), np.int32)
        nc, mc = C.c_int32(), C.c_longlong()
        _check(lib.mf_graph_scc(self._h, _p(comp, C.c_int32), C.byref(nc), C.byref(mc)))
        k = mc.value
        cu, cv, cc = np.zeros(max(k, 1), np.int32), np.zeros(max(k, 1), np.int32), np.zeros(max(k, 1), np.int64)
        _check(lib.mf_graph_scc_contracted(self._h, _p(cu, C.c_int32), _p(cv, C.c_int32), _p(cc, C.c_int64),
                                           max(k, 1)))
        return comp[:n], nc.value, (cu[:k], cv[:k], cc[:k])

    def solve(self, s, t, o=None):
        f = C.c_int64()
        st = MfStats()
        _check(lib.mf_solve(self._h, int(s), int(t), C.byref(o or opts()), C.byref(f), C.byref(st)))
        return f.value, st

    def solve_batch(self, s, t, o=None, with_stats=False):
        s, t = _i32(s), _i32(t)
        nq = len(s)
        flows = np.zeros(nq, np.int64)
        sts = (MfStats * max(nq, 1))() if with_stats else None
        _check(lib.mf_solve_batch(self._h, nq, _p(s, C.c_int32), _p(t, C.c_int32), C.byref(o or opts()),
                                  _p(flows, C.c_int64), sts))
        return (flows, list(sts)[:nq]) if with_stats else flows

    def solve_batch_override(self, s, t, u, v, caps, o=None, with_stats=False):
        """Batch where query i gives arcs u[j]->v[j] the capacities caps[i, j]."""
        s, t, u, v = _i32(s), _i32(t), _i32(u), _i32(v)
        nq, nb = len(s), len(u)
        caps = np.ascontiguousarray(np.asarray(caps, np.int64).reshape(nq, nb))
        flows = np.zeros(nq, np.int64)
        sts = (MfStats * max(nq, 1))() if with_stats else None
        _check(lib.mf_solve_batch_override(self._h, nq, _p(s, C.c_int32), _p(t, C.c_int32), nb,
                                           _p(u, C.c_int32), _p(v, C.c_int32), _p(caps, C.c_int64),
                                           C.byref(o or opts()), _p(flows, C.c_int64), sts))
        return (flows, list(sts)[:nq]) if with_stats else flows

    @property
    def last_device_ms(self):
        return lib.mf_last_device_ms(self._h)

    def certify(self, s, t, o=None):
        f = C.c_int64()
        st = MfStats()
        rc = lib.mf_certify(self._h, int(s), int(t), C.byref(o or opts()), C.byref(f), C.byref(st))
        _check(rc)
        return f.value, st

    def prune_mask(self, s, t, mode=1, use_kept_cache=1):
        n = self.info[0]
        m = np.zeros(n, np.uint8)
        kept = C.c_int()
        _check(lib.mf_debug_prune_mask(self._h, int(s), int(t),
                                       C.byref(opts(prune_mode=mode, use_kept_cache=use_kept_cache)),
                                       _p(m, C.c_uint8), C.byref(kept)))
        return m

    def initial_heights(self, s, t, mode=1):
        n = self.info[0]
        h = np.zeros(n, np.int32)
        _check(lib.mf_debug_initial_heights(self._h, int(s), int(t), C.byref(opts(prune_mode=mode)),
                                            _p(h, C.c_int32)))
        return h

    def solve_residual(self, s, t, o=None):
        arcs = self.info[1]
        res = np.zeros(max(arcs, 1), np.int64)
        f = C.c_int64()
        st = MfStats()
        _check(lib.mf_solve_residual(self._h, int(s), int(t), C.byref(o or opts()), C.byref(f),
                                     _p(res, C.c_int64), C.byref(st)))
        return f.value, res[:arcs], st

    def update_caps(self, u, v, delta):
        u, v, d = _i32(u), _i32(v), _i64(delta)
        sk = C.c_int()
        _check(lib.mf_update_caps(self._h, len(u), _p(u, C.c_int32), _p(v, C.c_int32), _p(d, C.c_int64),
                                  C.byref(sk)))
        return sk.value

    def autotune(self, s, t, base=None):
        s, t = _i32(s), _i32(t)
        best = MfOpts()
        R = C.c_int()
        _check(lib.mf_autotune(self._h, len(s), _p(s, C.c_int32), _p(t, C.c_int32),
                               C.byref(base or opts()), C.byref(best), C.byref(R)))
        return best, R.value


class Session:
    """Resident queries whose residual state stays on the GPU across capacity updates."""

    def __init__(self, graph, s, t, o=None):
        self.graph = graph
        s, t = _i32(s), _i32(t)
        self.nq = len(s)
        h = C.c_void_p()
        _check(lib.mf_session_create(graph._h, self.nq, _p(s, C.c_int32), _p(t, C.c_int32),
                                     C.byref(o or opts()), C.byref(h)))
        self._h = h

    def solve(self):
        f = np.zeros(self.nq, np.int64)
        _check(lib.mf_session_solve(self._h, _p(f, C.c_int64), None))
        return f

    def update(self, u, v, delta, with_stats=False):
        u, v, d = _i32(u), _i32(v), _i64(delta)
        f = np.zeros(self.nq, np.int64)
        sts = (MfStats * max(self.nq, 1))() if with_stats else None
        _check(lib.mf_session_update(self._h, len(u), _p(u, C.c_int32), _p(v, C.c_int32), _p(d, C.c_int64),
                                     _p(f, C.c_int64), sts))
        return (f, list(sts)[:self.nq]) if with_stats else f

    def close(self):
        if self._h:
            lib.mf_session_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching server over several device-resident graphs."""

    def __init__(self, graphs, o=None, max_slots=0):
        self.graphs = list(graphs)
        arr = (C.c_void_p * len(self.graphs))(*[g._h.value for g in self.graphs])
        h = C.c_void_p()
        _check(lib.mf_server_create(arr, len(self.graphs), C.byref(o or opts()), int(max_slots), C.byref(h)))
        self._h = h

    @property
    def slots(self):
        n = C.c_int()
        _check(lib.mf_server_slots(self._h, C.byref(n)))
        return n.value

    def submit(self, graph, s, t):
        tk = C.c_longlong()
        _check(lib.mf_server_submit(self._h, int(graph), int(s), int(t), C.byref(tk)))
        return tk.value

    def update(self, graph, u, v, delta):
        """Enqueue a capacity-update batch on `graph`; returns its ticket."""
        u, v, d = _i32(u), _i32(v), _i64(delta)
        tk = C.c_longlong()
        _check(lib.mf_server_update(self._h, int(graph), len(u), _p(u, C.c_int32), _p(v, C.c_int32),
                                    _p(d, C.c_int64), C.byref(tk)))
        return tk.value

    def poll(self, ticket):
        done, f, lat, st = C.c_int(), C.c_int64(), C.c_double(), C.c_int()
        _check(lib.mf_server_poll(self._h, int(ticket), C.byref(done), C.byref(f), C.byref(lat), C.byref(st)))
        return (bool(done.value), f.value, lat.value, st.value)

    def drain(self):
        _check(lib.mf_server_drain(self._h))

    def close(self):
        if self._h:
            lib.mf_server_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- synthetic workloads ---------------------------------------------------

def gen_uniform(n, m, lo, hi, seed):
    u = np.zeros(m, np.int32)
    v = np.zeros(m, np.int32)
    c = np.zeros(m, np.int64)
    _check(lib.mf_gen_uniform(int(n), int(m), int(lo), int(hi), int(seed), _p(u, C.c_int32),
                              _p(v, C.c_int32), _p(c, C.c_int64)))
    return u, v, c


def gen_rmat(scale, m, a=0.57, b=0.19, c=0.19, lo=1, hi=1000, seed=1):
    u = np.zeros(m, np.int32)
    v = np.zeros(m, np.int32)
    cp = np.zeros(m, np.int64)
    kept = C.c_longlong()
    _check(lib.mf_gen_rmat(int(scale), int(m), a, b, c, int(lo), int(hi), int(seed), _p(u, C.c_int32),
                           _p(v, C.c_int32), _p(cp, C.c_int64), C.byref(kept)))
    k = kept.value
    return u[:k].copy(), v[:k].copy(), cp[:k].copy()


def gen_grid(W, H, seed):
    cap_len = 5 * W * H
    u = np.zeros(cap_len, np.int32)
    v = np.zeros(cap_len, np.int32)
    c = np.zeros(cap_len, np.int64)
    m = C.c_longlong()
    _check(lib.mf_gen_grid(int(W), int(H), int(seed), _p(u, C.c_int32), _p(v, C.c_int32),
                           _p(c, C.c_int64), C.byref(m)))
    k = m.value
    return u[:k].copy(), v[:k].copy(), c[:k].copy()


def gen_grid_terminal_sets(W, H, nq, seed, wmax=255):
    """Segmentation grid whose queries vary the terminal set: the graph holds
    the neighbour arcs of gen_grid plus S->p and p->T for every pixel p at
    capacity wmax; query i keeps one of the two per pixel (seeded mask) at a
    weight uniform in [0, wmax] and zeroes the other.  Returns the graph
    (n, u, v, cap), the overridden arcs (tu, tv) and caps[nq, 2*W*H]."""
    u, v, c = gen_grid(W, H, seed)
    S, T = W * H, W * H + 1
    nb = (u < S) & (v < S)
    px = np.arange(W * H, dtype=np.int32)
    tu = np.concatenate([np.full(W * H, S, np.int32), px])
    tv = np.concatenate([px, np.full(W * H, T, np.int32)])
    gu = np.concatenate([u[nb], tu])
    gv = np.concatenate([v[nb], tv])
    gc = np.concatenate([c[nb], np.full(2 * W * H, wmax, np.int64)])
    rng = np.random.default_rng(seed)
    caps = np.zeros((nq, 2 * W * H), np.int64)
    for i in range(nq):
        to_src = rng.integers(0, 2, W * H, dtype=np.int8).astype(bool)
        w = rng.integers(0, wmax + 1, W * H, dtype=np.int64)
        caps[i, :W * H] = np.where(to_src, w, 0)
        caps[i, W * H:] = np.where(to_src, 0, w)
    return W * H + 2, gu, gv, gc, tu, tv, caps


def gen_queries_hub(n, u, v, nhub, nuni, seed):
    u, v = _i32(u), _i32(v)
    s = np.zeros(nhub + nuni, np.int32)
    t = np.zeros(nhub + nuni, np.int32)
    _check(lib.mf_gen_queries_hub(int(n), len(u), _p(u, C.c_int32), _p(v, C.c_int32), int(nhub), int(nuni),
                                  int(seed), _p(s, C.c_int32), _p(t, C.c_int32)))
    return s, t


def write_graph_txt(path, n, u, v, cap):
    u, v, cap = _i32(u), _i32(v), _i64(cap)
    _check(lib.mf_write_graph_txt(path.encode(), int(n), len(u), _p(u, C.c_int32), _p(v, C.c_int32),
                                  _p(cap, C.c_int64)))


def write_test_txt(path, s, t):
    s, t = _i32(s), _i32(t)
    _check(lib.mf_write_test_txt(path.encode(), len(s), _p(s, C.c_int32), _p(t, C.c_int32)))


def read_graph_txt(path):
    n, m = C.c_int(), C.c_longlong()
    _check(lib.mf_graph_txt_header(path.encode(), C.byref(n), C.byref(m)))
    cap_len = max(m.value, 0)
    u = np.zeros(max(cap_len, 1), np.int32)
    v = np.zeros(max(cap_len, 1), np.int32)
    c = np.zeros(max(cap_len, 1), np.int64)
    got = C.c_longlong()
    _check(lib.mf_read_graph_txt(path.encode(), C.byref(n), C.byref(got), _p(u, C.c_int32), _p(v, C.c_int32),
                                 _p(c, C.c_int64), cap_len))
    k = got.value
    return n.value, u[:k].copy(), v[:k].copy(), c[:k].copy()


def run_cli(input_dir, output_dir, mode="static", extra=(), timeout=None):
    """Run the drop-in CLI; returns (returncode, stderr)."""
    r = subprocess.run([CLI_PATH, input_dir, output_dir, mode, *extra], capture_output=True,
                       text=True, timeout=timeout)
    return r.returncode, r.stderr
