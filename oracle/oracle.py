"""ctypes view of the CPU oracle (oracle/oracle.c) — TEST INFRASTRUCTURE ONLY.

Imported only by tests/, the smoke check in __graft_entry__.py and the
cpu_baseline leg of bench.py, as the checker.  The engine never uses it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "ra_ref")
REF_SCC_BIN = os.path.join(HERE, "_ref", "scc_contract")


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(
        os.path.getmtime(os.path.join(HERE, f)) for f in ("oracle.c", "gen.c", "scc.c")):
    build()
_lib = C.CDLL(LIB)

i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
u8p = C.POINTER(C.c_uint8)
f64p = C.POINTER(C.c_double)
_sig = {
    "or_parse_graph": (C.c_longlong, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_longlong), i32p, i32p, i64p, C.c_longlong]),
    "or_parse_queries": (C.c_longlong, [C.c_char_p, i32p, i32p, C.c_longlong]),
    "or_build_csr": (C.c_longlong, [C.c_int, C.c_longlong, i32p, i32p, i64p, i32p, i32p, i64p, i32p]),
    "or_degree_stats": (None, [C.c_int, i32p, i32p, i64p, i64p, i64p, i32p, i32p]),
    "or_det_log": (C.c_double, [C.c_double]),
    "or_score": (C.c_double, [C.c_longlong, C.c_longlong, C.c_int, C.c_int]),
    "or_partition": (None, [C.c_int, C.c_int, i64p, i64p, i32p, i32p, i32p, f64p]),
    "or_partition_libm": (None, [C.c_int, C.c_int, i64p, i64p, i32p, i32p, i32p, f64p]),
    "or_reorder": (None, [C.c_int, C.c_int, i32p, i32p, i32p, i64p, i32p, i32p, i32p, i32p, i32p, i32p, i64p, i32p]),
    "or_prune_mask": (C.c_int, [C.c_int, i32p, i32p, i64p, i32p, C.c_int, C.c_int, C.c_int, u8p]),
    "or_induced_subgraph": (C.c_longlong, [C.c_int, i32p, i32p, i64p, i32p, u8p, C.POINTER(C.c_int), i32p, i32p, i32p, i32p, i64p, i32p]),
    "or_boundary_core_mask": (C.c_int, [C.c_int, C.c_int, i32p, i32p, i32p, C.c_int, C.c_int, C.c_int, u8p]),
    "or_bfs_heights": (None, [C.c_int, i32p, i32p, i32p, i64p, C.c_int, u8p, u8p, i32p]),
    "or_dinic": (C.c_longlong, [C.c_int, i32p, i32p, i64p, i32p, C.c_int, C.c_int, i64p]),
    "or_dinic_batch": (None, [C.c_int, i32p, i32p, i64p, i32p, C.c_int, i32p, i32p, i64p, C.c_int]),
    "or_push_relabel": (C.c_longlong, [C.c_int, i32p, i32p, i64p, i32p, C.c_int, C.c_int, i64p]),
    "or_certify": (C.c_int, [C.c_int, i32p, i32p, i64p, i32p, C.c_int, C.c_int, i64p, C.c_longlong, C.c_int, C.POINTER(C.c_longlong)]),
    "gn_rmat": (C.c_longlong, [C.c_int, C.c_longlong, C.c_double, C.c_double, C.c_double, C.c_longlong, C.c_longlong,
                               C.c_uint64, i32p, i32p, i64p]),
    "gn_queries_hub": (C.c_int, [C.c_int, C.c_longlong, i32p, i32p, C.c_int, C.c_int, C.c_uint64, i32p, i32p]),
    "gn_write_graph_txt": (C.c_int, [C.c_char_p, C.c_int, C.c_longlong, i32p, i32p, i64p]),
    "gn_write_test_txt": (C.c_int, [C.c_char_p, C.c_int, i32p, i32p]),
    "or_scc_kosaraju": (C.c_int, [C.c_int, C.c_longlong, i32p, i32p, i64p, i32p]),
    "or_scc_contract": (C.c_longlong, [C.c_int, C.c_longlong, i32p, i32p, i64p, i32p, i32p, i32p, i64p]),
}
for _n, (_r, _a) in _sig.items():
    _f = getattr(_lib, _n)
    _f.restype = _r
    _f.argtypes = _a


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def _c(a, dt):
    return np.ascontiguousarray(np.asarray(a, dtype=dt))


class CSR:
    def __init__(self, n, row, col, cap, rev):
        self.n, self.row, self.col, self.cap, self.rev = n, row, col, cap, rev

    @property
    def arcs(self):
        return int(self.row[self.n])

    def args(self):
        return (self.n, _p(self.row, C.c_int32), _p(self.col, C.c_int32), _p(self.cap, C.c_int64),
                _p(self.rev, C.c_int32))


def parse_graph(path):
    with open(path) as f:
        head = f.readline().split()
    m = max(int(head[1]), 0) if len(head) >= 2 else 0
    u = np.zeros(max(m, 1), np.int32)
    v = np.zeros(max(m, 1), np.int32)
    c = np.zeros(max(m, 1), np.int64)
    n = C.c_int()
    mh = C.c_longlong()
    k = _lib.or_parse_graph(path.encode(), C.byref(n), C.byref(mh), _p(u, C.c_int32), _p(v, C.c_int32),
                            _p(c, C.c_int64), m)
    if k < 0:
        raise IOError(path)
    return n.value, u[:k] - 1, v[:k] - 1, c[:k]


def parse_queries(path, cap=1 << 20):
    s = np.zeros(cap, np.int32)
    t = np.zeros(cap, np.int32)
    k = _lib.or_parse_queries(path.encode(), _p(s, C.c_int32), _p(t, C.c_int32), cap)
    return s[:k] - 1, t[:k] - 1


def build_csr(n, u, v, cap):
    u, v, cap = _c(u, np.int32), _c(v, np.int32), _c(cap, np.int64)
    m = len(u)
    row = np.zeros(n + 1, np.int32)
    col = np.zeros(max(2 * m, 1), np.int32)
    cp = np.zeros(max(2 * m, 1), np.int64)
    rev = np.zeros(max(2 * m, 1), np.int32)
    arcs = _lib.or_build_csr(n, m, _p(u, C.c_int32), _p(v, C.c_int32), _p(cap, C.c_int64), _p(row, C.c_int32),
                             _p(col, C.c_int32), _p(cp, C.c_int64), _p(rev, C.c_int32))
    return CSR(n, row, col[:arcs].copy(), cp[:arcs].copy(), rev[:arcs].copy())


def degree_stats(g):
    n = g.n
    so = np.zeros(n, np.int64)
    si = np.zeros(n, np.int64)
    do = np.zeros(n, np.int32)
    di = np.zeros(n, np.int32)
    _lib.or_degree_stats(n, _p(g.row, C.c_int32), _p(g.col, C.c_int32), _p(g.cap, C.c_int64),
                         _p(so, C.c_int64), _p(si, C.c_int64), _p(do, C.c_int32), _p(di, C.c_int32))
    return so, si, do, di


def det_log(x):
    return _lib.or_det_log(float(x))


def partition(g, R):
    so, si, do, di = degree_stats(g)
    part = np.zeros(g.n, np.int32)
    score = np.zeros(g.n, np.float64)
    _lib.or_partition(g.n, R, _p(so, C.c_int64), _p(si, C.c_int64), _p(do, C.c_int32), _p(di, C.c_int32),
                      _p(part, C.c_int32), _p(score, C.c_double))
    return part, score


def partition_libm(g, R):
    """The partition with the reference's libm log (RA:1147-1151)."""
    so, si, do, di = degree_stats(g)
    part = np.zeros(g.n, np.int32)
    score = np.zeros(g.n, np.float64)
    _lib.or_partition_libm(g.n, R, _p(so, C.c_int64), _p(si, C.c_int64), _p(do, C.c_int32), _p(di, C.c_int32),
                           _p(part, C.c_int32), _p(score, C.c_double))
    return part, score


def reorder(g, R, part):
    n, A = g.n, g.arcs
    part = _c(part, np.int32)
    new_id = np.zeros(n, np.int32)
    old_id = np.zeros(n, np.int32)
    rs = np.zeros(R + 1, np.int32)
    row2 = np.zeros(n + 1, np.int32)
    col2 = np.zeros(max(A, 1), np.int32)
    cap2 = np.zeros(max(A, 1), np.int64)
    rev2 = np.zeros(max(A, 1), np.int32)
    _lib.or_reorder(n, R, _p(part, C.c_int32), *[_p(x, t) for x, t in (
        (g.row, C.c_int32), (g.col, C.c_int32), (g.cap, C.c_int64), (g.rev, C.c_int32),
        (new_id, C.c_int32), (old_id, C.c_int32), (rs, C.c_int32), (row2, C.c_int32),
        (col2, C.c_int32), (cap2, C.c_int64), (rev2, C.c_int32))])
    return CSR(n, row2, col2[:A].copy(), cap2[:A].copy(), rev2[:A].copy()), new_id, old_id, rs


def prune_mask(g, s, t, mode):
    m = np.zeros(g.n, np.uint8)
    _lib.or_prune_mask(*g.args(), int(s), int(t), int(mode), _p(m, C.c_uint8))
    return m


def induced_subgraph(g, mask):
    mask = _c(mask, np.uint8)
    n, A = g.n, g.arcs
    sub_n = C.c_int()
    o2s = np.zeros(n, np.int32)
    s2o = np.zeros(n, np.int32)
    row2 = np.zeros(n + 1, np.int32)
    col2 = np.zeros(max(A, 1), np.int32)
    cap2 = np.zeros(max(A, 1), np.int64)
    rev2 = np.zeros(max(A, 1), np.int32)
    arcs = _lib.or_induced_subgraph(*g.args(), _p(mask, C.c_uint8), C.byref(sub_n), _p(o2s, C.c_int32),
                                    _p(s2o, C.c_int32), _p(row2, C.c_int32), _p(col2, C.c_int32),
                                    _p(cap2, C.c_int64), _p(rev2, C.c_int32))
    k = sub_n.value
    return CSR(k, row2[:k + 1].copy(), col2[:arcs].copy(), cap2[:arcs].copy(), rev2[:arcs].copy()), o2s, s2o[:k].copy()


def boundary_core_mask(g, R, region_of, s, t, hop_limit=2):
    m = np.zeros(g.n, np.uint8)
    ro = _c(region_of, np.int32)
    _lib.or_boundary_core_mask(g.n, R, _p(g.row, C.c_int32), _p(g.col, C.c_int32), _p(ro, C.c_int32),
                               int(s), int(t), int(hop_limit), _p(m, C.c_uint8))
    return m


def bfs_heights(g, res, t, seed=None, blocked=None):
    res = _c(res, np.int64)
    d = np.zeros(g.n, np.int32)
    sd = None if seed is None else _p(_c(seed, np.uint8), C.c_uint8)
    bl = None if blocked is None else _p(_c(blocked, np.uint8), C.c_uint8)
    _lib.or_bfs_heights(g.n, _p(g.row, C.c_int32), _p(g.col, C.c_int32), _p(g.rev, C.c_int32),
                        _p(res, C.c_int64), int(t), sd, bl, _p(d, C.c_int32))
    return d


def dinic(g, s, t, want_res=False):
    res = np.zeros(max(g.arcs, 1), np.int64) if want_res else None
    f = _lib.or_dinic(*g.args(), int(s), int(t), _p(res, C.c_int64) if want_res else None)
    return (f, res[:g.arcs]) if want_res else f


def dinic_batch(g, s, t, threads=1):
    s, t = _c(s, np.int32), _c(t, np.int32)
    out = np.zeros(len(s), np.int64)
    _lib.or_dinic_batch(*g.args(), len(s), _p(s, C.c_int32), _p(t, C.c_int32), _p(out, C.c_int64), int(threads))
    return out


def push_relabel(g, s, t):
    return _lib.or_push_relabel(*g.args(), int(s), int(t), None)


def certify(g, s, t, res, value, require_flow=False):
    res = _c(res, np.int64)
    cut = C.c_longlong()
    rc = _lib.or_certify(*g.args(), int(s), int(t), _p(res, C.c_int64), int(value), int(require_flow),
                         C.byref(cut))
    return rc, cut.value


# ---- workload generators (the engine's seeded generators restated, gen.c) --

def gen_rmat(scale, m, a=0.57, b=0.19, c=0.19, lo=1, hi=1000, seed=1):
    u = np.zeros(max(m, 1), np.int32)
    v = np.zeros(max(m, 1), np.int32)
    cp = np.zeros(max(m, 1), np.int64)
    k = _lib.gn_rmat(int(scale), int(m), a, b, c, int(lo), int(hi), int(seed), _p(u, C.c_int32), _p(v, C.c_int32),
                     _p(cp, C.c_int64))
    if k < 0:
        raise ValueError("gn_rmat: bad arguments")
    return u[:k].copy(), v[:k].copy(), cp[:k].copy()


def gen_queries_hub(n, u, v, nhub, nuni, seed=1):
    u, v = _c(u, np.int32), _c(v, np.int32)
    s = np.zeros(max(nhub + nuni, 1), np.int32)
    t = np.zeros(max(nhub + nuni, 1), np.int32)
    if _lib.gn_queries_hub(int(n), len(u), _p(u, C.c_int32), _p(v, C.c_int32), int(nhub), int(nuni), int(seed),
                           _p(s, C.c_int32), _p(t, C.c_int32)) != 0:
        raise ValueError("gn_queries_hub: bad arguments")
    return s[:nhub + nuni].copy(), t[:nhub + nuni].copy()


def write_graph_txt(path, n, u, v, cap):
    u, v, cap = _c(u, np.int32), _c(v, np.int32), _c(cap, np.int64)
    if _lib.gn_write_graph_txt(path.encode(), int(n), len(u), _p(u, C.c_int32), _p(v, C.c_int32),
                               _p(cap, C.c_int64)) != 0:
        raise IOError(path)


def write_test_txt(path, s, t):
    s, t = _c(s, np.int32), _c(t, np.int32)
    if _lib.gn_write_test_txt(path.encode(), len(s), _p(s, C.c_int32), _p(t, C.c_int32)) != 0:
        raise IOError(path)


def scc_kosaraju(n, u, v, cap):
    """Component of every vertex (0-based, Kosaraju's discovery order;
    SCC_CONTRACT/scc_contract.cpp:43-96) and the number of components."""
    u, v, cap = _c(u, np.int32), _c(v, np.int32), _c(cap, np.int64)
    comp = np.zeros(max(n, 1), np.int32)
    k = _lib.or_scc_kosaraju(int(n), len(u), _p(u, C.c_int32), _p(v, C.c_int32), _p(cap, C.c_int64),
                             _p(comp, C.c_int32))
    if k < 0:
        raise MemoryError("or_scc_kosaraju")
    return comp[:n].copy(), int(k)


def scc_contract(n, u, v, cap, comp):
    """Contracted arcs (cu, cv, summed cap) in increasing (cu, cv) for the
    labelling comp (SCC_CONTRACT/scc_contract.cpp:98-128)."""
    u, v, cap, comp = _c(u, np.int32), _c(v, np.int32), _c(cap, np.int64), _c(comp, np.int32)
    m = max(len(u), 1)
    cu, cv, cc = np.zeros(m, np.int32), np.zeros(m, np.int32), np.zeros(m, np.int64)
    k = _lib.or_scc_contract(int(n), len(u), _p(u, C.c_int32), _p(v, C.c_int32), _p(cap, C.c_int64),
                             _p(comp, C.c_int32), _p(cu, C.c_int32), _p(cv, C.c_int32), _p(cc, C.c_int64))
    if k < 0:
        raise MemoryError("or_scc_contract")
    return cu[:k].copy(), cv[:k].copy(), cc[:k].copy()


def write_scc_files(path, n, comp, ncomp, cu, cv, cc):
    """The reference tool's two outputs: path ("n' m'" then "cu cv cap"
    lines, 1-based) and path + ".map" ("vertex component" lines, 1-based)."""
    with open(path, "w") as f:
        f.write("%d %d\n" % (ncomp, len(cu)))
        f.writelines("%d %d %d\n" % (a + 1, b + 1, c) for a, b, c in zip(cu.tolist(), cv.tolist(), cc.tolist()))
    with open(path + ".map", "w") as f:
        f.writelines("%d %d\n" % (i + 1, x + 1) for i, x in enumerate(np.asarray(comp)[:n].tolist()))
