"""Generates the golden fixtures under tests/golden/<case>/.

Each case directory holds the reference program's inputs (graph.txt,
test.txt, 1-based ids) and
  expected.txt   one flow per query from the oracle's Dinic solver;
  ref_res_mt.txt the reference CUDA program's own res_mt.txt for the same
                 inputs (flow time_ms), when produced with --with-ref on a
                 machine with a GPU and the reference build oracle/_ref/ra_ref
                 (oracle/build_ref.sh).  Only its flow column is used.
Inputs are seeded synthetic graphs made by the engine's generators (the
same ones the benchmark uses) plus small hand-written edge cases.

usage: python tests/golden/make_golden.py [--with-ref] [--only CASE]
"""
import argparse
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import mscresearch_b200 as mf  # noqa: E402  (generators only; host code, no GPU)
from oracle import oracle as O  # noqa: E402


def case_c1():
    # n=4096, m=32768 uniform, caps U[1,100], 16 uniform queries (s != t)
    u, v, c = mf.gen_uniform(4096, 32768, 1, 100, seed=1)
    rng = np.random.default_rng(11)
    s = rng.integers(0, 4096, 16)
    t = rng.integers(0, 4096, 16)
    t = np.where(t == s, (t + 1) % 4096, t)
    return 4096, u, v, c, s, t


def case_hand():
    # parallel + antiparallel arcs, a self loop, out-of-range ids, cap <= 0,
    # queries with s == t, invalid ids and unreachable sinks
    E = [(0, 1, 5), (0, 1, 3), (1, 0, 4), (1, 2, 6), (2, 2, 9), (0, 2, 2), (2, 3, 7),
         (3, 1, 1), (1, 3, 2), (4, 3, 8), (0, 9, 5), (-1, 2, 3), (2, 4, 0), (3, 4, -2),
         (5, 6, 10), (6, 5, 10), (0, 5, 1)]
    u = np.array([e[0] for e in E])
    v = np.array([e[1] for e in E])
    c = np.array([e[2] for e in E])
    s = np.array([0, 0, 3, 0, 2, 0, 4, 6, 1, 0])
    t = np.array([3, 2, 0, 0, 3, 6, 3, 5, 3, 4])
    return 8, u, v, c, s, t


def case_rmat():
    u, v, c = mf.gen_rmat(10, 8192, lo=1, hi=1000, seed=3)
    s, t = mf.gen_queries_hub(1 << 10, u, v, 8, 8, seed=5)
    return 1 << 10, u, v, c, s, t


def case_grid():
    W = H = 24
    u, v, c = mf.gen_grid(W, H, seed=7)
    S, T = W * H, W * H + 1
    s = np.array([S, S, 0, 5 * W + 3])
    t = np.array([T, 17 * W + 20, T, T])
    return W * H + 2, u, v, c, s, t


def case_chain():
    # a long path with side branches: deep relabel BFS, sparse active phase
    n = 600
    u, v, c = [], [], []
    for i in range(n - 1):
        u.append(i); v.append(i + 1); c.append(50 + (i * 37) % 100)
        if i % 7 == 0 and i + 3 < n:
            u.append(i); v.append(i + 3); c.append(5)
        if i % 11 == 0 and i > 2:
            u.append(i); v.append(i - 2); c.append(9)
    s = np.array([0, 0, 100, 599])
    t = np.array([599, 300, 500, 0])
    return n, np.array(u), np.array(v), np.array(c), s, t


def case_layered():
    # source -> layer A -> layer B -> sink with dense random bipartite middle
    rng = np.random.default_rng(21)
    a, b = 40, 40
    S, T = 0, 1 + a + b
    u, v, c = [], [], []
    for i in range(a):
        u.append(S); v.append(1 + i); c.append(int(rng.integers(10, 60)))
    for i in range(b):
        u.append(1 + a + i); v.append(T); c.append(int(rng.integers(10, 60)))
    for _ in range(600):
        i, j = int(rng.integers(0, a)), int(rng.integers(0, b))
        u.append(1 + i); v.append(1 + a + j); c.append(int(rng.integers(1, 20)))
        if rng.random() < 0.2:
            u.append(1 + a + j); v.append(1 + i); c.append(int(rng.integers(1, 20)))
    s = np.array([S, S, 1, T])
    t = np.array([T, 1 + a + 3, T, S])
    return T + 1, np.array(u), np.array(v), np.array(c), s, t


CASES = {
    "c1_uniform": case_c1,
    "hand_edge_cases": case_hand,
    "rmat_s10": case_rmat,
    "grid_24": case_grid,
    "chain_600": case_chain,
    "layered_80": case_layered,
}


def write_case(name, fn):
    d = os.path.join(HERE, name)
    os.makedirs(d, exist_ok=True)
    n, u, v, c, s, t = fn()
    # raw 1-based text exactly as the reference reads it (invalid ids kept)
    with open(os.path.join(d, "graph.txt"), "w") as f:
        f.write("%d %d\n" % (n, len(u)))
        for a, b, w in zip(u, v, c):
            f.write("%d %d %d\n" % (a + 1, b + 1, w))
    with open(os.path.join(d, "test.txt"), "w") as f:
        for a, b in zip(s, t):
            f.write("%d %d\n" % (a + 1, b + 1))
    n2, pu, pv, pc = O.parse_graph(os.path.join(d, "graph.txt"))
    g = O.build_csr(n2, pu, pv, pc)
    qs, qt = O.parse_queries(os.path.join(d, "test.txt"))
    flows = [O.dinic(g, a, b) if (0 <= a < n2 and 0 <= b < n2 and a != b) else 0 for a, b in zip(qs, qt)]
    with open(os.path.join(d, "expected.txt"), "w") as f:
        for x in flows:
            f.write("%d\n" % x)
    return d


def run_ref(d, timeout=300):
    """Run the reference program in static and dynamic mode; keep its result
    files and its per-query log lines (prune / upload sizes)."""
    if not os.path.exists(O.REF_BIN):
        raise SystemExit("reference build missing: run oracle/build_ref.sh first")
    ok = True
    for mode, res_name, out_name in (("static", "res_mt.txt", "ref_res_mt.txt"),
                                     ("dynamic", "res_dynamic.txt", "ref_res_dynamic.txt")):
        out = tempfile.mkdtemp()
        try:
            r = subprocess.run(["timeout", str(timeout), O.REF_BIN, d, out, mode], capture_output=True,
                               text=True)
            if r.returncode != 0:
                print("reference %s failed on %s (rc %d): %s" % (mode, d, r.returncode, r.stderr[-400:]))
                ok = False
                continue
            shutil.copy(os.path.join(out, res_name), os.path.join(d, out_name))
            keep = [l for l in r.stderr.splitlines()
                    if l.startswith("[QueryPrune") or l.startswith("[Static]") or l.startswith("[Dynamic] Query")
                    or l.startswith("Graph (") or l.startswith("Exceeded")]
            with open(os.path.join(d, "ref_log_%s.txt" % mode), "w") as f:
                f.write("\n".join(keep) + "\n")
        finally:
            shutil.rmtree(out, ignore_errors=True)
    return ok


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--with-ref", action="store_true")
    ap.add_argument("--only")
    a = ap.parse_args()
    for name, fn in CASES.items():
        if a.only and name != a.only:
            continue
        d = write_case(name, fn)
        if a.with_ref:
            run_ref(d)
        print("wrote", d)


if __name__ == "__main__":
    main()
