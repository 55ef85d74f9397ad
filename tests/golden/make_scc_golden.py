"""Generates the SCC-contraction golden fixtures.

For every graph.txt under tests/golden/<case>/ and tests/golden_scc/<case>/
it runs the reference's own SCC tool (SCC_CONTRACT/scc_contract.cpp,
compiled from its source into oracle/_ref/scc_contract by
oracle/build_ref.sh) and keeps its two outputs beside the graph:
  ref_scc.txt      the contracted graph ("n' m'", then "cu cv cap", 1-based)
  ref_scc.txt.map  "vertex component" per vertex, 1-based
The cases under tests/golden_scc/ are made here first: seeded graphs rich in
non-trivial components (overlapping random cycles joined by one-way edges,
with parallel edges, self loops, zero or negative capacities and ids out of
range, which the reader skips) and a sparse R-MAT, each with a query file
scc_queries.txt (pairs in range, ends out of range, 0 and negative).
The reference's two query tools (convert_test_to_scc.cpp,
split_queries_by_scc.cpp, also compiled by oracle/build_ref.sh) then run on
every case's queries (test.txt, or scc_queries.txt) against its
ref_scc.txt.map; their outputs are kept as ref_scc_test.txt,
ref_scc_inter.txt (+ .index) and ref_scc_intra.txt.

usage: python tests/golden/make_scc_golden.py
"""
import glob
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
SCC_DIR = os.path.join(ROOT, "tests", "golden_scc")
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402


def write_raw(path, n, u, v, c):
    """graph.txt with 1-based ids exactly as given (invalid ones included)."""
    with open(path, "w") as f:
        f.write("%d %d\n" % (n, len(u)))
        f.writelines("%d %d %d\n" % (a + 1, b + 1, x) for a, b, x in zip(u.tolist(), v.tolist(), c.tolist()))


def case_cycles(seed=3, n=3000):
    rng = np.random.default_rng(seed)
    us, vs = [], []
    for _ in range(260):  # random cycles over random vertices (they overlap and merge)
        k = int(rng.integers(2, 14))
        cyc = rng.integers(0, n, k)
        us.append(cyc)
        vs.append(np.roll(cyc, -1))
    us.append(rng.integers(0, n, 2200))  # one-way joins
    vs.append(rng.integers(0, n, 2200))
    u, v = np.concatenate(us), np.concatenate(vs)
    c = rng.integers(1, 50, len(u))
    # parallel edges, self loops, non-positive capacities, ids out of range
    dup = rng.integers(0, len(u), 300)
    u, v, c = np.concatenate([u, u[dup]]), np.concatenate([v, v[dup]]), np.concatenate([c, c[dup] + 1])
    extra = 200
    su = rng.integers(0, n, extra)
    u = np.concatenate([u, su, rng.integers(0, n, extra), rng.integers(n, n + 5, 20), rng.integers(0, n, 20)])
    v = np.concatenate([v, su, rng.integers(0, n, extra), rng.integers(0, n, 20), -rng.integers(2, 6, 20)])
    c = np.concatenate([c, rng.integers(1, 9, extra), rng.integers(-3, 1, extra), np.ones(40, np.int64)])
    p = rng.permutation(len(u))
    return n, u[p], v[p], c[p]


def case_rmat12():
    u, v, c = O.gen_rmat(12, 3 << 12, seed=12)
    return 1 << 12, u, v, c


def main():
    ref = O.REF_SCC_BIN
    if not os.path.exists(ref):
        sys.exit("build the reference SCC tool first: oracle/build_ref.sh <reference root>")
    for name, fn in (("cycles_3000", case_cycles), ("rmat12_sparse", case_rmat12)):
        d = os.path.join(SCC_DIR, name)
        os.makedirs(d, exist_ok=True)
        n, u, v, c = fn()
        write_raw(os.path.join(d, "graph.txt"), n, u, v, c)
        rng = np.random.default_rng(len(name))
        q = rng.integers(1, n + 1, (200, 2))
        q[:6] = [[0, 5], [5, 0], [-3, 4], [4, n + 1], [n, n], [1, 1]]
        with open(os.path.join(d, "scc_queries.txt"), "w") as f:
            f.writelines("%d %d\n" % (a, b) for a, b in q.tolist())
    graphs = sorted(glob.glob(os.path.join(HERE, "*", "graph.txt")) + glob.glob(os.path.join(SCC_DIR, "*", "graph.txt")))
    ref_dir = os.path.dirname(ref)
    for g in graphs:
        d = os.path.dirname(g)
        out = os.path.join(d, "ref_scc.txt")
        subprocess.run([ref, g, out], check=True, stderr=subprocess.DEVNULL)
        print(os.path.relpath(out, ROOT), open(out).readline().strip())
        qf = os.path.join(d, "test.txt")
        if not os.path.exists(qf):
            qf = os.path.join(d, "scc_queries.txt")
        subprocess.run([os.path.join(ref_dir, "convert_test_to_scc"), qf, out + ".map",
                        os.path.join(d, "ref_scc_test.txt")], check=True, stderr=subprocess.DEVNULL)
        subprocess.run([os.path.join(ref_dir, "split_queries_by_scc"), qf, out + ".map",
                        os.path.join(d, "ref_scc_inter.txt"), os.path.join(d, "ref_scc_intra.txt")],
                       check=True, stderr=subprocess.DEVNULL)


if __name__ == "__main__":
    main()
