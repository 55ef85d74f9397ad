"""Strongly connected components and SCC contraction
(SCC_CONTRACT/scc_contract.cpp, "SC").

CPU: the oracle's Kosaraju restatement writes byte-identical files to the
reference tool's own outputs (tests/golden*/*/ref_scc.txt{,.map}, made by
tests/golden/make_scc_golden.py from the tool compiled out of its source),
and the CLI's two query-tool modes write byte-identical files to the
reference's convert_test_to_scc and split_queries_by_scc.
GPU: the device decomposition (mf_graph_scc, and the CLI's --scc-contract)
gives the reference's partition and, under the bijection between the two
numberings, its contracted graph; on larger seeded graphs, and after
capacity updates, the oracle's.
"""
import glob
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CASES = sorted(os.path.dirname(p) for p in glob.glob(os.path.join(ROOT, "tests", "golden*", "*", "ref_scc.txt")))
IDS = [os.path.basename(d) for d in CASES]


def _read_ref(d):
    with open(os.path.join(d, "ref_scc.txt")) as f:
        nc, mc = map(int, f.readline().split())
        arcs = [tuple(map(int, line.split())) for line in f]
    with open(os.path.join(d, "ref_scc.txt.map")) as f:
        comp = np.array([int(line.split()[1]) - 1 for line in f], np.int64)
    assert len(arcs) == mc
    return nc, comp, arcs


def _bijection(a, b):
    """The map a-label -> b-label if the two labellings are the same
    partition, else None."""
    m = {}
    inv = {}
    for x, y in zip(np.asarray(a).tolist(), np.asarray(b).tolist()):
        if m.setdefault(x, y) != y or inv.setdefault(y, x) != x:
            return None
    return m


def _check_against(n, comp, ncomp, contracted, ref_comp, ref_nc, ref_arcs):
    """Same partition, component count and contracted graph (ref_arcs are
    1-based (cu, cv, cap) triples) as the reference."""
    assert ncomp == ref_nc
    bij = _bijection(comp[:n], ref_comp[:n])
    assert bij is not None, "different partitions"
    cu, cv, cc = contracted
    mine = sorted((bij[int(a)] + 1, bij[int(b)] + 1, int(c)) for a, b, c in zip(cu, cv, cc))
    assert mine == sorted(ref_arcs)
    # the engine's own numbering: by smallest vertex id, arcs in (cu, cv) order
    first = {}
    for x, c in enumerate(np.asarray(comp[:n]).tolist()):
        first.setdefault(c, x)
    assert sorted(first, key=first.get) == list(range(ncomp))
    assert list(zip(cu.tolist(), cv.tolist())) == sorted(zip(cu.tolist(), cv.tolist()))


@pytest.mark.parametrize("d", CASES, ids=IDS)
def test_oracle_kosaraju_writes_the_reference_files(d, tmp_path):
    n, u, v, c = O.parse_graph(os.path.join(d, "graph.txt"))
    comp, nc = O.scc_kosaraju(n, u, v, c)
    cu, cv, cc = O.scc_contract(n, u, v, c, comp)
    out = str(tmp_path / "scc.txt")
    O.write_scc_files(out, n, comp, nc, cu, cv, cc)
    for suffix in ("", ".map"):
        with open(out + suffix, "rb") as a, open(os.path.join(d, "ref_scc.txt" + suffix), "rb") as b:
            assert a.read() == b.read(), suffix


def _queries(d):
    q = os.path.join(d, "test.txt")
    return q if os.path.exists(q) else os.path.join(d, "scc_queries.txt")


@pytest.mark.parametrize("d", CASES, ids=IDS)
def test_cli_query_tools_write_the_reference_files(d, tmp_path):
    """--scc-convert-test and --scc-split-queries (host text work, no device
    call) on each case's queries and the reference tool's map: byte for byte
    the files of SCC_CONTRACT/convert_test_to_scc.cpp and
    split_queries_by_scc.cpp, including ends out of range, 0 and negative."""
    import mscresearch_b200 as mf
    mp = os.path.join(d, "ref_scc.txt.map")
    a = str(tmp_path / "test_scc.txt")
    subprocess.run([mf.CLI_PATH, "--scc-convert-test", _queries(d), mp, a], check=True, capture_output=True)
    inter, intra = str(tmp_path / "inter.txt"), str(tmp_path / "intra.txt")
    subprocess.run([mf.CLI_PATH, "--scc-split-queries", _queries(d), mp, inter, intra], check=True,
                   capture_output=True)
    for mine, ref in ((a, "ref_scc_test.txt"), (inter, "ref_scc_inter.txt"), (intra, "ref_scc_intra.txt"),
                      (inter + ".index", "ref_scc_inter.txt.index")):
        with open(mine, "rb") as x, open(os.path.join(d, ref), "rb") as y:
            assert x.read() == y.read(), ref


def test_oracle_kosaraju_numbering_is_topological():
    """Kosaraju's second pass finds the components in a topological order of
    the condensation: every contracted arc goes from a lower to a higher id."""
    for d in CASES:
        _, comp, arcs = _read_ref(d)
        assert all(a < b for a, b, _ in arcs), d


@pytest.mark.gpu
@pytest.mark.parametrize("d", CASES, ids=IDS)
def test_device_scc_matches_reference_tool(d):
    import mscresearch_b200 as mf
    ref_nc, ref_comp, ref_arcs = _read_ref(d)
    with mf.Graph.load(os.path.join(d, "graph.txt"), R=8) as g:
        n = g.info[0]
        comp, nc, con = g.scc()
        _check_against(n, comp, nc, con, ref_comp, ref_nc, ref_arcs)


@pytest.mark.gpu
def test_cli_scc_contract_matches_reference_tool(tmp_path):
    import mscresearch_b200 as mf
    for d in CASES:
        out = str(tmp_path / (os.path.basename(d) + ".txt"))
        subprocess.run([mf.CLI_PATH, "--scc-contract", os.path.join(d, "graph.txt"), out], check=True,
                       capture_output=True)
        ref_nc, ref_comp, ref_arcs = _read_ref(d)
        with open(out) as f:
            nc, mc = map(int, f.readline().split())
            arcs = [tuple(map(int, line.split())) for line in f]
        comp = np.array([int(line.split()[1]) - 1 for line in open(out + ".map")], np.int64)
        assert mc == len(arcs) and nc == ref_nc
        bij = _bijection(comp, ref_comp)
        assert bij is not None, d
        assert sorted((bij[a - 1] + 1, bij[b - 1] + 1, c) for a, b, c in arcs) == sorted(ref_arcs), d


def _oracle_scc(n, u, v, c):
    comp, nc = O.scc_kosaraju(n, u, v, c)
    cu, cv, cc = O.scc_contract(n, u, v, c, comp)
    return comp, nc, [(int(a) + 1, int(b) + 1, int(x)) for a, b, x in zip(cu, cv, cc)]


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["rmat16", "rmat14_dense", "grid", "cycles"])
def test_device_scc_matches_oracle_on_larger_graphs(kind):
    import mscresearch_b200 as mf
    rng = np.random.default_rng(5)
    if kind == "rmat16":
        n = 1 << 16
        u, v, c = O.gen_rmat(16, 3 << 16, seed=7)
    elif kind == "rmat14_dense":
        n = 1 << 14
        u, v, c = O.gen_rmat(14, 16 << 14, seed=8)
    elif kind == "grid":
        # 300 x 300 grid, both directions, some arcs at capacity 0 (one-way
        # or cut links), a source row and a sink column
        w = 300
        n = w * w + 2
        ids = np.arange(w * w).reshape(w, w)
        a = np.concatenate([ids[:, :-1].ravel(), ids[:-1, :].ravel()])
        b = np.concatenate([ids[:, 1:].ravel(), ids[1:, :].ravel()])
        u = np.concatenate([a, b, np.full(w, w * w), ids[:, -1]])
        v = np.concatenate([b, a, ids[0, :], np.full(w, w * w + 1)])
        c = rng.integers(0, 4, len(u))
    else:
        n = 20000
        us, vs = [], []
        for _ in range(3000):
            k = int(rng.integers(2, 30))
            cyc = rng.integers(0, n, k)
            us.append(cyc)
            vs.append(np.roll(cyc, -1))
        u = np.concatenate(us + [rng.integers(0, n, 15000)])
        v = np.concatenate(vs + [rng.integers(0, n, 15000)])
        c = rng.integers(1, 9, len(u))
    ref_comp, ref_nc, ref_arcs = _oracle_scc(n, u, v, c)
    with mf.Graph.from_edges(n, u, v, c, R=32) as g:
        comp, nc, con = g.scc()
        _check_against(n, comp, nc, con, ref_comp, ref_nc, ref_arcs)


@pytest.mark.gpu
def test_device_scc_follows_capacity_updates():
    """Capacity updates that drop edges to 0 (or raise them from 0) change
    the components; mf_graph_scc reads the current capacities."""
    import mscresearch_b200 as mf
    rng = np.random.default_rng(9)
    n = 1 << 12
    u, v, c = O.gen_rmat(12, 8 << 12, seed=3)
    with mf.Graph.from_edges(n, u, v, c, R=16) as g:
        comp0, nc0, _ = g.scc()
        idx = rng.choice(len(u), 3000, replace=False)
        d = np.where(rng.random(3000) < 0.8, -2000, 5)
        g.update_caps(u[idx], v[idx], d)
        c2 = c.copy()
        # an update applies to the first edge u -> v of the input order
        first = {}
        for i, (a, b) in enumerate(zip(u.tolist(), v.tolist())):
            first.setdefault((a, b), i)
        for i, dd in zip(idx.tolist(), d.tolist()):
            j = first[(int(u[i]), int(v[i]))]
            c2[j] = max(0, c2[j] + dd)
        ref_comp, ref_nc, ref_arcs = _oracle_scc(n, u, v, c2)
        comp, nc, con = g.scc()
        assert nc != nc0
        _check_against(n, comp, nc, con, ref_comp, ref_nc, ref_arcs)
