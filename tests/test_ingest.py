"""Graph ingest: the device tokenizer of graph.txt, the device CSR build and
the binary CSR cache.

CPU part: the tokenizer's per-byte rule (an integer starts at a sign followed
by a digit, or at a digit preceded by neither a digit nor a sign; the stream
ends at the first byte that is neither white space, a digit, nor a sign
followed by a digit), restated here in numpy, against the oracle's fscanf
reader on fuzzed files.  GPU part: mf_graph_load_file / from_device_edges /
the cache against graphs built from the oracle reader's edges, array for
array."""
import os

import numpy as np
import pytest

from oracle import oracle as O

TRICKY = [
    "5 6\n1 2 3\n  2   3\n4\n4 5 -7\n3 z 1\n1 5 2\n",          # stops at 'z'
    "4 5\n1 2 3\n2 3 4\n3 x 1\n3 4 5\n",                      # stops at 'x'
    "4 3\r\n1 2 3\r\n2 3 4\r\n3 4 5\r\n",                     # CRLF
    "4 9\t1\t2\t3 2 3 4\n\n\n3 4 5",                          # tabs, no final newline
    "4 3\n1 2 +3\n2 3 4-1\n3 4 5\n",                          # "4-1" scans as 4, -1
    "4 3\n1 2 3\n2 3 4\n3 4 5\n1 2 9\n",                      # more triples than m
    "4 9\n1 2 3\n2 3 4\n3 4",                                 # incomplete last triple
    "4 4\n1 2 3\n2 3 - 4\n3 4 5\n",                           # lone sign
    "4 4\n1 2 3\n2 3 ++4\n3 4 5\n",                           # double sign
    "4 4\n1 2 3\n2 3 007\n3 4 5\n",                           # leading zeros
    "4 4\n1 1 3\n0 2 3\n2 9 4\n2 3 0\n3 4 5\n",               # dropped by the build rules
    "4 4\n1 2 3\n2 3 4\n3 4 5\n\x00 1 2 3\n",                 # NUL ends the stream
    "6 0\n1 2 3\n",                                           # m = 0
    "4 3\n1 2 99999999999999999999999\n2 3 -99999999999999999999\n3 4 5\n",  # saturation
    "4 2\n4294967298 3 5\n-4294967295 2 7\n",                 # ids keep the low 32 bits
]


def model_tokens(data):
    """The device rule, restated: the integers of the fscanf token stream."""
    b = np.frombuffer(data, np.uint8).astype(np.int32)
    S = len(b)
    sp = (b == 32) | ((b >= 9) & (b <= 13))
    dg = (b >= 48) & (b <= 57)
    sg = (b == 43) | (b == 45)
    nx_dg = np.zeros(S, bool)
    nx_dg[:-1] = dg[1:]
    pv_dg = np.zeros(S, bool)
    pv_dg[1:] = dg[:-1]
    pv_sg = np.zeros(S, bool)
    pv_sg[1:] = sg[:-1]
    sgn_ok = sg & nx_dg
    bad = ~sp & ~dg & ~sgn_ok
    start = sgn_ok | (dg & ~pv_dg & ~pv_sg)
    end = int(np.argmax(bad)) if bad.any() else S
    toks = []
    for i in np.nonzero(start[:end])[0]:
        j, neg = i, False
        if sg[j]:
            neg = b[j] == 45
            j += 1
        x = 0
        while j < S and dg[j]:
            x = x * 10 + int(b[j] - 48)
            j += 1
        x = -x if neg else x
        toks.append(min(max(x, -(1 << 63)), (1 << 63) - 1))   # strtoll saturates
    return toks


def model_edges(data):
    t = model_tokens(data)
    if len(t) < 2:
        return None
    n, m = t[0], t[1]
    k = min(max(m, 0), (len(t) - 2) // 3)
    e = np.array(t[2:2 + 3 * k], np.int64).reshape(k, 3)
    # "%d" stores the long value into an int (low 32 bits)
    ids = e[:, :2].astype(np.int32)
    return int(np.int64(n).astype(np.int32)), ids[:, 0] - np.int32(1), ids[:, 1] - np.int32(1), e[:, 2]


def _check_model(tmp_path, text):
    p = tmp_path / "graph.txt"
    p.write_bytes(text.encode("latin-1") if isinstance(text, str) else text)
    n, u, v, c = O.parse_graph(str(p))
    got = model_edges(p.read_bytes())
    assert got is not None
    assert got[0] == n
    assert list(got[1]) == list(u) and list(got[2]) == list(v) and list(got[3]) == list(c)
    # the library's host reader (mf_read_graph_txt) follows the same rules
    import mscresearch_b200 as mf
    n2, u2, v2, c2 = mf.read_graph_txt(str(p))
    assert n2 == n and list(u2) == list(u) and list(v2) == list(v) and list(c2) == list(c)


@pytest.mark.parametrize("i", range(len(TRICKY)))
def test_tokenizer_rule_matches_fscanf_reader(tmp_path, i):
    _check_model(tmp_path, TRICKY[i])


def test_tokenizer_rule_fuzz(tmp_path):
    rng = np.random.default_rng(7)
    alpha = list(" \t\n\r+-0123456789") + ["x"]
    w = np.array([6, 1, 3, 1, 1, 1] + [2] * 10 + [0.05])
    w = w / w.sum()
    for trial in range(300):
        body = "".join(rng.choice(alpha, int(rng.integers(0, 80)), p=w))
        _check_model(tmp_path, "7 %d\n%s" % (int(rng.integers(0, 12)), body))


def model_csr(n, u, v, c):
    """The device CSR build, restated: half-arcs h = 2i + side keyed by their
    tail (n for dropped edges), stably sorted; positions give the arcs."""
    u, v, c = np.asarray(u, np.int64), np.asarray(v, np.int64), np.asarray(c, np.int64)
    m = len(u)
    kept = (u >= 0) & (u < n) & (v >= 0) & (v < n) & (u != v) & (c > 0)
    key = np.empty(2 * m, np.int64)
    key[0::2] = np.where(kept, u, n)
    key[1::2] = np.where(kept, v, n)
    order = np.argsort(key, kind="stable")
    arcs = int(2 * kept.sum())
    h = order[:arcs]
    pos = np.empty(2 * m, np.int64)
    pos[h] = np.arange(arcs)
    i, back = h >> 1, (h & 1) == 1
    col = np.where(back, u[i], v[i])
    cap = np.where(back, 0, c[i])
    rev = pos[h ^ 1]
    row = np.searchsorted(key[order], np.arange(n + 1), side="left")
    return row, col, cap, rev


def test_half_arc_sort_reproduces_reader_order():
    """A stable sort of half-arcs by tail gives exactly the arc order of the
    reference reader's build loop (the oracle's build_csr), dropped edges,
    parallel arcs and hubs included."""
    import mscresearch_b200 as mf
    for scale, m, seed in ((8, 3000, 1), (11, 40000, 2)):
        n = 1 << scale
        u, v, c = mf.gen_rmat(scale, m, seed=seed)
        u, v, c = u.copy(), v.copy(), c.copy()
        rng = np.random.default_rng(seed)
        k = rng.integers(0, len(u), 60)
        c[k[:20]] = 0
        u[k[20:40]] = v[k[20:40]]
        v[k[40:]] = n + 5
        g = O.build_csr(n, u, v, c)
        row, col, cap, rev = model_csr(n, u, v, c)
        assert np.array_equal(row, g.row) and np.array_equal(col, g.col)
        assert np.array_equal(cap, g.cap) and np.array_equal(rev, g.rev)


# ---- GPU --------------------------------------------------------------------

def _same_graph(a, b):
    ea, eb = a.export(), b.export()
    for k in ("row", "col", "cap", "rev", "new_id", "region_start", "score", "part"):
        assert np.array_equal(ea[k], eb[k]), k


@pytest.mark.gpu
@pytest.mark.parametrize("i", range(len(TRICKY)))
def test_device_load_equals_oracle_reader(tmp_path, i):
    import mscresearch_b200 as mf
    p = tmp_path / "graph.txt"
    p.write_bytes(TRICKY[i].encode("latin-1"))
    n, u, v, c = O.parse_graph(str(p))
    with mf.Graph.load(str(p), R=2) as g, mf.Graph.from_edges(n, u, v, c, R=2) as h:
        _same_graph(g, h)


@pytest.mark.gpu
def test_device_load_rejects_bad_headers(tmp_path):
    import mscresearch_b200 as mf
    for text in ("", "   \n", "x 3\n1 2 3\n", "0 3\n1 2 3\n", "5 -1\n1 2 3\n", "5\n"):
        p = tmp_path / "graph.txt"
        p.write_text(text)
        with pytest.raises(mf.MaxflowError):
            mf.Graph.load(str(p))
    with pytest.raises(mf.MaxflowError):
        mf.Graph.load(str(tmp_path / "missing.txt"))


@pytest.mark.gpu
def test_device_csr_matches_oracle_build():
    """Device CSR + partition == the oracle's build + reorder (R-MAT with
    parallel arcs, dropped edges, hubs)."""
    import mscresearch_b200 as mf
    u, v, c = mf.gen_rmat(14, 200000, seed=5)
    rng = np.random.default_rng(1)
    k = rng.integers(0, len(u), 500)
    c = c.copy()
    c[k[:250]] = 0                      # dropped: cap <= 0
    u = u.copy()
    u[k[250:]] = v[k[250:]]             # dropped: self loops
    n = 1 << 14
    g0 = O.build_csr(n, u, v, c)
    part, score = O.partition(g0, 64)
    g2, new_id, old_id, rs = O.reorder(g0, 64, part)
    with mf.Graph.from_edges(n, u, v, c, R=64) as g:
        ex = g.export()
        assert np.array_equal(ex["row"], g2.row) and np.array_equal(ex["col"], g2.col)
        assert np.array_equal(ex["cap"], g2.cap) and np.array_equal(ex["rev"], g2.rev)
        assert np.array_equal(ex["new_id"], new_id)


@pytest.mark.gpu
def test_from_device_edges_equals_host_edges():
    import torch
    import mscresearch_b200 as mf
    u, v, c = mf.gen_uniform(3000, 40000, 1, 50, seed=3)
    du = torch.from_numpy(u).cuda()
    dv = torch.from_numpy(v).cuda()
    dc = torch.from_numpy(c).cuda()
    torch.cuda.synchronize()
    with mf.Graph.from_device_edges(3000, len(u), du.data_ptr(), dv.data_ptr(), dc.data_ptr(), R=16) as g, \
            mf.Graph.from_edges(3000, u, v, c, R=16) as h:
        _same_graph(g, h)
        s, t = [0, 5, 17], [2999, 6, 400]
        assert list(g.solve_batch(s, t)) == list(h.solve_batch(s, t))


@pytest.mark.gpu
def test_binary_cache_round_trip_and_rejects(tmp_path):
    import mscresearch_b200 as mf
    u, v, c = mf.gen_rmat(13, 100000, seed=8)
    n = 1 << 13
    p = str(tmp_path / "g.mfb")
    with mf.Graph.from_edges(n, u, v, c, R=32) as g:
        g.save(p)
        s, t = mf.gen_queries_hub(n, u, v, 4, 4, seed=3)
        exp = list(g.solve_batch(s, t))
        with mf.Graph.load_binary(p) as h:
            _same_graph(g, h)
            assert h.info == g.info
            assert list(h.solve_batch(s, t)) == exp
            assert [h.solve(a, b)[0] for a, b in zip(s, t)] == exp
    raw = bytearray(open(p, "rb").read())
    bad = tmp_path / "bad.mfb"
    for mutate in ("truncate", "magic", "rev", "permutation"):
        b = bytearray(raw)
        if mutate == "truncate":
            b = b[:-5]
        elif mutate == "magic":
            b[0] ^= 1
        elif mutate == "rev":
            hdr = 40
            nn = int.from_bytes(b[12:16], "little")
            A = int.from_bytes(b[16:24], "little")
            off = hdr + 4 * (nn + 1) + 4 * A + 8 * A      # rev[0]
            x = int.from_bytes(b[off:off + 4], "little")
            b[off:off + 4] = ((x + 1) % A).to_bytes(4, "little")
        else:
            nn = int.from_bytes(b[12:16], "little")
            A = int.from_bytes(b[16:24], "little")
            R = int.from_bytes(b[24:28], "little")
            off = 40 + 4 * (nn + 1) + 17 * A + 4 * (R + 1) + 4 * nn   # new_id[0]
            b[off:off + 4] = b[off + 4:off + 8]
        bad.write_bytes(bytes(b))
        with pytest.raises(mf.MaxflowError):
            mf.Graph.load_binary(str(bad))


@pytest.mark.gpu
def test_full_size_text_load_equals_edges(tmp_path):
    """R-MAT 2^20 written as graph.txt and loaded through the device
    tokenizer: the same graph as the edge-array build, and the load time."""
    import time
    import mscresearch_b200 as mf
    u, v, c = mf.gen_rmat(20, 1 << 24, seed=1)
    n = 1 << 20
    p = str(tmp_path / "graph.txt")
    mf.write_graph_txt(p, n, u, v, c)
    with mf.Graph.from_edges(n, u, v, c, R=128) as h:
        t0 = time.perf_counter()
        g = mf.Graph.load(p, R=128)
        dt = time.perf_counter() - t0
        with g:
            _same_graph(g, h)
            cp = str(tmp_path / "g.mfb")
            g.save(cp)
            t1 = time.perf_counter()
            with mf.Graph.load_binary(cp) as k:
                dt2 = time.perf_counter() - t1
                _same_graph(k, h)
    print("graph.txt %.1f MB: device load %.3f s; binary cache load %.3f s" % (
        os.path.getsize(p) / 1e6, dt, dt2))


@pytest.mark.gpu
def test_cli_csr_cache(tmp_path):
    """The CLI with --csr-cache: the first run builds from graph.txt and
    writes the cache, the second loads it; both give the expected answers."""
    import glob
    import mscresearch_b200 as mf
    golden = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    d = sorted(x for x in glob.glob(os.path.join(golden, "*")) if os.path.isdir(x))[0]
    exp = np.loadtxt(os.path.join(d, "expected.txt"), dtype=np.int64, ndmin=1)
    cache = str(tmp_path / "g.mfb")
    for k in range(2):
        out = str(tmp_path / ("out%d" % k))
        rc, err = mf.run_cli(d, out, "static", ("--csr-cache", cache), timeout=600)
        assert rc == 0, err[-2000:]
        res = np.loadtxt(os.path.join(out, "res_mt.txt"), dtype=np.int64, ndmin=2)
        assert list(res[:, 0]) == list(exp)
        assert os.path.exists(cache)
