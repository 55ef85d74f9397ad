"""Benchmark: exact max-flow queries/s (+ p50/p99 latency), batched vs plain,
on the R-MAT power-law workload (n = 2^20, 2^24 draws with
(a,b,c,d) = (0.57,0.19,0.19,0.05), self loops dropped, capacities uniform
in [1,1000], R = 128 regions, 256 queries: 128 between top-1% out-degree
and top-1% in-degree vertices, 128 uniform; seeded synthetic data).

One step = one batched persistent launch solving all 256 queries exactly
(mf_solve_batch) on a device-resident graph.  `value` is device-timed
(CUDA events around the launch, on its stream); `e2e` is the host clock
around the same public C-ABI calls from host buffers (query upload, answers
and per-query records back), in the same steps, so e2e >= value's time.
The graph (~0.9 GB) and the per-query residual slots (~0.3 GB each) exceed
the 126 MB L2, so no L2 flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

--impl reference runs the reference's own CUDA program (built from its
sources by oracle/build_ref.sh into oracle/_ref/ra_ref) on the same graph
and a bounded sample of the same queries, and reports its own per-query
times (res_mt.txt, integer ms, prune included, RA:2808).
Multi-GPU (torchrun): queries shard across ranks (one graph replica per
GPU, no data-path collective); timing is the max over ranks.

A full 1-GPU headline run also runs the three other workloads below, each
in its own process after the headline measurement, and appends their
figures to its line as "other_workloads" (--no-other skips them, and so
does --no-cpu, which marks a measurement-only run such as a profiling one).

Other workloads (their own lines when run alone):
  --workload mix       8 device-resident R-MAT graphs (2^14..2^20) served to
                       Poisson-arriving requests, against the plain loop;
  --workload gridsets  a 2048 x 2048 segmentation grid, 64 queries that vary
                       the terminal set (mf_solve_batch_override), relabel
                       frequency, group size and R tuned on 16 of the sets;
  --workload dynamic   R-MAT 2^22 with 32 resident queries: 1k/10k/100k
                       capacity-update batches, incremental repair against a
                       fresh batched solve.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "exact max-flow queries/sec + p50/p99 latency, batched vs plain, same B200"
WORKLOAD = "rmat20_256q"
SCALE, DRAWS, NHUB, NUNI, R = 20, 1 << 24, 128, 128, 128
GRAPH_SEED, QUERY_SEED = 1, 2
QOUT_BYTES = 208  # device per-query record copied back by mf_solve_batch


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, gpu=0):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu),
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 6:
                continue
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except ValueError:
                continue
            for nm, val in zip(names, f[2:6]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_workload(rank=0, scale=SCALE, nhub=NHUB, nuni=NUNI):
    import mscresearch_b200 as mf
    u, v, c = mf.gen_rmat(scale, 16 << scale, 0.57, 0.19, 0.19, 1, 1000, GRAPH_SEED)
    n = 1 << scale
    s, t = mf.gen_queries_hub(n, u, v, nhub, nuni, QUERY_SEED + 1000 * rank)
    return n, u, v, c, s, t


def pct(xs, q):
    return float(np.percentile(np.asarray(xs, dtype=np.float64), q)) if len(xs) else None


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return rank, world


def dist_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_baseline(n, u, v, c, s, t, budget_s=20.0):
    """Oracle Dinic on the box's host cores over a bounded sample of the same
    queries (hub and uniform alternating), queries spread over threads."""
    from oracle import oracle as O
    t0 = time.time()
    g = O.build_csr(n, u, v, c)
    build_s = time.time() - t0
    threads = os.cpu_count() or 1
    order = [i for pair in zip(range(NHUB), range(NHUB, NHUB + NUNI)) for i in pair]
    done, flows, t_solve = 0, [], 0.0
    k = max(threads, 4)
    while done < len(order) and t_solve < budget_s:
        idx = order[done:done + k]
        t1 = time.time()
        flows += list(O.dinic_batch(g, s[idx], t[idx], threads))
        t_solve += time.time() - t1
        done += len(idx)
    # the same solver on one core, over the first queries of the sample
    one, t_one = 0, 0.0
    while one < done and t_one < budget_s / 4:
        t1 = time.time()
        O.dinic_batch(g, s[order[one:one + 1]], t[order[one:one + 1]], 1)
        t_one += time.time() - t1
        one += 1
    return {"value": done / t_solve, "unit": "queries/s", "cores": threads, "kind": "port",
            "value_1core": (one / t_one) if t_one > 0 else None,
            "sample": "%d of the 256 queries (alternating hub/uniform), C Dinic over %d threads, "
                      "%.1f s solve (+%.1f s CSR build); 1 core: first %d of them, %.1f s" % (
                          done, threads, t_solve, build_s, one, t_one)}, \
        order[:done], flows


def run_engine(args):
    rank, world = dist_init(args)
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    import mscresearch_b200 as mf
    n, u, v, c, s, t = make_workload(rank, args.scale, args.nhub, args.nuni)
    g = mf.Graph.from_edges(n, u, v, c, R=R)
    _, arcs, _ = g.info
    o = mf.opts(group_ctas=args.group)
    if args.K:
        o.kernel_cycles = args.K
    if args.threads:
        o.threads = args.threads
    for kv in args.opt:
        k, v = kv.split("=", 1)
        setattr(o, k, type(getattr(o, k))(float(v)) if isinstance(getattr(o, k), float) else int(v))
    if args.gr_freq:
        o.gr_freq = args.gr_freq
    if args.gr_alpha is not None:
        o.gr_work_alpha = args.gr_alpha
    nq = len(s)
    # warm-up (also sizes the residual slot pool)
    for _ in range(args.warmup):
        g.solve_batch(s, t, o)
    # ---- timed region: each step is one public C-ABI call from host arrays
    # (queries up, answers and per-query records back); `value` takes the
    # batched launch's device time (CUDA events on its stream, the inputs
    # resident), `e2e` the host time of the whole call, in the same steps
    dev_ms, e2e_ms, stats_last = [], [], None
    s_host, t_host = np.ascontiguousarray(s), np.ascontiguousarray(t)
    dist_barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for k in range(args.steps):
            t0 = time.perf_counter()
            flows, sts = g.solve_batch(s_host, t_host, o, with_stats=True)
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
            dev_ms.append(g.last_device_ms)
            stats_last = sts
    torch.cuda.synchronize()
    dist_barrier(world)
    step_ms = dist_max(float(np.mean(dev_ms)), world)
    total_q = nq * world
    value = total_q / (step_ms / 1e3)
    e2e_step = dist_max(float(np.mean(e2e_ms)), world)
    # ---- plain per-query solver on the same queries (drop-in path)
    plain_ms, plain_flows, plain_st = [], [], []
    if not args.no_plain:
        for a, b in zip(s, t):
            f, st = g.solve(a, b)
            plain_ms.append(st.time_ms)
            plain_flows.append(f)
            plain_st.append(st)
        assert list(plain_flows) == list(flows), "plain and batched answers differ"
    plain_total = dist_max(float(np.sum(plain_ms)), world) if plain_ms else None
    # ---- served: Poisson arrivals at ~60% of batched capacity
    served = None
    if args.serve:
        served = serve_run(mf, g, s, t, flows, o, rate=0.6 * nq / (step_ms / 1e3))
    # ---- every answer certified on the device, outside the timed region:
    # excess returned to s (zero-excess flow), residuals non-negative and
    # pair-conserved, s-t cut capacity equal to the flow
    certified = None
    if not args.no_certify:
        oc = type(o).from_buffer_copy(o)
        oc.certify = 1
        try:
            cfl, cst = g.solve_batch(s, t, oc, with_stats=True)
            ok = sum(1 for f, st in zip(cfl, cst) if st.status == 0 and st.cut_capacity == f)
            certified = {"queries": nq, "certified": ok, "flows_equal_timed": bool(list(cfl) == list(flows))}
        except mf.MaxflowError as e:
            certified = {"queries": nq, "certified": None, "error": str(e)}
    # roofline: algorithmic bytes = 16 B x (arc + vertex examinations)
    ax = sum(x.arcs_examined for x in stats_last)
    vx = sum(x.vertices_examined for x in stats_last)
    alg_bytes = 16.0 * (ax + vx)
    # implementation-independent reference figure: what a classic top-down
    # relabel reads (every kept arc once per global relabel performed); the
    # direction-optimizing search reads less
    full_scan_bytes = 16.0 * sum(x.mask_arcs * x.global_relabels for x in stats_last)
    hbm, kind = peaks()
    achieved = alg_bytes / (np.mean(dev_ms) / 1e3) / 1e9
    # DRAM traffic of one batched launch, from the committed ncu capture of
    # the same workload (null for other workload sizes)
    traffic = None
    tp = os.path.join(ROOT, "profiles", "mf_kernel_rmat20_traffic.json")
    workload = "rmat%d_%dq" % (args.scale, nq)
    if os.path.exists(tp):
        tj = json.load(open(tp))
        if tj.get("workload") == workload:
            traffic = tj.get("bytes_per_launch")
    edges = sum(x.mask_arcs for x in stats_last)
    finish = [x.finish_ms for x in stats_last]
    res = {
        "metric": METRIC, "value": round(value, 3), "unit": "queries/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(step_ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic (seeded R-MAT 2^20, 2^24 draws, caps U[1,1000]; 128 hub + 128 uniform queries)",
        "config": {"workload": "rmat%d_%dq" % (args.scale, nq), "n": n, "edges": len(u), "arcs": arcs, "queries_per_gpu": nq,
                   "R": R, "prune": "fwd(s) & bwd(t)", "group_ctas": o.group_ctas,
                   "K": o.kernel_cycles, "threads": o.threads or 512, "gr_freq": o.gr_freq, "gr_alpha": o.gr_work_alpha,
                   "opt": list(args.opt),
                   "l2": "inputs larger than L2 (graph %.2f GB, residual slot %.2f GB)" % (
                       arcs * 20 / 1e9, arcs * 8 / 1e9),
                   "parallelism": "query shards, graph replica per GPU"},
        "e2e": {"value": round(total_q / (e2e_step / 1e3), 3), "unit": "queries/s",
                "h2d_bytes_per_step": 12 * nq, "d2h_bytes_per_step": QOUT_BYTES * nq + 8},
        "gpu_launches": 2 * args.steps,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": hbm, "unit": "GB/s",
                     "frac": round(achieved / hbm, 4), "traffic": traffic,
                     "peak_kind": kind, "alg_bytes_per_launch": alg_bytes,
                     "relabel_full_scan_bytes_per_launch": full_scan_bytes,
                     "traffic_gbs": (round(traffic / (np.mean(dev_ms) / 1e3) / 1e9, 1) if traffic else None),
                     "traffic_frac": (round(traffic / (np.mean(dev_ms) / 1e3) / 1e9 / hbm, 4) if traffic else None)},
        "batched": {"qps": round(value, 3), "p50_ms": pct(finish, 50), "p99_ms": pct(finish, 99),
                    "edges_per_s": edges / (np.mean(dev_ms) / 1e3)},
        "plain": {"qps": round(total_q / (plain_total / 1e3), 3) if plain_total else None,
                  "p50_ms": pct(plain_ms, 50), "p99_ms": pct(plain_ms, 99)},
        "clocks": clk.summary(),
    }
    if served:
        res["served"] = served
    if certified:
        res["certified"] = certified
    if rank == 0 and world == 1 and not args.no_cpu:
        cb, idx, cflows = cpu_baseline(n, u, v, c, s, t, budget_s=args.cpu_budget)
        assert [int(flows[i]) for i in idx] == [int(x) for x in cflows], "engine differs from oracle"
        res["cpu_baseline"] = cb
        res["oracle_agreement"] = "%d of %d sampled answers equal to the oracle's Dinic" % (len(idx), len(idx))
    if rank == 0 and world == 1 and not args.no_other and not args.no_cpu:
        res["other_workloads"] = other_workloads(args)
    if rank == 0:
        print(json.dumps(res), flush=True)
    if args.dump and rank == 0:
        keys = ["flow", "mask_vertices", "mask_arcs", "rounds", "global_relabels", "arcs_examined",
                "vertices_examined", "pushes", "path_push_rounds", "hot_sweeps", "rm_fixed", "service_ms",
                "finish_ms", "prune_ms", "relabel_ms", "rounds_ms", "relabel_arcs", "hub_arcs", "hub_passes", "hub_relabels", "levels", "levels_bottom_up", "levels_solo"]
        with open(args.dump, "w") as f:
            for i, x in enumerate(stats_last):
                row = {k: getattr(x, k) for k in keys}
                row.update(q=i, s=int(s[i]), t=int(t[i]), plain_ms=plain_ms[i] if plain_ms else None)
                if plain_st:
                    row.update(plain_rounds=plain_st[i].rounds, plain_relabels=plain_st[i].global_relabels,
                               plain_arcs=plain_st[i].arcs_examined, plain_prune_ms=plain_st[i].prune_ms,
                               plain_relabel_ms=plain_st[i].relabel_ms, plain_rounds_ms=plain_st[i].rounds_ms)
                f.write(json.dumps(row) + "\n")
    g.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


OTHER_KEYS = {
    "gridsets": ["metric", "value", "unit", "ms_per_step", "e2e", "roofline", "oracle_agreement"],
    "dynamic": ["metric", "value", "unit", "initial_exact", "batches"],
    "mix": ["metric", "value", "unit", "plain", "served", "served_with_updates"],
}


def other_workloads(args):
    """The three other workload shapes, each run as its own process after the
    headline measurement (outside its timed region; a failure there is
    recorded, not raised): their own JSON lines, trimmed to the figures."""
    out = {}
    for wl, keys in OTHER_KEYS.items():
        cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--workload", wl, "--no-cpu"]
        t0 = time.perf_counter()
        try:
            p = subprocess.run(cmd, capture_output=True, text=True, timeout=args.other_timeout)
            lines = [x for x in p.stdout.splitlines() if x.startswith("{")]
            if p.returncode != 0 or not lines:
                out[wl] = {"error": "exit %d: %s" % (p.returncode, (p.stderr or "").strip()[-300:])}
                continue
            d = json.loads(lines[-1])
            out[wl] = {k: d[k] for k in keys if k in d}
        except subprocess.TimeoutExpired:
            out[wl] = {"error": "no result within %d s" % args.other_timeout}
        out[wl]["wall_s"] = round(time.perf_counter() - t0, 1)
    return out


def serve_run(mf, g, s, t, flows, o, rate, nreq=256, seed=0):
    """Continuous batching: requests arrive by a Poisson process; latency is
    host-measured from submission to the answer being visible.  The server
    is warmed first (one burst of the queries, drained, untimed), so that
    its residual slots are admitted as in a server that has been running."""
    sv = mf.Server([g], o)
    warm = [sv.submit(0, int(a), int(b)) for a, b in zip(s, t)]
    sv.drain()
    assert [sv.poll(tk)[1] for tk in warm] == [int(f) for f in flows], "warm-up answers differ"
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, nreq)
    idx = rng.integers(0, len(s), nreq)
    sub_t, tickets = [], []
    t0 = time.perf_counter()
    nxt = t0
    done_t = {}
    for k in range(nreq):
        nxt += gaps[k]
        while time.perf_counter() < nxt:
            for tk in tickets:
                if tk not in done_t and sv.poll(tk)[0]:
                    done_t[tk] = time.perf_counter()
        sub_t.append(time.perf_counter())
        tickets.append(sv.submit(0, int(s[idx[k]]), int(t[idx[k]])))
    while len(done_t) < nreq:
        for tk in tickets:
            if tk not in done_t and sv.poll(tk)[0]:
                done_t[tk] = time.perf_counter()
    wall = time.perf_counter() - t0
    lat = [(done_t[tk] - sub_t[i]) * 1e3 for i, tk in enumerate(tickets)]
    exact = all(sv.poll(tk)[1] == int(flows[idx[i]]) for i, tk in enumerate(tickets))
    slots = sv.slots
    sv.close()
    assert exact, "served answers differ from the batched ones"
    return {"arrival_rate_qps": round(rate, 2), "requests": nreq, "qps": round(nreq / wall, 3),
            "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99), "slots": slots, "exact": exact,
            "warmed": "one untimed burst of the %d queries admitted the server's slots first" % len(s)}


MIX_SCALES = [14, 15, 16, 16, 17, 18, 19, 20]


def run_mix(args):
    """Serving mix: 8 device-resident R-MAT graphs of uneven size (n = 2^14 ..
    2^20, average out-degree 16, caps U[1,1000]), requests whose graph is
    drawn Zipf(1.1) over a seeded ranking and whose (s, t) is uniform.  The
    plain per-query loop is timed first (its answers are the reference for
    exactness); then Poisson streams at rates swept around its throughput go
    through the continuous-batching server."""
    rank = int(os.environ.get("RANK", "0"))
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    import mscresearch_b200 as mf
    rng = np.random.default_rng(1234)
    graphs, sizes, edges = [], [], []
    for k, sc in enumerate(MIX_SCALES):
        n = 1 << sc
        u, v, c = mf.gen_rmat(sc, 16 * n, seed=100 + k)
        graphs.append(mf.Graph.from_edges(n, u, v, c, R=min(128, n)))
        sizes.append(n)
        edges.append((u, v, c))
    ranks = rng.permutation(len(graphs))
    w = 1.0 / np.arange(1, len(graphs) + 1) ** 1.1
    p_graph = np.zeros(len(graphs))
    p_graph[ranks] = w / w.sum()
    nreq = args.mix_requests
    gi = rng.choice(len(graphs), nreq, p=p_graph)
    qs = np.array([rng.integers(0, sizes[g]) for g in gi], np.int32)
    qt = np.array([rng.integers(0, sizes[g]) for g in gi], np.int32)
    same = qs == qt
    qt[same] = (qt[same] + 1) % np.array(sizes)[gi[same]]
    o = mf.opts(group_ctas=args.group)
    for g in graphs:  # kept-set caches, slot pools
        g.solve_batch(qs[:4] % g.info[0], qt[:4] % g.info[0], o)
    # plain per-query loop (drop-in path): one whole-GPU solve per request
    plain_ms, plain_f = [], []
    t0 = time.perf_counter()
    for g, a, b in zip(gi, qs, qt):
        f, st = graphs[g].solve(int(a), int(b))
        plain_f.append(f)
        plain_ms.append(st.time_ms)
    plain_wall = time.perf_counter() - t0
    plain_qps = nreq / plain_wall
    runs = []
    for mult in args.mix_rates:
        rate = mult * plain_qps
        sv = mf.Server(graphs, o)
        gaps = rng.exponential(1.0 / rate, nreq)
        sub_t, tickets, done_t = [], [], {}
        t0 = time.perf_counter()
        nxt = t0
        for k in range(nreq):
            nxt += gaps[k]
            while time.perf_counter() < nxt:
                for tk in tickets:
                    if tk not in done_t and sv.poll(tk)[0]:
                        done_t[tk] = time.perf_counter()
            sub_t.append(time.perf_counter())
            tickets.append(sv.submit(int(gi[k]), int(qs[k]), int(qt[k])))
        while len(done_t) < nreq:
            for tk in tickets:
                if tk not in done_t and sv.poll(tk)[0]:
                    done_t[tk] = time.perf_counter()
        wall = time.perf_counter() - t0
        lat = [(done_t[tk] - sub_t[i]) * 1e3 for i, tk in enumerate(tickets)]
        exact = all(sv.poll(tk)[1] == int(plain_f[i]) for i, tk in enumerate(tickets))
        slots = sv.slots
        sv.close()
        runs.append({"arrival_rate_qps": round(rate, 1), "qps": round(nreq / wall, 2),
                     "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99), "slots": slots, "exact": exact})
    # served with capacity updates: ~10% of the requests are update batches
    # (256 changes of +-U[1,100] on random edges of the request's graph),
    # the rest queries, at twice the plain loop's rate.  Every answer is
    # checked against an in-order replay on a second copy of the graphs
    # (mf_update_caps then mf_solve, in submission order).
    upd_run = None
    if args.mix_update_share > 0:
        rate = 2.0 * plain_qps
        kinds = rng.random(nreq) < args.mix_update_share
        batches = {}
        for k in np.nonzero(kinds)[0]:
            u, v, c = edges[gi[k]]
            idx = rng.integers(0, len(u), 256)
            d = rng.integers(1, 101, 256) * np.where(rng.random(256) < 0.5, -1, 1)
            batches[k] = (u[idx], v[idx], d)
        sv = mf.Server(graphs, o)
        gaps = rng.exponential(1.0 / rate, nreq)
        sub_t, tickets, done_t = [], [], {}
        t0 = time.perf_counter()
        nxt = t0
        for k in range(nreq):
            nxt += gaps[k]
            while time.perf_counter() < nxt:
                for tk in tickets:
                    if tk not in done_t and sv.poll(tk)[0]:
                        done_t[tk] = time.perf_counter()
            sub_t.append(time.perf_counter())
            if kinds[k]:
                tickets.append(sv.update(int(gi[k]), *batches[k]))
            else:
                tickets.append(sv.submit(int(gi[k]), int(qs[k]), int(qt[k])))
        while len(done_t) < nreq:
            for tk in tickets:
                if tk not in done_t and sv.poll(tk)[0]:
                    done_t[tk] = time.perf_counter()
        wall = time.perf_counter() - t0
        served_f = [sv.poll(tk)[1] for tk in tickets]
        slots = sv.slots
        sv.close()
        # replay
        replay = []
        for k, (u, v, c) in enumerate(edges):
            replay.append(mf.Graph.from_edges(sizes[k], u, v, c, R=min(128, sizes[k])))
        exact = True
        for k in range(nreq):
            if kinds[k]:
                replay[gi[k]].update_caps(*batches[k])
            elif replay[gi[k]].solve(int(qs[k]), int(qt[k]))[0] != served_f[k]:
                exact = False
        for g in replay:
            g.close()
        qlat = [(done_t[tk] - sub_t[i]) * 1e3 for i, tk in enumerate(tickets) if not kinds[i]]
        ulat = [(done_t[tk] - sub_t[i]) * 1e3 for i, tk in enumerate(tickets) if kinds[i]]
        upd_run = {"arrival_rate_rps": round(rate, 1), "requests": nreq, "update_batches": int(kinds.sum()),
                   "changes_per_batch": 256, "rps": round(nreq / wall, 2),
                   "query_p50_ms": pct(qlat, 50), "query_p99_ms": pct(qlat, 99),
                   "update_p50_ms": pct(ulat, 50), "update_p99_ms": pct(ulat, 99), "slots": slots,
                   "exact": exact}
        assert exact, "served answers with updates differ from the in-order replay"
    best = max(runs, key=lambda r: r["qps"])
    res = {"metric": "exact max-flow queries/sec + p50/p99 latency, serving mix vs plain loop",
           "value": best["qps"], "unit": "queries/s", "n_gpus": 1, "higher_is_better": True,
           "dtype": "int64",
           "data": "synthetic (8 seeded R-MAT graphs, n = 2^14..2^20, out-degree 16, caps U[1,1000]; "
                   "graph choice Zipf(1.1), (s,t) uniform; Poisson arrivals)",
           "config": {"workload": "serving_mix_8rmat", "graph_scales": MIX_SCALES, "requests": nreq,
                      "group_ctas": o.group_ctas},
           "plain": {"qps": round(plain_qps, 2), "p50_ms": pct(plain_ms, 50), "p99_ms": pct(plain_ms, 99)},
           "served": runs}
    if upd_run:
        res["served_with_updates"] = upd_run
    for g in graphs:
        g.close()
    if rank == 0:
        print(json.dumps(res), flush=True)


# (gr_freq, gr_work_alpha, CTAs per query group) tried on a sample of the sets
GRID_TUNE = [(16, 0.35, 8), (4, 0.35, 8), (1, 0.35, 8), (64, 2.0, 8), (16, 0.35, 4), (16, 0.35, 16)]


def run_gridsets(args):
    """Segmentation grid W x W (4-connected, neighbour caps
    1 + floor(255 exp(-d^2/50)), d ~ N(0, 40)) with queries that vary the
    terminal set: each of the nq queries keeps S->p or p->T per pixel (seeded
    mask) at a weight uniform in [0, 255].  One step = one
    mf_solve_batch_override launch over all sets, the terminal capacities
    resident on the device; gr_freq / gr_work_alpha, the group size, R and
    the prune are tuned on a sample of the sets before timing (R orders the
    vertices: within a region they keep the input's row-major order)."""
    rank = int(os.environ.get("RANK", "0"))
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    import mscresearch_b200 as mf
    W, nq = args.grid_w, args.grid_sets
    n, gu, gv, gc, tu, tv, caps = mf.gen_grid_terminal_sets(W, W, nq, seed=9 + 1000 * rank)
    S, T = W * W, W * W + 1
    s = np.full(nq, S, np.int32)
    t = np.full(nq, T, np.int32)
    g = mf.Graph.from_edges(n, gu, gv, gc, R=R)
    _, arcs, _ = g.info
    # tuning (untimed): relabel frequency and group size on a sample of the
    # sets, then R.  A sample launch runs ceil(smp / groups) waves of queries
    # and the batch ceil(nq / groups), so the sample time is scaled by that
    # ratio (groups = resident CTAs / G) to compare group sizes.
    smp = min(16, nq)
    ctas = 2 * torch.cuda.get_device_properties(0).multi_processor_count
    tune = []
    best_o, best_ms, best_R = None, None, R

    def est(ms, G):
        gr = max(1, ctas // G)
        return ms * (-(-nq // gr)) / (-(-smp // gr))

    for gf, al, G in GRID_TUNE:
        o = mf.opts(group_ctas=G, gr_freq=gf, gr_work_alpha=al)
        g.solve_batch_override(s[:smp], t[:smp], tu, tv, caps[:smp], o)
        ms = est(g.last_device_ms, G)
        tune.append({"gr_freq": gf, "gr_alpha": al, "G": G, "R": R, "batch_ms_est": round(ms, 2)})
        if best_ms is None or ms < best_ms:
            best_o, best_ms = o, ms
    # then R (it orders the vertices) with each prune: fwd(s) & bwd(t)
    # (default) or every vertex kept
    for r in (R, 1, 8, 32, 512):
        if g.info[2] != r:
            g.repartition(r)
        for pm in (1, 2):
            if r == R and pm == best_o.prune_mode:
                continue  # measured above
            o2 = type(best_o).from_buffer_copy(best_o)
            o2.prune_mode = pm
            g.solve_batch_override(s[:smp], t[:smp], tu, tv, caps[:smp], o2)
            ms = est(g.last_device_ms, o2.group_ctas)
            tune.append({"gr_freq": o2.gr_freq, "gr_alpha": o2.gr_work_alpha, "G": o2.group_ctas, "R": r,
                         "prune_mode": pm, "batch_ms_est": round(ms, 2)})
            if ms < best_ms:
                best_o, best_ms, best_R = o2, ms, r
    if g.info[2] != best_R:
        g.repartition(best_R)
    o = best_o
    for _ in range(args.warmup):
        g.solve_batch_override(s, t, tu, tv, caps, o)
    dev_ms, e2e_ms = [], []
    torch.cuda.synchronize()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for k in range(args.steps):
            t0 = time.perf_counter()
            flows, sts = g.solve_batch_override(s, t, tu, tv, caps, o, with_stats=True)
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
            dev_ms.append(g.last_device_ms)
    torch.cuda.synchronize()
    step_ms = float(np.mean(dev_ms))
    ax = sum(x.arcs_examined for x in sts)
    vx = sum(x.vertices_examined for x in sts)
    hbm, kind = peaks()
    alg_bytes = 16.0 * (ax + vx)
    finish = [x.finish_ms for x in sts]
    res = {"metric": "exact max-flow queries/sec, grid terminal sets", "value": round(nq / (step_ms / 1e3), 3),
           "unit": "queries/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(step_ms, 3), "higher_is_better": True, "dtype": "int64",
           "data": "synthetic (seeded %dx%d grid, neighbour caps 1+floor(255 exp(-d^2/50)), d~N(0,40); "
                   "per-query terminal masks, weights U[0,255])" % (W, W),
           "config": {"workload": "grid%d_%dsets" % (W, nq), "n": n, "arcs": arcs, "queries": nq,
                      "R": best_R, "gr_freq": o.gr_freq, "gr_alpha": o.gr_work_alpha, "group_ctas": o.group_ctas,
                      "prune_mode": o.prune_mode, "overridden_arcs": len(tu), "tuning": tune,
                      "l2": "inputs larger than L2 (capacities %.2f GB)" % (caps.nbytes / 1e9)},
           "e2e": {"value": round(nq / (float(np.mean(e2e_ms)) / 1e3), 3), "unit": "queries/s",
                   "h2d_bytes_per_step": int(caps.nbytes + 8 * len(tu) + 8 * nq),
                   "d2h_bytes_per_step": QOUT_BYTES * nq + 4},
           "gpu_launches": 3 * args.steps,
           "roofline": {"bound": "hbm", "achieved": round(alg_bytes / (step_ms / 1e3) / 1e9, 2), "peak": hbm,
                        "unit": "GB/s", "frac": round(alg_bytes / (step_ms / 1e3) / 1e9 / hbm, 4),
                        "traffic": None, "peak_kind": kind, "alg_bytes_per_launch": alg_bytes},
           "batched": {"p50_ms": pct(finish, 50), "p99_ms": pct(finish, 99),
                       "global_relabels": int(sum(x.global_relabels for x in sts)),
                       "rounds": int(sum(x.rounds for x in sts)),
                       "per_query_mean": {k: round(float(np.mean([getattr(x, k) for x in sts])), 2) for k in (
                           "service_ms", "prune_ms", "relabel_ms", "rounds_ms", "rounds", "global_relabels",
                           "levels", "levels_bottom_up", "levels_solo", "arcs_examined", "relabel_arcs",
                           "vertices_examined", "pushes", "mask_vertices", "mask_arcs")}},
           "clocks": clk.summary()}
    if not args.no_cpu and rank == 0:
        # oracle Dinic on a graph built for each sampled terminal set
        from oracle import oracle as O
        nbr = len(gu) - len(tu)
        t0, k, ok = time.time(), 0, 0
        while k < nq and time.time() - t0 < args.cpu_budget:
            keep = caps[k] > 0
            go = O.build_csr(n, np.concatenate([gu[:nbr], tu[keep]]), np.concatenate([gv[:nbr], tv[keep]]),
                             np.concatenate([gc[:nbr], caps[k][keep]]))
            ok += int(O.dinic(go, S, T) == int(flows[k]))
            k += 1
        el = time.time() - t0
        res["cpu_baseline"] = {"value": round(k / el, 4), "unit": "queries/s", "cores": 1, "kind": "port",
                               "sample": "first %d sets: CSR build + C Dinic each, %.1f s" % (k, el)}
        res["oracle_agreement"] = "%d of %d sampled answers equal to the oracle's Dinic" % (ok, k)
    g.close()
    if rank == 0:
        print(json.dumps(res), flush=True)


def run_dynamic(args):
    """Dynamic updates: R-MAT n = 2^22, 2^26 draws, caps U[1,1000]; 32
    resident queries (16 hub, 16 uniform) in one session; batches of 1k, 10k
    and 100k seeded capacity changes (+-U[1,100], clamped at 0), each applied
    to the graph and followed by the incremental repair of every resident
    query (mf_session_update), every answer checked against a fresh batched
    solve of the same queries on the updated graph."""
    rank = int(os.environ.get("RANK", "0"))
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    import mscresearch_b200 as mf
    scale = 22
    u, v, c = mf.gen_rmat(scale, 1 << (scale + 4), 0.57, 0.19, 0.19, 1, 1000, 5)
    n = 1 << scale
    s, t = mf.gen_queries_hub(n, u, v, 16, 16, 6 + 1000 * rank)
    rng = np.random.default_rng(7)
    g = mf.Graph.from_edges(n, u, v, c, R=R)
    _, arcs, _ = g.info
    o = mf.opts(group_ctas=args.group)
    g.solve_batch(s, t, o)  # kept-set cache and slots
    ss = mf.Session(g, s, t, o)
    t0 = time.perf_counter()
    f0 = ss.solve()
    solve_wall = (time.perf_counter() - t0) * 1e3
    exact0 = list(f0) == list(g.solve_batch(s, t, o))
    runs = []
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for k in (1000, 10000, 100000):
            idx = rng.integers(0, len(u), k)
            d = rng.integers(1, 101, k) * rng.choice([-1, 1], k)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            fr = ss.update(u[idx], v[idx], d)
            upd_wall = (time.perf_counter() - t0) * 1e3
            rep_ms = g.last_device_ms
            fresh = g.solve_batch(s, t, o)
            fresh_ms = g.last_device_ms
            runs.append({"updates": k, "update_and_repair_wall_ms": round(upd_wall, 2),
                         "repair_device_ms": round(rep_ms, 2), "fresh_batch_device_ms": round(fresh_ms, 2),
                         "repair_speedup_vs_fresh": round(fresh_ms / rep_ms, 2) if rep_ms > 0 else None,
                         "exact": bool(list(fr) == list(fresh))})
    ss.close()
    g.close()
    mid = runs[1]
    res = {"metric": "exact max-flow queries/sec after a capacity-update batch (incremental repair)",
           "value": round(len(s) / (mid["update_and_repair_wall_ms"] / 1e3), 3), "unit": "queries/s",
           "n_gpus": 1, "higher_is_better": True, "dtype": "int64",
           "data": "synthetic (seeded R-MAT 2^22, 2^26 draws, caps U[1,1000]; 16 hub + 16 uniform queries; "
                   "updates +-U[1,100] on random edges, clamped at 0)",
           "config": {"workload": "rmat22_32q_updates", "n": n, "arcs": arcs, "queries": len(s), "R": R,
                      "group_ctas": o.group_ctas, "value_from": "10k-update batch, host wall time of "
                      "mf_session_update (capacity updates + repair of all 32 queries)"},
           "initial_session_solve_wall_ms": round(solve_wall, 2), "initial_exact": exact0,
           "batches": runs, "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(res), flush=True)


def reference_workload(scale=SCALE, nhub=NHUB, nuni=NUNI):
    """The headline workload from the oracle's restatement of the engine's
    generators (identical arrays, tests/test_oracle.py), so that the process
    timing the reference never loads the engine's library."""
    from oracle import oracle as O
    u, v, c = O.gen_rmat(scale, 16 << scale, 0.57, 0.19, 0.19, 1, 1000, GRAPH_SEED)
    n = 1 << scale
    s, t = O.gen_queries_hub(n, u, v, nhub, nuni, QUERY_SEED)
    return n, u, v, c, s, t


def classify_reference_mismatches(stderr_text, n_full, arcs_full, mismatched):
    """Classify each query whose reference flow differs from the oracle's.
    The reference keeps one graph on the device and, when a query's run graph
    has the same (V, E, R) as the one there, re-uploads only the capacities
    (init_global_graph_on_device, RA:1303-1331) onto the previous topology.
    A mismatch on such a query is 'stale-topology'; any other is
    'unexplained'.  Uses the reference's own per-query log lines
    ('[QueryPrune+RegionBoundary] ... run_n=.., run_m=..', RA:2815-2819)."""
    import re
    dims = []
    for line in stderr_text.splitlines():
        if line.startswith("[QueryPrune+RegionBoundary]"):
            mn = re.search(r"run_n=(\d+)", line)
            mm = re.search(r"run_m=(\d+)", line)
            dims.append((int(mn.group(1)), int(mm.group(1))) if mn and mm else None)
    out = {}
    for i in mismatched:
        if i >= len(dims) or dims[i] is None:
            out[i] = "unexplained (no log line)"
            continue
        prev = dims[i - 1] if i > 0 else (n_full, arcs_full)
        out[i] = "stale-topology" if dims[i] == prev else "unexplained"
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    if not os.path.exists(O.REF_BIN):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ra_ref not built "
                          "(needs the reference sources; oracle/build_ref.sh)"}))
        return
    n, u, v, c, s, t = reference_workload()
    per_step = args.ref_queries_per_step
    nsteps = args.warmup + args.steps
    order = [i for pair in zip(range(NHUB), range(NHUB, NHUB + NUNI)) for i in pair]
    idx = order[: per_step * nsteps]
    d = tempfile.mkdtemp()
    out = os.path.join(d, "out")
    O.write_graph_txt(os.path.join(d, "graph.txt"), n, u, v, c)
    O.write_test_txt(os.path.join(d, "test.txt"), s[idx], t[idx])
    t0 = time.time()
    with ClockSampler(0) as clk:
        r = subprocess.run(["timeout", str(args.ref_timeout), O.REF_BIN, d, out, "static"],
                           capture_output=True, text=True)
    wall = time.time() - t0
    if r.returncode != 0 or not os.path.exists(os.path.join(out, "res_mt.txt")):
        print(json.dumps({"impl": "reference", "unavailable": "reference run failed (rc %d): %s" % (
            r.returncode, r.stderr.strip().splitlines()[-1] if r.stderr.strip() else "")}))
        return
    res = np.loadtxt(os.path.join(out, "res_mt.txt"), dtype=np.int64, ndmin=2)
    times = res[:, 1].astype(np.float64)
    timed = times[args.warmup * per_step:]
    ms_step = float(np.mean([timed[i * per_step:(i + 1) * per_step].sum() for i in range(args.steps)]))
    value = per_step / (ms_step / 1e3) if ms_step > 0 else None
    sample = "%d queries (alternating hub/uniform of the 256), %d per step; reference's own per-query " \
             "times from res_mt.txt (integer ms, prune included, upload excluded); run wall %.1f s" % (
                 len(idx), per_step, wall)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic (seeded R-MAT 2^20, 2^24 draws, caps U[1,1000])",
            "config": {"workload": WORKLOAD, "n": n, "edges": len(u), "queries_sampled": len(idx), "R": 128,
                       "sample": "queries 0,128,1,129,... of the 256 (hub and uniform alternating)"},
            "p50_ms": pct(timed, 50), "p99_ms": pct(timed, 99),
            "cpu_baseline": {"value": value, "unit": "queries/s", "cores": 1, "kind": "reference",
                             "sample": sample + "; the reference is a CUDA program: host prune on 1 core "
                                                "+ kernels on the B200"},
            "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "inputs": "graph.txt / test.txt written by the oracle's generators (oracle/gen.c); "
                      "this process loads no engine library",
            "clocks": clk.summary()}
    if not args.no_check:
        g = O.build_csr(n, u, v, c)
        exp = O.dinic_batch(g, s[idx], t[idx], os.cpu_count() or 1)
        got = res[:, 0]
        bad = [i for i in range(len(idx)) if int(got[i]) != int(exp[i])]
        line["flows_match_oracle"] = len(idx) - len(bad)
        line["flows_checked"] = len(idx)
        if bad:
            cls = classify_reference_mismatches(r.stderr, n, g.arcs, bad)
            line["mismatches"] = [{"query": int(idx[i]), "reference": int(got[i]), "oracle": int(exp[i]),
                                   "class": cls[i]} for i in bad]
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--group", type=int, default=8)
    ap.add_argument("--serve", type=int, default=1)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--ref-queries-per-step", type=int, default=2)
    ap.add_argument("--ref-timeout", type=int, default=900)
    ap.add_argument("--no-check", action="store_true",
                    help="reference arm: skip checking its flows against the oracle's Dinic")
    ap.add_argument("--no-certify", action="store_true", help="skip the untimed certification pass")
    ap.add_argument("--scale", type=int, default=SCALE)
    ap.add_argument("--nhub", type=int, default=NHUB)
    ap.add_argument("--nuni", type=int, default=NUNI)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--dump", default=None, help="write per-query stats (jsonl)")
    ap.add_argument("--K", type=int, default=0, help="discharge cycles (0 = library default)")
    ap.add_argument("--threads", type=int, default=0, help="threads per CTA (0 = library default)")
    ap.add_argument("--opt", action="append", default=[], metavar="FIELD=VALUE",
                    help="set any mf_opts field (repeatable), e.g. --opt use_hot_sweep=0")
    ap.add_argument("--gr-freq", type=int, default=0, help="max rounds between global relabels")
    ap.add_argument("--gr-alpha", type=float, default=None, help="relabel after alpha x kept arcs of work")
    ap.add_argument("--workload", default="rmat", choices=["rmat", "mix", "gridsets", "dynamic"],
                    help="rmat: the headline R-MAT 2^20 batch; mix: the serving mix of 8 graphs; "
                         "gridsets: one segmentation grid, queries that vary the terminal set; "
                         "dynamic: capacity-update batches on R-MAT 2^22 with resident queries")
    ap.add_argument("--grid-w", type=int, default=2048)
    ap.add_argument("--grid-sets", type=int, default=64)
    ap.add_argument("--mix-requests", type=int, default=512)
    ap.add_argument("--mix-update-share", type=float, default=0.1,
                    help="mix: share of requests that are capacity-update batches in the extra served run")
    ap.add_argument("--no-other", action="store_true",
                    help="headline run: skip the other workloads (gridsets, dynamic, mix) that a full 1-GPU "
                         "run appends to its line as other_workloads (--no-cpu skips them too)")
    ap.add_argument("--other-timeout", type=int, default=420, help="seconds allowed to each other workload")
    ap.add_argument("--mix-rates", type=float, nargs="+", default=[0.5, 1.0, 2.0, 4.0],
                    help="arrival rates as multiples of the plain loop's throughput")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "mix":
        run_mix(args)
    elif args.workload == "gridsets":
        run_gridsets(args)
    elif args.workload == "dynamic":
        run_dynamic(args)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
