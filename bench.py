"""Benchmark: sampled edges per second (SEPS) on one B200 (or N replicas).

Workload (one step): the mid-size power-law graph -- a seeded synthetic
directed graph with 875,713 vertices and 5,105,039 edges, out-degree power
law exponent 2.1 capped at 460, int32 CSR, lognormal(0,1) weights -- run with
  (a) degree-biased neighbor sampling: 4000 samples, FrontierSize 4,
      NeighborSize 20, Depth 3;
  (b) degree-biased random walks: 4000 walks of length 64.
value = (edges of a + edges of b) / device time of the step.  Inputs are
resident in HBM; between timed steps a 256 MiB buffer is written to flush L2.
e2e = the same metric through the host-buffer entry points (csaw_sample_host
for the plain form, csaw_sample_batch with host buffers for the batched form):
host seeds in, host edge list (src, dst, sample) out, copies inside the timed
region.
Three forms run on the same graph, seeds and keys: "plain" (one warp per
item, level by level, gathered degree bias, jobs one after the other),
"batched" (load-balanced expansion, neighbor records, concurrent jobs,
CUDA-graph replay, degree-rule granularity) and "learned" (batched with the
learned granularity scheduler, trained on the GPU on profiles recorded on a
few warm-up steps).  value is the last form of --forms (default: learned).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl csaw|reference]

--impl reference times the CPU oracle (a port of the reference's sampling
semantics; the reference itself has no CPU implementation and its CUDA
kernels read out of bounds, so they are not run) on all host threads, on a
bounded sample of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "c-saw_b200")]

GRAPH = dict(n_vertices=875_713, n_edges=5_105_039, gamma=2.1, max_degree=460, seed=20, weight="lognormal")
WORK_A = dict(mode=0, bias=1, n_samples=4000, frontier_size=4, neighbor_size=20, depth=3)
WORK_B = dict(mode=1, bias=1, n_samples=4000, frontier_size=1, neighbor_size=1, depth=64)
SEED_A, SEED_B = 0xC5A0, 0xC5A1
FLUSH_BYTES = 256 << 20
# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum, mean over
# the three level launches of one step) from one full ncu capture of the
# batched form of this workload; the capture is summarised under profiles/.
DRAM_TRAFFIC = {"k_select_fast": 5.01e6, "k_coop_fast": 13.8e6, "k_walk_fast": 43.1e6}


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.idx = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.2)
        self.proc.terminate()
        self.proc.wait()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    return int(os.environ.get("RANK", "0")), ws, int(os.environ.get("LOCAL_RANK", "0"))


def build_graph():
    from csaw import graphgen
    return graphgen.powerlaw_directed(**GRAPH)


def workload_desc():
    return {"workload": "powerlaw_v875713_e5105039: (a) degree-biased neighbor sampling 4000 samples F4 N20 D3 "
                        "+ (b) degree-biased random walks 4000 x 64",
            "graph": GRAPH, "a": WORK_A, "b": WORK_B, "l2": "flushed between timed steps (256 MiB write)"}


def run_reference(args):
    """CPU oracle on all host threads, bounded sample of the workload per step."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    g = build_graph()
    threads = os.cpu_count() or 1
    na, nb = 1000, 1000   # a quarter of each workload per step
    seeds_a = oracle.make_seeds(g.rowptr, na * WORK_A["frontier_size"], SEED_A)
    seeds_b = oracle.make_seeds(g.rowptr, nb, SEED_B)

    def step():
        ea = oracle.run(g.rowptr, g.col, g.weight, seeds_a, 0, 1, na, 4, 3, [20, 20, 20], seed=SEED_A,
                        n_threads=threads)
        eb = oracle.run(g.rowptr, g.col, g.weight, seeds_b, 1, 1, nb, 1, 64, seed=SEED_B, n_threads=threads)
        return len(ea[0]) + len(eb[0])

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    edges = sum(step() for _ in range(args.steps))
    dt = time.perf_counter() - t0
    v = edges / dt
    desc = workload_desc()
    desc["sample"] = f"{na} of 4000 samples of (a) and {nb} of 4000 walks of (b) per step"
    line = {"impl": "reference", "metric": "sampled_edges_per_sec", "value": v, "unit": "edges/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+int32", "data": "synthetic", "config": desc,
            "cpu_baseline": {"value": v, "unit": "edges/s", "cores": threads, "kind": "port",
                             "sample": desc["sample"]},
            "e2e": {"value": v, "unit": "edges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def cpu_baseline(g):
    """Oracle timed on the host cores on a bounded sample (reported baseline only)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    threads = os.cpu_count() or 1
    na, nb = 1000, 1000
    sa = oracle.make_seeds(g.rowptr, na * 4, SEED_A)
    sb = oracle.make_seeds(g.rowptr, nb, SEED_B)
    edges, t0, reps = 0, time.perf_counter(), 0
    while True:
        ea = oracle.run(g.rowptr, g.col, g.weight, sa, 0, 1, na, 4, 3, [20, 20, 20], seed=SEED_A, n_threads=threads)
        eb = oracle.run(g.rowptr, g.col, g.weight, sb, 1, 1, nb, 1, 64, seed=SEED_B, n_threads=threads)
        edges += len(ea[0]) + len(eb[0])
        reps += 1
        if time.perf_counter() - t0 > 10.0:
            break
    dt = time.perf_counter() - t0
    return {"value": edges / dt, "unit": "edges/s", "cores": threads, "kind": "port",
            "sample": f"{reps} x ({na} of 4000 samples of (a) + {nb} of 4000 walks of (b)), {dt:.1f} s"}


def learned_gain(args):
    """Degree rule vs learned granularity on a heavy-tailed graph: R-MAT
    (a=.6, b=.2, c=.15) scale 20, edge factor 16, Pareto(1.5) weights,
    edge-weight-biased sampling, 8192 samples, F 8, N 10, D 3 (the shape of
    the scale-25 learned-scheduler configuration at 1/32 of its vertices),
    with the per-vertex prefix cache (the default for this graph) and without
    it.  Prints one JSON line with both times per variant; identical edges
    are asserted."""
    import torch
    import csaw
    from csaw import graphgen
    g = graphgen.rmat(20, 16, a=0.6, b=0.2, c=0.15, seed=25, weight="pareto:1.5")
    out = torch.empty((3, 8192 * 8 * (10 + 100 + 1000)), dtype=torch.int32, device="cuda")
    res = {"graph": {"V": g.n_vertices, "E": g.n_edges, "max_degree": int(np.diff(g.rowptr).max())}}
    for variant, cache in (("cache", None), ("no_cache", False)):
        G = csaw.Graph(g, cdf_cache=cache)
        seeds = G.make_seeds(8192 * 8, 0x25)
        r = {}
        for form, sch in (("batched", csaw.SCHED_BATCHED), ("learned", csaw.SCHED_LEARNED)):
            p = csaw.make_params(0, 2, 8192, 8, 10, 3, seed=0x25, schedule=sch)
            job = [csaw.BatchJob(p, seeds, out.shape[1], out, with_depth=False)]
            if form == "learned":
                G.sched_record(400_000)
                for _ in range(3):
                    G.sample_batch(job)
                r["train_loss"] = G.sched_train(epochs=400, lr=3e-3, seed=1)
                for _ in range(6):   # timed trial of the model against the degree rule
                    G.sample_batch(job)
                r["class_mask"] = G.sched_info()["class_mask"]
            for _ in range(args.warmup):
                G.sample_batch(job)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            n = 0
            for _ in range(args.steps):
                n += G.sample_batch(job)[0][0].numel()
            e1.record()
            torch.cuda.synchronize()
            r[form] = {"ms_per_step": e0.elapsed_time(e1) / args.steps, "edges_per_step": n / args.steps}
            G.profile(True)
            G.sample_batch(job)
            r[form]["kernels"] = {k: G.kernel_stats(k) for k in ("expand", "select", "heavy", "setup")}
            G.profile(False)
        assert r["batched"]["edges_per_step"] == r["learned"]["edges_per_step"]
        r["learned_speedup"] = r["batched"]["ms_per_step"] / r["learned"]["ms_per_step"]
        res[variant] = r
        G.close()
    print(json.dumps({"learned_gain": res}))


SERVE_GRAPH = dict(scale=22, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=22, weight="uniform")
SERVE_RATE = 2000.0          # requests per second, Poisson
SERVE_SEEDS = (512, 1.0, 64, 8192)   # lognormal median, sigma, clip


def serve_requests(csaw, g, n, rng, kind=None, n_seeds=None):
    """Requests of the serving mix: 2-hop [25,10] and 3-hop [15,10,5]
    edge-weight-biased neighbor sampling and edge-weight-biased walks of
    length U{10..80}, in equal shares; seeds per request lognormal (median
    512, sigma 1) clipped to [64, 8192], uniform over non-isolated vertices."""
    med, sig, lo, hi = SERVE_SEEDS
    deg = np.diff(g.rowptr)
    non = np.flatnonzero(deg > 0).astype(np.int32)
    out = []
    for i in range(n):
        k = kind if kind is not None else int(rng.integers(0, 3))
        m = n_seeds or int(np.clip(np.round(med * np.exp(sig * rng.standard_normal())), lo, hi))
        seeds = non[rng.integers(0, non.size, m)]
        if k == 0:
            p = csaw.make_params(0, 2, m, 1, 25, 2, [25, 10], seed=1 + i, schedule=csaw.SCHED_BATCHED)
        elif k == 1:
            p = csaw.make_params(0, 2, m, 1, 15, 3, [15, 10, 5], seed=1 + i, schedule=csaw.SCHED_BATCHED)
        else:
            p = csaw.make_params(1, 2, m, 1, 1, int(rng.integers(10, 81)), seed=1 + i,
                                 schedule=csaw.SCHED_BATCHED)
        out.append((k, m, p, seeds))
    return out


def run_stream(csaw, S, reqs, rate, rng, pool):
    """Open-loop Poisson arrivals at `rate`: a submitter thread issues each
    request at its arrival time, a waiter collects results in order.  Output
    buffers are page-locked (direct device-to-host copies), from a pool by
    size class.  Latency is measured inside the library (submit to result in
    host memory)."""
    import threading
    gaps = rng.exponential(1.0 / rate, len(reqs))
    tickets = [None] * len(reqs)
    ready = threading.Semaphore(0)
    lat = [0.0] * len(reqs)
    edges = [0] * len(reqs)

    def waiter():
        for i in range(len(reqs)):
            ready.acquire()
            t, buf, cls = tickets[i]
            n, ms, _ = S.wait(t)
            lat[i], edges[i] = ms, n
            pool.put(cls, buf)

    th = threading.Thread(target=waiter)
    th.start()
    t0 = time.perf_counter()
    due = t0
    for i, (k, m, p, seeds) in enumerate(reqs):
        due += gaps[i]
        cap = csaw.edge_bound(p)
        cls, buf = pool.get(cap)
        while True:
            left = due - time.perf_counter()
            if left <= 0:
                break
            if left > 3e-4:
                time.sleep(left - 3e-4)
        tickets[i] = (S.submit(p, seeds, out=buf, capacity=cap, with_sample=False, with_depth=False), buf, cls)
        ready.release()
    th.join()
    wall = time.perf_counter() - t0
    return np.array(lat), np.array(edges), wall


def run_closed(csaw, S, reqs, window, pool):
    """Closed loop: at most `window` requests outstanding, the next one
    submitted as soon as the oldest returns (the loop's sustained capacity)."""
    from collections import deque
    out = deque()
    t0 = time.perf_counter()
    edges = 0
    for k, m, p, seeds in reqs:
        if len(out) >= window:
            t, buf, cls = out.popleft()
            edges += S.wait(t)[0]
            pool.put(cls, buf)
        cap = csaw.edge_bound(p)
        cls, buf = pool.get(cap)
        out.append((S.submit(p, seeds, out=buf, capacity=cap, with_sample=False, with_depth=False), buf, cls))
    while out:
        t, buf, cls = out.popleft()
        edges += S.wait(t)[0]
        pool.put(cls, buf)
    return edges, time.perf_counter() - t0


class PinnedPool:
    """Page-locked (2, cap) int32 buffers by power-of-two size class."""

    def __init__(self):
        self.free = {}

    def get(self, cap):
        import torch
        cls = max(1 << 12, 1 << int(np.ceil(np.log2(max(cap, 1)))))
        lst = self.free.setdefault(cls, [])
        if lst:
            return cls, lst.pop()
        return cls, torch.empty((2, cls), dtype=torch.int32).pin_memory()

    def put(self, cls, buf):
        self.free[cls].append(buf)

    def prefill(self, cap, n):
        """n buffers of cap's class, allocated before timing."""
        import torch
        cls = max(1 << 12, 1 << int(np.ceil(np.log2(max(cap, 1)))))
        lst = self.free.setdefault(cls, [])
        while len(lst) < n:
            lst.append(torch.empty((2, cls), dtype=torch.int32).pin_memory())


def serving(args, n_slots=8):
    """Serving workload: R-MAT scale 22, edge factor 16, U(0,1] weights (4.19M
    vertices, generated on the GPU), a Poisson stream of mixed requests at
    2000 req/s, plus a stream of 1024-seed 2-hop requests at the same rate.
    Returns p50/p99 latency and throughput of each."""
    import torch
    import csaw
    from csaw import graphgen
    sys.setswitchinterval(2e-4)   # the waiter thread returns buffers promptly
    g = graphgen.rmat_device(**SERVE_GRAPH)
    torch.cuda.empty_cache()
    G = csaw.Graph(g)
    S = csaw.Server(G, n_slots=n_slots, device_budget=2 << 30)
    rng = np.random.default_rng(2000)
    pool = PinnedPool()
    res = {"graph": {"workload": f"rmat{SERVE_GRAPH['scale']}_ef{SERVE_GRAPH['edge_factor']}",
                     "n_vertices": g.n_vertices, "n_edges": g.n_edges,
                     "max_degree": int(np.diff(g.rowptr).max())},
           "rate_per_s": SERVE_RATE, "n_slots": n_slots, "device_budget": 2 << 30}
    # warm-up: every request kind at the largest sizes (job scratch, staging, caches)
    for k in range(3):   # n_slots largest requests at once: every slot grows its scratch once
        run_stream(csaw, S, serve_requests(csaw, g, n_slots, rng, kind=k, n_seeds=8192), 1e6, rng, pool)
    run_stream(csaw, S, serve_requests(csaw, g, 400, rng), SERVE_RATE, rng, pool)
    # and the 1024-seed 2-hop shape, so its page-locked output buffers exist
    # before timing (allocating them takes the CUDA driver's lock for milliseconds)
    run_stream(csaw, S, serve_requests(csaw, g, 200, rng, kind=0, n_seeds=1024), SERVE_RATE, rng, pool)
    pool.prefill(1024 * (25 + 250), 64)   # a burst of late waits must not allocate mid-stream
    S.stats(reset=True)
    for name, rate, reqs in (
            ("mixed", SERVE_RATE, serve_requests(csaw, g, args.serve_requests, rng)),
            ("twohop_1024", SERVE_RATE, serve_requests(csaw, g, args.serve_requests, rng, kind=0, n_seeds=1024)),
            # closed loop, 4 requests per slot outstanding: the loop's capacity
            ("mixed_saturated", None, serve_requests(csaw, g, args.serve_requests, rng))):
        if rate is None:
            e, wall = run_closed(csaw, S, reqs, 4 * n_slots, pool)
            edges = np.array([e])
        else:
            lat, edges, wall = run_stream(csaw, S, reqs, rate, rng, pool)
        st = S.stats(reset=True)
        res[name] = {"requests": len(reqs), "p50_ms": st["p50_ms"], "p90_ms": st["p90_ms"], "p99_ms": st["p99_ms"],
                     "max_ms": st["max_ms"], "mean_ms": st["mean_ms"], "p99_queue_ms": st["p99_queue_ms"],
                     "p99_launch_ms": st["p99_launch_ms"], "p99_gpu_ms": st["p99_gpu_ms"], "edges": int(edges.sum()),
                     "seps": float(edges.sum()) / (st["last_done_s"] - st["first_submit_s"]),
                     "offered_rate": len(reqs) / wall, "failed": st["failed"],
                     "peak_device_bytes": st["peak_device_bytes"]}
    S.close()
    G.close()
    return res


SCALE25_GRAPH = dict(scale=25, edge_factor=16, a=0.6, b=0.2, c=0.15, seed=25, symmetrize=False,
                     weight="pareto:1.5")


def scale25(args):
    """Learned scheduler at scale: R-MAT (a=.6, b=.2, c=.15) scale 25, edge
    factor 16, directed, int64 rowptr, int32 col, Pareto(1.5) weights
    (generated on the GPU); one step = 65,536 edge-weight-biased samples
    (F 8, N 10, D 3) and 1M edge-weight-biased walks of length 40 as one
    batch.  The batched (degree rule) and learned forms are timed; the
    learned one is trained on profiles recorded on warm-up steps."""
    import torch
    import csaw
    from csaw import graphgen
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    sc = args.s25_scale
    g = graphgen.rmat_device(**dict(SCALE25_GRAPH, scale=sc))
    gen_s = time.perf_counter() - t0
    torch.cuda.empty_cache()
    G = csaw.Graph(g, rowptr64=True)
    ns, nw = 65536 >> (25 - sc), (1 << 20) >> (25 - sc)
    seeds_a = G.make_seeds(ns * 8, 0x25A)
    seeds_b = G.make_seeds(nw, 0x25B)
    res = {"graph": {"workload": f"rmat{sc}_ef16_a.6_b.2_c.15_pareto1.5", "n_vertices": g.n_vertices,
                     "n_edges": g.n_edges, "max_degree": int(np.diff(g.rowptr).max()), "generate_s": gen_s},
           "a": dict(mode=0, bias=2, n_samples=ns, frontier_size=8, neighbor_size=10, depth=3),
           "b": dict(mode=1, bias=2, n_samples=nw, depth=40)}
    del g
    peak, peak_kind = load_peaks()
    outs = {}
    forms = [f for f in (("batched", csaw.SCHED_BATCHED), ("learned", csaw.SCHED_LEARNED))
             if f[0] in args.s25_forms.split(",")]
    for form, sch in forms:
        pa = csaw.make_params(0, 2, ns, 8, 10, 3, seed=0x25A, schedule=sch)
        pb = csaw.make_params(1, 2, nw, 1, 1, 40, seed=0x25B, schedule=sch)
        if "a" not in outs:
            outs["a"] = torch.empty((3, csaw.edge_bound(pa)), dtype=torch.int32, device="cuda")
            outs["b"] = torch.empty((3, csaw.edge_bound(pb)), dtype=torch.int32, device="cuda")
        jobs = [csaw.BatchJob(pa, seeds_a, outs["a"].shape[1], outs["a"], with_depth=False),
                csaw.BatchJob(pb, seeds_b, outs["b"].shape[1], outs["b"], with_depth=False)]
        r = {}
        if form == "learned":
            G.sched_record(400_000)
            for _ in range(2):
                G.sample_batch(jobs)
            r["train_loss"] = G.sched_train(epochs=400, lr=3e-3, seed=1)
            for _ in range(6):   # timed trial of the model against the degree rule
                G.sample_batch(jobs)
            r["class_mask"] = G.sched_info()["class_mask"]
        for _ in range(args.warmup):
            G.sample_batch(jobs)
        if form == "batched":
            r["autotune"] = G.autotune(jobs)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        n = 0
        for _ in range(args.steps):
            res_b = G.sample_batch(jobs)
            n += res_b[0][0].numel() + res_b[1][0].numel()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        G.profile(True)
        G.sample_batch(jobs)
        ks = {k: G.kernel_stats(k) for k in ("expand", "select", "hub", "pair", "heavy", "walk", "setup")}
        G.profile(False)
        tot_bytes = sum(v["bytes"] for v in ks.values())
        r.update({"ms_per_step": ms, "edges_per_step": n / args.steps, "seps": n / args.steps / (ms * 1e-3),
                  "algorithmic_bytes_per_step": tot_bytes,
                  "achieved_gbs": tot_bytes / (ms * 1e-3) / 1e9,
                  "roofline_frac": tot_bytes / (ms * 1e-3) / 1e9 / peak,
                  "kernels": {k: v for k, v in ks.items() if v["launches"]}})
        res[form] = r
    res["peak_gbs"] = peak
    res["peak_source"] = peak_kind
    if "batched" in res and "learned" in res:
        res["learned_speedup"] = res["batched"]["ms_per_step"] / res["learned"]["ms_per_step"]
    G.close()
    return res


STREAM_GRAPH = dict(scale=26, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=29, symmetrize=False, weight="uniform")


def streaming(args):
    """Streaming (out-of-budget) workload at 1/8 of the scale-29 configuration:
    R-MAT scale 26, edge factor 16, directed, U(0,1] weights (generated on the
    GPU), adjacency in page-locked host memory with the device partition
    budget capped at 4 GiB (under half of the 8.5 GB adjacency) and 2^17-vertex
    partitions (512, as many as the scale-29 configuration has); one step = 131,072 edge-weight-biased walks of length 20 and
    32,768 edge-weight-biased samples F1 N10 D2.  The same jobs on the
    in-memory graph give the reference time and check the edge counts."""
    import torch
    import csaw
    from csaw import graphgen
    torch.cuda.set_device(0)
    g = graphgen.rmat_device(**STREAM_GRAPH)
    torch.cuda.empty_cache()
    budget = 4 << 30
    res = {"graph": {"workload": "rmat26_ef16_uniform", "n_vertices": g.n_vertices, "n_edges": g.n_edges,
                     "host_adjacency_bytes": int(g.col.nbytes + g.weight.nbytes + g.rowptr.nbytes)},
           "partition_bits": 17, "device_budget": budget,
           "walks": dict(n=1 << 17, length=20), "samples": dict(n=1 << 15, F=1, N=10, D=2)}
    pw = csaw.make_params(1, 2, 1 << 17, 1, 1, 20, seed=0x29A)
    ps = csaw.make_params(0, 2, 1 << 15, 1, 10, 2, seed=0x29B)
    # the in-memory reference also runs the batched schedule (cache, records)
    pwb = csaw.make_params(1, 2, 1 << 17, 1, 1, 20, seed=0x29A, schedule=csaw.SCHED_BATCHED)
    psb = csaw.make_params(0, 2, 1 << 15, 1, 10, 2, seed=0x29B, schedule=csaw.SCHED_BATCHED)
    S = csaw.StreamGraph(g, partition_bits=17, slot_budget_bytes=budget, rowptr64=True)
    G = csaw.Graph(g, rowptr64=True)
    sw = G.make_seeds(1 << 17, 0x29C)
    ss = G.make_seeds(1 << 15, 0x29D)
    outs = {k: torch.empty((4, csaw.edge_bound(p)), dtype=torch.int32, device="cuda") for k, p in (("w", pw), ("s", ps))}

    def step(obj, batched=False):
        a = obj.sample(pwb if batched else pw, sw, out=outs["w"])
        b = obj.sample(psb if batched else ps, ss, out=outs["s"])
        return a[0].numel() + b[0].numel()

    for name, obj, bt in (("stream", S, False), ("in_memory", G, False), ("in_memory_batched", G, True)):
        for _ in range(args.warmup):
            step(obj, bt)
        torch.cuda.synchronize()
        i0 = S.info() if name == "stream" else None
        t0 = time.perf_counter()
        e = sum(step(obj, bt) for _ in range(args.steps))
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / args.steps
        r = {"ms_per_step": dt * 1e3, "edges_per_step": e / args.steps, "seps": e / args.steps / dt}
        if name == "stream":
            i1 = S.info()
            r["h2d_bytes_per_step"] = (i1["bytes_h2d"] - i0["bytes_h2d"]) / args.steps
            r["partition_loads_per_step"] = (i1["partition_loads"] - i0["partition_loads"]) / args.steps
            r["partitions"] = i1["n_partitions"]
            r["slots"] = i1["n_slots"]
            r["h2d_gbs"] = r["h2d_bytes_per_step"] / dt / 1e9
        res[name] = r
    assert res["stream"]["edges_per_step"] == res["in_memory"]["edges_per_step"] == \
        res["in_memory_batched"]["edges_per_step"]
    res["stream_vs_in_memory"] = res["stream"]["seps"] / res["in_memory"]["seps"]
    S.close()
    G.close()
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="csaw", choices=["csaw", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--learned-gain", action="store_true",
                    help="time the degree rule vs the learned scheduler on a heavy-tailed R-MAT graph instead")
    ap.add_argument("--serve", action="store_true", help="run only the serving (request loop) workload")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving workload in the default run")
    ap.add_argument("--scale25", action="store_true", help="run only the R-MAT scale-25 learned-scheduler workload")
    ap.add_argument("--stream", action="store_true", help="run only the streaming (out-of-budget) workload")
    ap.add_argument("--s25-scale", type=int, default=25,
                    help="R-MAT scale for --scale25 (samples and walks scale with 2^scale; smaller for profiling)")
    ap.add_argument("--s25-forms", default="batched,learned", help="forms timed by --scale25")
    ap.add_argument("--serve-requests", type=int, default=4000, help="requests per serving stream")
    ap.add_argument("--forms", default="plain,batched,learned",
                    help="forms to time; the last one is reported as value (profiling runs use one form)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
        return
    if args.learned_gain:
        learned_gain(args)
        return
    if args.stream:
        print(json.dumps({"streaming": streaming(args)}))
        return
    if args.scale25:
        print(json.dumps({"scale25": scale25(args)}))
        return
    if args.serve:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps({"serving": serving(args)}))
        return

    import torch
    import csaw
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    g = build_graph()
    G = csaw.Graph(g)                       # one resident CSR for both forms
    stream = torch.cuda.current_stream()
    seeds_a = G.make_seeds(4000 * 4, SEED_A + 7919 * rank)
    seeds_b = G.make_seeds(4000, SEED_B + 7919 * rank)
    from csaw import dist as cdist
    # replicas (weak scaling): same job shape, rank-disjoint global sample ids
    params = {f: (cdist.replica_params(csaw.make_params(**WORK_A, seed=SEED_A, schedule=sch), rank),
                  cdist.replica_params(csaw.make_params(**WORK_B, seed=SEED_B, schedule=sch), rank))
              for f, sch in (("plain", csaw.SCHED_PLAIN), ("batched", csaw.SCHED_BATCHED),
                             ("learned", csaw.SCHED_LEARNED))}
    pa, pb = params["batched"]
    cap_a, cap_b = csaw.edge_bound(pa), csaw.edge_bound(pb)
    out_a = torch.empty((3, cap_a), dtype=torch.int32, device="cuda")
    out_b = torch.empty((3, cap_b), dtype=torch.int32, device="cuda")
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.int32, device="cuda")

    batch_jobs = {f: [csaw.BatchJob(params[f][0], seeds_a, cap_a, out_a, with_depth=False),
                      csaw.BatchJob(params[f][1], seeds_b, cap_b, out_b, with_depth=False)]
                  for f in ("batched", "learned")}

    def step(form):
        if form == "plain":   # one job after the other, as the reference runs them
            qa, qb = params[form]
            a = G.sample(qa, seeds_a, capacity=cap_a, out=out_a, with_depth=False)
            b = G.sample(qb, seeds_b, capacity=cap_b, out=out_b, with_depth=False)
            return a[0].numel() + b[0].numel()
        res = G.sample_batch(batch_jobs[form])   # both workloads as one batch
        return res[0][0].numel() + res[1][0].numel()

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def timed(form, clocks=None, profile=False):
        """K device-timed steps (L2 flushed before each); returns edges, ms, kernel stats, launches.
        With profile=True every kernel is bracketed by CUDA events (and CUDA-graph replay is off)."""
        for _ in range(args.warmup):
            step(form)
        G.profile(profile)
        launches0 = G.stats()["kernel_launches"]
        if clocks:
            clocks.start()
        barrier()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        edges = 0
        for i in range(args.steps):
            flush.zero_()
            evs[i][0].record(stream)
            edges += step(form)
            evs[i][1].record(stream)
        barrier()
        clk = clocks.stop() if clocks else None
        launches = G.stats()["kernel_launches"] - launches0
        ms = sum(x.elapsed_time(y) for x, y in evs)
        ks = {k: G.kernel_stats(k) for k in ("expand", "select", "hub", "pair", "heavy", "walk", "setup")}
        G.profile(False)
        return edges, ms, ks, launches, clk

    forms = [f.strip() for f in args.forms.split(",") if f.strip()]
    main_form = forms[-1]
    plain_ms, plain_k = None, {}
    other = {}
    if "plain" in forms and main_form != "plain":
        plain_edges, plain_ms, plain_k, _, _ = timed("plain", profile=True)
    tune = None
    if "batched" in forms:   # the launch-shape autotuner, on the batched form's own batch
        for _ in range(args.warmup):
            step("batched")
        tune = G.autotune(batch_jobs["batched"])
    if "batched" in forms and main_form != "batched":
        other["batched"] = timed("batched")[1]
    sched = None
    if "learned" in forms:
        # the learned scheduler: record execution profiles, train on the GPU
        G.sched_record(400_000)
        for _ in range(3):
            step("learned")
        t0 = time.perf_counter()
        loss = G.sched_train(epochs=400, lr=3e-3, seed=rank)
        train_s = time.perf_counter() - t0
        for _ in range(6):   # timed trial of the model against the degree rule
            step("learned")
        sched = {"records": G.sched_info()["records"], "train_loss": loss, "train_s": train_s,
                 "class_mask": G.sched_info()["class_mask"]}
    # per-kernel events for the roofline come from a profiled pass of the same
    # steps; the reported value is the unprofiled pass (graph replay allowed)
    _, prof_ms, kstats, _, _ = timed(main_form, profile=True)
    edges, ms, _, launches, clk = timed(main_form, Clocks(local))
    if plain_ms is not None and edges != plain_edges:
        raise SystemExit(f"plain and {main_form} forms emitted different edge counts: {plain_edges} vs {edges}")
    pa, pb = params[main_form]

    # ---- end to end through the host-buffer entry point
    seeds_a_h = seeds_a.cpu().numpy()
    seeds_b_h = seeds_b.cpu().numpy()
    host_a = torch.empty((3, cap_a), dtype=torch.int32).pin_memory().numpy()
    host_b = torch.empty((3, cap_b), dtype=torch.int32).pin_memory().numpy()
    sa_pin = torch.from_numpy(seeds_a_h).pin_memory().numpy()
    sb_pin = torch.from_numpy(seeds_b_h).pin_memory().numpy()
    host_jobs = [csaw.BatchJob(pa, sa_pin, cap_a, host_a, with_depth=False, host=True),
                 csaw.BatchJob(pb, sb_pin, cap_b, host_b, with_depth=False, host=True)]

    def e2e_step():
        if main_form == "plain":
            ra = G.sample_host(pa, sa_pin, capacity=cap_a, out=host_a, with_depth=False, stream=stream.cuda_stream)
            rb = G.sample_host(pb, sb_pin, capacity=cap_b, out=host_b, with_depth=False, stream=stream.cuda_stream)
        else:
            ra, rb = G.sample_batch(host_jobs, stream=stream.cuda_stream)
        return ra[0].size + rb[0].size

    e2e_steps = max(3, args.steps // 2)

    def e2e_time(parts):
        # parts: CSAW_OPT_HOST_PARTS (0 = by output size; -1 = copy after sampling)
        G.set_option(csaw._lib.OPT_HOST_PARTS, parts)
        e2e_step()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        n = 0
        for _ in range(e2e_steps):
            n += e2e_step()
        e1.record(stream)
        barrier()
        return n, e0.elapsed_time(e1)

    one_edges, one_ms = e2e_time(-1)
    e2e_edges, e2e_ms = e2e_time(0)

    # ---- MDRW, as the reference dispatches FrontierSize > 1 (main.cu:281-288):
    # 4000 degree-biased samples, frontier 4, 3 steps (timed separately)
    pm = cdist.replica_params(csaw.make_params(2, 1, 4000, 4, 20, 3, seed=SEED_A ^ 0x5A, schedule=csaw.SCHED_BATCHED),
                              rank)
    out_m = torch.empty((3, csaw.edge_bound(pm)), dtype=torch.int32, device="cuda")
    for _ in range(args.warmup):
        G.sample(pm, seeds_a, out=out_m, with_depth=False)
    m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    m0.record(stream)
    m_edges = 0
    for _ in range(args.steps):
        m_edges += G.sample(pm, seeds_a, out=out_m, with_depth=False)[0].numel()
    m1.record(stream)
    barrier()
    mdrw = {"samples": 4000, "frontier_size": 4, "depth": 3, "bias": "degree",
            "ms_per_step": m0.elapsed_time(m1) / args.steps, "edges_per_step": m_edges / args.steps,
            "seps": m_edges / (m0.elapsed_time(m1) * 1e-3)}

    # ---- whole-job totals: edges summed, device time max over ranks
    t_s = ms / 1e3
    if world > 1:
        all_edges, t_max = cdist.reduce_totals(edges, t_s)
        e2e_all, e2e_t = cdist.reduce_totals(e2e_edges, e2e_ms / 1e3)
        one_all, one_t = cdist.reduce_totals(one_edges, one_ms / 1e3)
        _, plain_t = cdist.reduce_totals(0, (plain_ms or 0.0) / 1e3)
    else:
        all_edges, t_max, e2e_all, e2e_t = float(edges), t_s, float(e2e_edges), e2e_ms / 1e3
        one_all, one_t = float(one_edges), one_ms / 1e3
        plain_t = (plain_ms or 0.0) / 1e3
    value = all_edges / t_max
    e2e_value = e2e_all / e2e_t

    peak, peak_kind = load_peaks()
    kernel_names = {"expand": "k_coop_fast" if main_form != "plain" else "k_expand_warp",
                    "select": "k_select_fast", "hub": "k_select_hub", "pair": "k_select_pair", "heavy": "k_expand_heavy",
                    "walk": "k_walk_fast" if main_form != "plain" else "k_walk_warp"}
    timed_kinds = [k for k in kernel_names if kstats.get(k, {}).get("launches")]
    dom = max(timed_kinds, key=lambda k: kstats[k]["ms"])
    kd = kstats[dom]
    achieved = kd["bytes"] / (kd["ms"] * 1e-3) / 1e9 if kd["ms"] > 0 else None
    roofline = {"bound": "hbm", "kernel": kernel_names[dom], "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind + " (hbm_gbs copy)",
                "traffic": DRAM_TRAFFIC.get(kernel_names[dom]),
                "algorithmic_bytes_per_launch": kd["bytes"] / kd["launches"],
                "launch_ms": kd["ms"] / kd["launches"],
                "note": "per-kernel CUDA events on the job streams, from a profiled pass of the same steps "
                        "(kernel by kernel, no graph replay); in the batched form the neighbor and walk jobs "
                        "overlap, so each kernel's time includes sharing the GPU"}

    if rank == 0:
        line = {"metric": "sampled_edges_per_sec", "value": value, "unit": "edges/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+int32",
                "data": "synthetic", "config": workload_desc(),
                "e2e": {"value": e2e_value, "unit": "edges/s",
                        "h2d_bytes_per_step": 4 * (seeds_a_h.size + seeds_b_h.size),
                        "d2h_bytes_per_step": int(12 * e2e_edges / e2e_steps)},
                "e2e_detail": {"host_parts": "by output size (one sample range per job here; edges copied back after every hop)",
                               "no_overlap_value": one_all / one_t,
                               "note": "no_overlap_value: the same calls with every host job's edges "
                                       "copied back after all of its sampling (CSAW_OPT_HOST_PARTS -1)"},
                "gpu_launches": int(launches), "clocks": clk, "roofline": roofline,
                "kernels": {k: v for k, v in kstats.items() if v["launches"]},
                "profiled_pass_ms_per_step": prof_ms / args.steps,
                "forms": {main_form: value, "plain": all_edges / plain_t if plain_t else None,
                          "speedup_vs_plain": plain_t / t_max if plain_t else None,
                          **{f: all_edges / (ms_f / 1e3) for f, ms_f in other.items()},
                          **({"learned_vs_batched": (other["batched"] / ms)} if "batched" in other else {}),
                          "scheduler": sched, "autotune": tune,
                          "plain_kernels": {k: v for k, v in plain_k.items() if v["launches"]}},
                "edges_per_step": all_edges / args.steps / world, "mdrw": mdrw}
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(g)
        if world == 1 and not args.no_serve:
            line["serving"] = serving(args)
        print(json.dumps(line))
    G.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
