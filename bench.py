"""Benchmark: sampled edges per second (SEPS) on one B200 (or N replicas).

Default workload, one step -- the learned-scheduler configuration at scale 25:
R-MAT (a=.6, b=.2, c=.15, d=.05) scale 25, edge factor 16, directed, with
self-loops and duplicate edges removed (33,554,432 vertices, 516,609,074
edges, max out-degree 986,212), int64 row offsets, int32 columns,
Pareto(1.5) FP32 weights, generated on the GPU from a fixed seed, then
  (a) edge-weight-biased neighbor sampling: 65,536 samples, FrontierSize 8,
      NeighborSize 10, Depth 3;
  (b) edge-weight-biased random walks: 1,048,576 walks of length 40.
value = (edges of a + edges of b) / device time of the step.  Inputs are
resident in HBM and far larger than L2; a 256 MiB buffer is also written
between timed steps.  e2e = the same metric through the host-buffer entry
point (csaw_sample_batch with host jobs): host seeds in, host edge list
(src, dst, sample) out, copies inside the timed region.

Three forms run on the same graph, seeds and keys: "plain" (one warp per
item, level by level, the bias prefix recomputed per expansion, jobs one
after the other), "batched" (load-balanced expansion, neighbor records,
per-vertex prefix cache, concurrent jobs, CUDA-graph replay, degree-rule
granularity, launch shape from the autotuner) and "learned" (batched with
the learned granularity scheduler, trained on the GPU on profiles recorded
on warm-up steps).  value is the last form of --forms (default: learned).
Every form's edge multiset is hashed; differing hashes abort the run.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl csaw|reference]
                  [--workload rmat25|powerlaw] [--scale S]

--workload powerlaw: the mid-size power-law graph (875,713 vertices,
5,105,039 edges, out-degree exponent 2.1 capped at 460, int32 CSR,
lognormal(0,1) weights), (a) 4000 degree-biased samples F4 N20 D3 and (b)
4000 degree-biased walks of 64.  The default run reports it, the request
loop (serving), MDRW and a streaming run (R-MAT scale 24 through a 1 GiB
partition budget; --stream for the larger shapes) as extra keys.

--impl reference times the CPU oracle (a port of the reference's sampling
semantics; the reference itself has no CPU implementation and its CUDA
kernels read out of bounds, so they are not run) on all host threads, on a
bounded seed subsample of the same workload and graph.
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "c-saw_b200")]

WORKLOADS = {
    "rmat25": dict(
        name="rmat{scale}_ef16_a.6_b.2_c.15_pareto1.5",
        generator="rmat_device",
        graph=dict(scale=25, edge_factor=16, a=0.6, b=0.2, c=0.15, seed=25, symmetrize=False, weight="pareto:1.5"),
        rowptr64=True,
        a=dict(mode=0, bias=2, n_samples=65536, frontier_size=8, neighbor_size=10, depth=3),
        b=dict(mode=1, bias=2, n_samples=1 << 20, frontier_size=1, neighbor_size=1, depth=40),
        seeds=(0x25A, 0x25B),
        cpu_fraction=1 / 512,   # oracle sample: this share of the samples of (a) and of the walks of (b)
        plain_fraction=1 / 8,   # the plain form runs this share (it rebuilds every hub's prefix per expansion)
        text="(a) edge-weight-biased neighbor sampling {na} samples F8 N10 D3 + (b) edge-weight-biased "
             "random walks {nb} x 40"),
    "powerlaw": dict(
        name="powerlaw_v875713_e5105039",
        generator="powerlaw_directed",
        graph=dict(n_vertices=875_713, n_edges=5_105_039, gamma=2.1, max_degree=460, seed=20, weight="lognormal"),
        rowptr64=False,
        a=dict(mode=0, bias=1, n_samples=4000, frontier_size=4, neighbor_size=20, depth=3),
        b=dict(mode=1, bias=1, n_samples=4000, frontier_size=1, neighbor_size=1, depth=64),
        seeds=(0xC5A0, 0xC5A1),
        cpu_fraction=1 / 4,
        plain_fraction=1,
        text="(a) degree-biased neighbor sampling {na} samples F4 N20 D3 + (b) degree-biased random walks {nb} x 64"),
}
FLUSH_BYTES = 256 << 20
KINDS = ("expand", "select", "select_thread", "hub", "pair", "heavy", "walk", "walk_thread", "setup")
TRAFFIC_TABLE = os.path.join(ROOT, "profiles", "dram_traffic_rmat22.md")


def kernel_name(kind, batched):
    return {"expand": "k_coop_fast" if batched else "k_expand_warp", "select": "k_select_fast",
            "select_thread": "k_select_thread",
            "hub": "k_select_hub", "pair": "k_select_pair", "heavy": "k_expand_heavy",
            "walk": "k_walk_fast" if batched else "k_walk_warp",
            "walk_thread": "k_walk_thread_fast" if batched else "k_walk_thread", "setup": "setup"}[kind]


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_per_item():
    """DRAM bytes per work item of each kernel, from the committed ncu summary
    (a capture of the same step at R-MAT scale 22: dram__bytes_read.sum +
    dram__bytes_write.sum over one step's launches / the step's items)."""
    out = {}
    if not os.path.exists(TRAFFIC_TABLE):
        return out
    with open(TRAFFIC_TABLE) as f:
        for line in f:
            m = re.match(r"\|\s*(k_\w+)\s*\|\s*([\d.]+)\s*\|\s*([\d.]+)\s*\|\s*([\d.]+)\s*\|\s*([\d.]+)\s*\|", line)
            if m:
                out[m.group(1)] = float(m.group(5))
    return out


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



def workload(name, scale=25):
    """The workload spec, with the R-MAT one scaled to 2^scale vertices
    (samples and walks scaled alike) for smaller profiling runs."""
    wl = {k: (dict(v) if isinstance(v, dict) else v) for k, v in WORKLOADS[name].items()}
    if name == "rmat25" and scale != 25:
        wl["graph"]["scale"] = scale
        for j in ("a", "b"):
            wl[j]["n_samples"] = max(1, wl[j]["n_samples"] >> (25 - scale))
    wl["name"] = wl["name"].format(scale=wl["graph"].get("scale", 0))
    wl["text"] = wl["text"].format(na=f"{wl['a']['n_samples']:,}", nb=f"{wl['b']['n_samples']:,}")
    return wl


def build_graph(wl):
    from csaw import graphgen
    return getattr(graphgen, wl["generator"])(**wl["graph"])


def workload_desc(wl):
    return {"workload": f"{wl['name']}: {wl['text']}", "graph": wl["graph"], "rowptr": "int64" if wl["rowptr64"]
            else "int32", "a": wl["a"], "b": wl["b"],
            "l2": "inputs larger than L2, and a 256 MiB buffer written between timed steps"}


def fanout(j):
    return [j["neighbor_size"]] * j["depth"] if j["mode"] == 0 else None


def oracle_sample(wl, g, threads):
    """A bounded seed subsample of the workload for the CPU oracle: the first
    cpu_fraction of the samples of (a) and of the walks of (b), with the
    same seeds (and so the same edges) as the GPU run gives them."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    A, B = wl["a"], wl["b"]
    na = max(1, int(A["n_samples"] * wl["cpu_fraction"]))
    nb = max(1, int(B["n_samples"] * wl["cpu_fraction"]))
    sa = oracle.make_seeds(g.rowptr, na * A["frontier_size"], wl["seeds"][0])
    sb = oracle.make_seeds(g.rowptr, nb, wl["seeds"][1])

    def rep():
        ea = oracle.run(g.rowptr, g.col, g.weight, sa, A["mode"], A["bias"], na, A["frontier_size"], A["depth"],
                        fanout(A), seed=wl["seeds"][0], n_threads=threads)
        eb = oracle.run(g.rowptr, g.col, g.weight, sb, B["mode"], B["bias"], nb, 1, B["depth"], None,
                        seed=wl["seeds"][1], n_threads=threads)
        return len(ea[0]) + len(eb[0])

    text = (f"the first {na:,} of {A['n_samples']:,} samples of (a) and {nb:,} of {B['n_samples']:,} walks of (b) "
            f"(same seeds and graph)")
    return rep, text


def run_reference(args):
    """The CPU oracle on all host threads, one bounded seed subsample of the
    workload per step.  The input graph is synthesised exactly as for the
    GPU arm (torch on the GPU for the R-MAT graph: input generation only);
    all sampling runs on the host."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    wl = workload(args.workload, args.scale)
    g = build_graph(wl)
    if wl["generator"] == "rmat_device":
        import torch
        torch.cuda.empty_cache()
    threads = os.cpu_count() or 1
    rep, text = oracle_sample(wl, g, threads)
    for _ in range(args.warmup):
        rep()
    t0 = time.perf_counter()
    edges = sum(rep() for _ in range(args.steps))
    dt = time.perf_counter() - t0
    v = edges / dt
    desc = workload_desc(wl)
    desc["sample"] = text + " per step"
    line = {"impl": "reference", "metric": "sampled_edges_per_sec", "value": v, "unit": "edges/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+int32", "data": "synthetic", "config": desc,
            "cpu_baseline": {"value": v, "unit": "edges/s", "cores": threads, "kind": "port",
                             "sample": desc["sample"]},
            "e2e": {"value": v, "unit": "edges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def cpu_baseline(wl, g, seconds=10.0):
    """Oracle timed on the host cores on a bounded sample (reported baseline only)."""
    threads = os.cpu_count() or 1
    rep, text = oracle_sample(wl, g, threads)
    edges, t0, reps = 0, time.perf_counter(), 0
    while True:
        edges += rep()
        reps += 1
        if time.perf_counter() - t0 > seconds:
            break
    dt = time.perf_counter() - t0
    return {"value": edges / dt, "unit": "edges/s", "cores": threads, "kind": "port",
            "sample": f"{reps} x ({text}), {dt:.1f} s"}


_M64 = (1 << 64) - 1


def _i64(c):
    return c - (1 << 64) if c >= 1 << 63 else c


def _mix(z):
    """splitmix64 finaliser on int64 tensors (wrapping arithmetic, logical shifts)."""
    z = z ^ ((z >> 30) & ((1 << 34) - 1))
    z = z * _i64(0xBF58476D1CE4E5B9)
    z = z ^ ((z >> 27) & ((1 << 37) - 1))
    z = z * _i64(0x94D049BB133111EB)
    return z ^ ((z >> 31) & ((1 << 33) - 1))


def edge_hash(out, n):
    """Order-independent hash of the multiset of (src, dst, sample) rows of an
    output: the wrapping sums of two independent 64-bit hashes of each edge,
    and the count (equal multisets give equal hashes in any order)."""
    import torch
    if n == 0:
        return "0:0:0"
    src, dst, smp = (out[i, :n].to(torch.int64) for i in range(3))
    x = (src & 0xFFFFFFFF) | (dst << 32)
    h1 = _mix(x ^ _mix(smp + 0x5851F42D))
    h2 = _mix(h1 ^ _i64(0xD6E8FEB86659FD93))
    return f"{n}:{int(h1.sum().item()) & _M64:016x}:{int(h2.sum().item()) & _M64:016x}"


def measure(args, wl, rank, world, local, headline=True):
    """Times the workload's forms and returns the JSON line's fields (rank 0)
    or None.  headline=False: an extra workload (fewer side measurements)."""
    import torch
    import csaw
    from csaw import dist as cdist
    t_gen = time.perf_counter()
    g = build_graph(wl)
    gen_s = time.perf_counter() - t_gen
    torch.cuda.empty_cache()
    G = csaw.Graph(g, rowptr64=wl["rowptr64"])
    stream = torch.cuda.current_stream()
    A, B = wl["a"], wl["b"]
    sa0, sb0 = wl["seeds"]
    seeds_a = G.make_seeds(A["n_samples"] * A["frontier_size"], sa0 + 7919 * rank)
    seeds_b = G.make_seeds(B["n_samples"], sb0 + 7919 * rank)
    # replicas (weak scaling): same job shape, rank-disjoint global sample ids
    scheds = (("plain", csaw.SCHED_PLAIN), ("batched", csaw.SCHED_BATCHED), ("learned", csaw.SCHED_LEARNED))
    params = {f: (cdist.replica_params(csaw.make_params(**A, seed=sa0, schedule=s), rank),
                  cdist.replica_params(csaw.make_params(**B, seed=sb0, schedule=s), rank)) for f, s in scheds}
    pa, pb = params["batched"]
    cap_a, cap_b = csaw.edge_bound(pa), csaw.edge_bound(pb)
    out_a = torch.empty((3, cap_a), dtype=torch.int32, device="cuda")
    out_b = torch.empty((3, cap_b), dtype=torch.int32, device="cuda")
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.int32, device="cuda")
    batch_jobs = {f: [csaw.BatchJob(params[f][0], seeds_a, cap_a, out_a, with_depth=False),
                      csaw.BatchJob(params[f][1], seeds_b, cap_b, out_b, with_depth=False)]
                  for f in ("batched", "learned")}
    last = {}
    # the plain form runs the first plain_fraction of the samples and walks
    # (same ids, seeds and so edges as in the full run); "sub" is the batched
    # form on that subsample, for the edge-multiset check
    frac = wl["plain_fraction"]
    sub_n = (max(1, int(A["n_samples"] * frac)), max(1, int(B["n_samples"] * frac)))

    def subsample(p, n):
        q = cdist.replica_params(p, 0)   # a copy
        q.n_samples = n
        return q

    params["sub"] = tuple(subsample(p, n) for p, n in zip(params["batched"], sub_n))
    plain_params = tuple(subsample(p, n) for p, n in zip(params["plain"], sub_n))
    sub_seeds = (seeds_a[:sub_n[0] * A["frontier_size"]], seeds_b[:sub_n[1]])
    batch_jobs["sub"] = [csaw.BatchJob(params["sub"][0], sub_seeds[0], cap_a, out_a, with_depth=False),
                         csaw.BatchJob(params["sub"][1], sub_seeds[1], cap_b, out_b, with_depth=False)]

    def step(form):
        if form == "plain":   # one job after the other, as the reference runs them
            qa, qb = plain_params
            a = G.sample(qa, sub_seeds[0], capacity=cap_a, out=out_a, with_depth=False)
            b = G.sample(qb, sub_seeds[1], capacity=cap_b, out=out_b, with_depth=False)
            last["n"] = (a[0].numel(), b[0].numel())
        else:
            res = G.sample_batch(batch_jobs[form])   # both workloads as one batch
            last["n"] = (res[0][0].numel(), res[1][0].numel())
        return sum(last["n"])

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def timed(form, steps, warmup, clocks=None, profile=False):
        """steps device-timed steps (L2 flushed before each); returns edges, ms,
        kernel stats, launches, clocks.  profile=True brackets every kernel with
        CUDA events on its own stream (no CUDA-graph replay)."""
        for _ in range(warmup):
            step(form)
        G.profile(profile)
        launches0 = G.stats()["kernel_launches"]
        if clocks:
            clocks.start()
        barrier()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        edges = 0
        for i in range(steps):
            flush.zero_()
            evs[i][0].record(stream)
            edges += step(form)
            evs[i][1].record(stream)
        barrier()
        clk = clocks.stop() if clocks else None
        launches = G.stats()["kernel_launches"] - launches0
        ms = sum(x.elapsed_time(y) for x, y in evs)
        ks = {k: G.kernel_stats(k) for k in KINDS}
        G.profile(False)
        return edges, ms, ks, launches, clk

    def form_hash():
        return edge_hash(out_a, last["n"][0]) + "|" + edge_hash(out_b, last["n"][1])

    forms = [f.strip() for f in args.forms.split(",") if f.strip()]
    main_form = forms[-1]
    hashes, other, info = {}, {}, {}
    plain_ms = plain_k = plain_edges = None
    if "plain" in forms and main_form != "plain":
        # the plain form recomputes every expanded hub's prefix: its steps are
        # bounded by a time budget (first warm-up step measured)
        t0 = time.perf_counter()
        step("plain")
        torch.cuda.synchronize()
        one = time.perf_counter() - t0
        k = max(2, min(args.steps, int(args.plain_budget_s / max(one, 1e-6))))
        plain_edges, plain_ms, plain_k, _, _ = timed("plain", k, max(args.warmup - 1, 2), profile=True)
        info["plain_steps"] = k
        plain_edges, plain_ms = plain_edges / k, plain_ms / k
        info["plain_sample"] = (f"first {sub_n[0]:,} of {A['n_samples']:,} samples of (a) and {sub_n[1]:,} of "
                                f"{B['n_samples']:,} walks of (b)" if frac < 1 else "the whole step")
        info["plain_edges_per_step"] = plain_edges
        h_plain = form_hash()
        step("sub")
        if form_hash() != h_plain:
            raise SystemExit("plain and batched forms emitted different edge multisets on the plain sample")
        hashes["plain (sample)" if frac < 1 else "plain"] = h_plain
    tune = None
    if "batched" in forms:   # the launch-shape autotuner, on the batched form's own batch
        for _ in range(args.warmup):
            step("batched")
        tune = G.autotune(batch_jobs["batched"])
        if main_form != "batched":
            e, ms, _, _, _ = timed("batched", args.steps, 1)
            other["batched"] = ms / args.steps
            hashes["batched"] = form_hash()
    sched = None
    if "learned" in forms:
        # the learned scheduler: record execution profiles, train on the GPU
        G.sched_record(400_000)
        for _ in range(2):
            step("learned")
        t0 = time.perf_counter()
        loss = G.sched_train(epochs=400, lr=3e-3, seed=rank)
        train_s = time.perf_counter() - t0
        for _ in range(6):   # timed trial of the model against the degree rule
            step("learned")
        si = G.sched_info()
        sched = {"records": si["records"], "train_loss": loss, "train_s": train_s, "class_mask": si["class_mask"],
                 "kept_model": si["class_mask"] != 0x3}
    # per-kernel events for the roofline come from a profiled pass of the same
    # steps; the reported value is the unprofiled pass (graph replay allowed)
    _, prof_ms, kstats, _, _ = timed(main_form, args.steps, args.warmup, profile=True)
    edges, ms, _, launches, clk = timed(main_form, args.steps, args.warmup, Clocks(local) if headline else None)
    hashes[main_form] = form_hash()
    edges_per_step = edges / args.steps
    if frac == 1 and plain_edges is not None and plain_edges != edges_per_step:
        raise SystemExit(f"plain and {main_form} forms emitted different edge counts: {plain_edges} vs "
                         f"{edges_per_step}")
    full = {k: v for k, v in hashes.items() if k != "plain (sample)"}
    if len(set(full.values())) != 1:
        raise SystemExit(f"forms emitted different edge multisets: {hashes}")
    qa, qb = params[main_form]

    # ---- end to end through the host-buffer entry point
    seeds_a_h = seeds_a.cpu().numpy()
    seeds_b_h = seeds_b.cpu().numpy()
    host_a = torch.empty((3, cap_a), dtype=torch.int32).pin_memory().numpy()
    host_b = torch.empty((3, cap_b), dtype=torch.int32).pin_memory().numpy()
    sa_pin = torch.from_numpy(seeds_a_h).pin_memory().numpy()
    sb_pin = torch.from_numpy(seeds_b_h).pin_memory().numpy()
    host_jobs = [csaw.BatchJob(qa, sa_pin, cap_a, host_a, with_depth=False, host=True),
                 csaw.BatchJob(qb, sb_pin, cap_b, host_b, with_depth=False, host=True)]

    def e2e_step():
        if main_form == "plain":
            ra = G.sample_host(qa, sa_pin, capacity=cap_a, out=host_a, with_depth=False, stream=stream.cuda_stream)
            rb = G.sample_host(qb, sb_pin, capacity=cap_b, out=host_b, with_depth=False, stream=stream.cuda_stream)
        else:
            ra, rb = G.sample_batch(host_jobs, stream=stream.cuda_stream)
        return ra[0].size + rb[0].size

    e2e_steps = max(3, args.steps // 2)

    def e2e_time(parts):
        # parts: CSAW_OPT_HOST_PARTS (0 = by output size; -1 = copy after sampling)
        G.set_option(csaw._lib.OPT_HOST_PARTS, parts)
        for _ in range(2):
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
    if e2e_edges != edges_per_step * e2e_steps:
        raise SystemExit(f"host-buffer run emitted {e2e_edges / e2e_steps} edges per step, device run "
                         f"{edges_per_step}")

    mdrw = None
    if not headline:
        # MDRW, as the reference dispatches FrontierSize > 1 (main.cu:281-288):
        # 4000 degree-biased samples, frontier 4, 3 steps (timed separately)
        pm = cdist.replica_params(csaw.make_params(2, 1, 4000, 4, 20, 3, seed=sa0 ^ 0x5A,
                                                   schedule=csaw.SCHED_BATCHED), rank)
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
        _, batched_t = cdist.reduce_totals(0, other.get("batched", 0.0) / 1e3)
    else:
        all_edges, t_max, e2e_all, e2e_t = float(edges), t_s, float(e2e_edges), e2e_ms / 1e3
        one_all, one_t = float(one_edges), one_ms / 1e3
        plain_t = (plain_ms or 0.0) / 1e3
        batched_t = other.get("batched", 0.0) / 1e3
    value = all_edges / t_max
    e2e_value = e2e_all / e2e_t
    plain_value = plain_edges * world / plain_t if plain_t else None   # the plain form's own edges per second

    peak, peak_kind = load_peaks()
    batched_form = main_form != "plain"
    timed_kinds = [k for k in KINDS if k != "setup" and kstats.get(k, {}).get("launches")]
    dom = max(timed_kinds, key=lambda k: kstats[k]["ms"])
    kd = kstats[dom]
    dname = kernel_name(dom, batched_form)
    achieved = kd["bytes"] / (kd["ms"] * 1e-3) / 1e9 if kd["ms"] > 0 else None
    per_item = traffic_per_item().get(dname)
    items_per_launch = kd["items"] / kd["launches"]
    roofline = {"bound": "hbm", "kernel": dname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind + " (hbm_gbs copy)",
                "traffic": per_item * items_per_launch if per_item else None,
                "traffic_source": (f"ncu dram__bytes_read.sum + dram__bytes_write.sum per item of {dname}, "
                                   f"{os.path.relpath(TRAFFIC_TABLE, ROOT)} (R-MAT scale 22 capture of the same "
                                   f"step), x {items_per_launch:.0f} items per launch") if per_item else
                                  "no committed capture for this kernel",
                "algorithmic_bytes_per_launch": kd["bytes"] / kd["launches"],
                "items_per_launch": items_per_launch, "launch_ms": kd["ms"] / kd["launches"],
                "step_counted_bytes": sum(v["bytes"] for v in kstats.values()) / args.steps,
                "step_frac": sum(v["bytes"] for v in kstats.values()) / args.steps / (ms / args.steps * 1e-3)
                / 1e9 / peak,
                "note": "per-kernel CUDA events on the job streams, from a profiled pass of the same steps "
                        "(kernel by kernel, no graph replay); the neighbor and walk jobs overlap, so each "
                        "kernel's time includes sharing the GPU; step_frac = all kernels' counted bytes / "
                        "the unprofiled step time"}
    res = {"value": value, "ms_per_step": ms / args.steps, "edges_per_step": all_edges / args.steps / world,
           "config": workload_desc(wl), "graph_stats": {"n_vertices": g.n_vertices, "n_edges": g.n_edges,
                                                        "max_degree": int(np.diff(g.rowptr).max()),
                                                        "generate_s": gen_s},
           "e2e": {"value": e2e_value, "unit": "edges/s",
                   "h2d_bytes_per_step": 4 * (seeds_a_h.size + seeds_b_h.size),
                   "d2h_bytes_per_step": int(12 * e2e_edges / e2e_steps)},
           "e2e_detail": {"host_parts": "by output size (CSAW_OPT_HOST_PARTS 0; edges copied back after every hop "
                                        "and every sample range)",
                          "no_overlap_value": one_all / one_t,
                          "note": "no_overlap_value: the same calls with every host job's edges copied back "
                                  "after all of its sampling (CSAW_OPT_HOST_PARTS -1)"},
           "gpu_launches": int(launches), "clocks": clk, "roofline": roofline,
           "kernels": {k: v for k, v in kstats.items() if v["launches"]},
           "profiled_pass_ms_per_step": prof_ms / args.steps,
           "forms": {main_form: value, "plain": plain_value,
                     "speedup_vs_plain": value / plain_value if plain_value else None,
                     # batched_t: seconds per step (max over ranks); t_max: all K steps
                     **({"batched": all_edges / args.steps / batched_t} if batched_t else {}),
                     **({"learned_vs_batched": batched_t / (t_max / args.steps)}
                        if batched_t and main_form == "learned" else {}),
                     "edge_multiset_hash": hashes, "scheduler": sched, "autotune": tune, **info,
                     "plain_kernels": {k: v for k, v in (plain_k or {}).items() if v["launches"]}}}
    if mdrw:
        res["mdrw"] = mdrw
    G.close()
    del host_a, host_b, out_a, out_b
    torch.cuda.empty_cache()
    return res, g


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
    """Page-locked (2, cls) int32 output buffers by power-of-two size class,
    carved from page-locked arenas allocated before timing: allocating
    page-locked memory takes the CUDA driver's lock for milliseconds, which
    would stall the request loop's worker mid-stream.  A class that runs out
    falls back to a fresh allocation, counted in `misses`."""

    def __init__(self):
        self.free = {}
        self.arenas = []
        self.misses = 0

    @staticmethod
    def cls_of(cap):
        return max(1 << 12, 1 << int(np.ceil(np.log2(max(cap, 1)))))

    def get(self, cap):
        import torch
        cls = self.cls_of(cap)
        lst = self.free.setdefault(cls, [])
        if lst:
            return cls, lst.pop()
        self.misses += 1
        return cls, torch.empty((2, cls), dtype=torch.int32).pin_memory()

    def put(self, cls, buf):
        self.free[cls].append(buf)

    def prefill(self, counts):
        """counts: {class: buffers}; one page-locked arena holds them all."""
        import torch
        total = sum(2 * c * n for c, n in counts.items())
        arena = torch.empty(total, dtype=torch.int32).pin_memory()
        self.arenas.append(arena)
        off = 0
        for c, n in sorted(counts.items()):
            lst = self.free.setdefault(c, [])
            for _ in range(n):
                lst.append(arena[off:off + 2 * c].view(2, c))
                off += 2 * c


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
    # every output class a request can need, with room for bursts of
    # outstanding requests (the waiter returns buffers in submission order)
    top = PinnedPool.cls_of(8192 * (15 + 150 + 750))
    pool.prefill({1 << k: (64 if (1 << k) <= (1 << 19) else 32 if (1 << k) <= (1 << 21) else 16)
                  for k in range(12, int(np.log2(top)) + 1)})
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
    misses0 = pool.misses
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
                     "peak_device_bytes": st["peak_device_bytes"],
                     "max_worker_call_ms": st["max_worker_call_ms"],
                     "worker_calls_over_1ms": st["worker_calls_over_1ms"],
                     "pinned_allocations_while_timed": pool.misses - misses0}
        misses0 = pool.misses
    S.close()
    G.close()
    return res



STREAM_GRAPH = dict(edge_factor=16, a=0.57, b=0.19, c=0.19, seed=29, weight="uniform")
EXTRA_STREAM_SHAPE = (24, 1.0, 16)   # scale, device budget (GiB), partition bits of the default line's key


def streaming(args):
    """Streaming (out-of-budget) workload: R-MAT (.57/.19/.19) at
    --stream-scale (default 26), edge factor 16, directed, U(0,1] weights
    (generated on the GPU; scales >= 27 per source range), adjacency in
    page-locked host memory, the device partition budget capped at
    --stream-budget-gb with 2^--stream-pbits-vertex partitions; one step =
    --stream-walks edge-weight-biased walks of length 20 and --stream-samples
    edge-weight-biased samples F1 N10 D2; with --stream-read-in-place 1
    (default) partitions outside the device arena are read in place from
    page-locked host memory (0: copied in and evicted by sweeps); with
    --stream-cache 1 (default) the
    streaming graph's weight-bias prefix cache is built first and streamed in
    place of the weights.  The defaults are 1/8 of the
    scale-29 configuration (131,072 walks, 32,768 samples, 4 GiB, 2^17-vertex
    partitions: 512, as many as scale 29 has); the configuration's own shape
    is --stream-scale 28 --stream-budget-gb 32 --stream-pbits 20
    --stream-walks 1048576 --stream-samples 262144.  The same jobs on the
    in-memory graph (plain schedule; the batched one too when the graph is
    small enough) check the edges by multiset hash and give the reference
    time."""
    import torch
    import csaw
    from csaw import graphgen
    torch.cuda.set_device(0)
    sc = args.stream_scale
    t0 = time.perf_counter()
    if sc >= 27:
        g = graphgen.rmat_device_bucketed(scale=sc, **{k: v for k, v in STREAM_GRAPH.items()})
    else:
        g = graphgen.rmat_device(scale=sc, symmetrize=False, **STREAM_GRAPH)
    gen_s = time.perf_counter() - t0
    torch.cuda.empty_cache()
    budget = int(args.stream_budget_gb * (1 << 30))
    nw, ns, pbits = args.stream_walks, args.stream_samples, args.stream_pbits
    res = {"graph": {"workload": f"rmat{sc}_ef16_uniform", "n_vertices": g.n_vertices, "n_edges": g.n_edges,
                     "max_degree": int(np.diff(g.rowptr).max()), "generate_s": gen_s,
                     "host_adjacency_bytes": int(g.col.nbytes + g.weight.nbytes + g.rowptr.nbytes)},
           "partition_bits": pbits, "device_budget": budget,
           "walks": dict(n=nw, length=20), "samples": dict(n=ns, F=1, N=10, D=2)}
    pw = csaw.make_params(1, 2, nw, 1, 1, 20, seed=0x29A)
    ps = csaw.make_params(0, 2, ns, 1, 10, 2, seed=0x29B)
    pwb = csaw.make_params(1, 2, nw, 1, 1, 20, seed=0x29A, schedule=csaw.SCHED_BATCHED)
    psb = csaw.make_params(0, 2, ns, 1, 10, 2, seed=0x29B, schedule=csaw.SCHED_BATCHED)
    t0 = time.perf_counter()
    S = csaw.StreamGraph(g, partition_bits=pbits, slot_budget_bytes=budget, rowptr64=True)
    S.set_option(csaw._lib.STREAM_OPT_READ_IN_PLACE, args.stream_read_in_place)
    res["stream_setup_s"] = time.perf_counter() - t0
    res["read_in_place"] = bool(args.stream_read_in_place)
    if args.stream_cache:   # the weight-bias prefix, streamed in place of the weights
        t0 = time.perf_counter()
        S.cache(2)
        res["prefix_cache_build_s"] = time.perf_counter() - t0
    res["prefix_cache"] = bool(args.stream_cache)
    # the in-memory comparison needs the graph, its neighbor records and
    # prefix cache on the device beside the arena (28 bytes per edge)
    free = torch.cuda.mem_get_info()[0]
    in_memory = g.n_edges * 28 + g.rowptr.nbytes + (2 << 30) < free
    G = csaw.Graph(g, rowptr64=True) if in_memory else None
    if G is not None:
        sw = G.make_seeds(nw, 0x29C)
        ss = G.make_seeds(ns, 0x29D)
    else:   # seeds uniform over the non-isolated vertices
        rng = np.random.default_rng(0x29C)
        non = np.flatnonzero(np.diff(g.rowptr) > 0).astype(np.int32)
        sw = torch.from_numpy(non[rng.integers(0, non.size, nw)]).cuda()
        ss = torch.from_numpy(non[rng.integers(0, non.size, ns)]).cuda()
        res["check"] = ("none at this size: the in-memory graph does not fit beside the arena; the same path is "
                        "checked against the in-memory run at scale 28")
    outs = {k: torch.empty((3, csaw.edge_bound(p)), dtype=torch.int32, device="cuda") for k, p in (("w", pw), ("s", ps))}
    last = {}

    def step(obj, batched=False):
        a = obj.sample(pwb if batched else pw, sw, out=outs["w"], with_depth=False)
        b = obj.sample(psb if batched else ps, ss, out=outs["s"], with_depth=False)
        last["h"] = edge_hash(outs["w"], a[0].numel()) + "|" + edge_hash(outs["s"], b[0].numel())
        return a[0].numel() + b[0].numel()

    # above 2^31 edges the plain in-memory run (every hub step rebuilds a
    # prefix of up to millions of edges) would take minutes: compare with
    # the batched in-memory run only
    big = g.n_edges > (1 << 31)
    runs = [("stream", S, False, args.stream_warmup, args.steps)]
    if G is not None and not big:
        runs.append(("in_memory", G, False, 0, 1))
    if G is not None:
        runs.append(("in_memory_batched", G, True, args.stream_warmup, args.steps))
    hashes = {}
    for name, obj, bt, warm, steps in runs:
        for _ in range(warm):
            step(obj, bt)
        torch.cuda.synchronize()
        i0 = S.info() if name == "stream" else None
        t0 = time.perf_counter()
        e = sum(step(obj, bt) for _ in range(steps))
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / steps
        hashes[name] = last["h"]
        r = {"ms_per_step": dt * 1e3, "steps": steps, "warmup": warm, "edges_per_step": e / steps,
             "seps": e / steps / dt}
        if name == "stream":
            i1 = S.info()
            r["h2d_bytes_per_step"] = (i1["bytes_h2d"] - i0["bytes_h2d"]) / steps
            r["partition_loads_per_step"] = (i1["partition_loads"] - i0["partition_loads"]) / steps
            r["items_read_in_place_per_step"] = (i1["items_read_in_place"] - i0["items_read_in_place"]) / steps
            r["partitions"] = i1["n_partitions"]
            r["slots"] = i1["n_slots"]
            r["h2d_gbs"] = r["h2d_bytes_per_step"] / dt / 1e9
        res[name] = r
    if len(set(hashes.values())) != 1:
        raise SystemExit(f"streaming and in-memory runs emitted different edge multisets: {hashes}")
    res["edge_multiset_hash"] = hashes
    if G is not None:
        ref = "in_memory" if "in_memory" in res else "in_memory_batched"
        res["stream_vs_in_memory"] = {"reference": ref, "ratio": res["stream"]["seps"] / res[ref]["seps"]}
        G.close()
    S.close()
    return res


def profile_step(args):
    """For ncu captures of one step: the batched form's batch, W warm-up steps,
    one step, then one profiled step whose per-kernel items and counted bytes
    are printed (the same for every step).  No autotuning, training, extra
    workloads or host copies."""
    import torch
    import csaw
    torch.cuda.set_device(0)
    wl = workload(args.workload, args.scale)
    g = build_graph(wl)
    torch.cuda.empty_cache()
    G = csaw.Graph(g, rowptr64=wl["rowptr64"])
    G.set_option(csaw._lib.OPT_CUDA_GRAPHS, 0)   # every step launches its kernels (ncu counts launches)
    A, B = wl["a"], wl["b"]
    sa = G.make_seeds(A["n_samples"] * A["frontier_size"], wl["seeds"][0])
    sb = G.make_seeds(B["n_samples"], wl["seeds"][1])
    pa = csaw.make_params(**A, seed=wl["seeds"][0], schedule=csaw.SCHED_BATCHED)
    pb = csaw.make_params(**B, seed=wl["seeds"][1], schedule=csaw.SCHED_BATCHED)
    oa = torch.empty((3, csaw.edge_bound(pa)), dtype=torch.int32, device="cuda")
    ob = torch.empty((3, csaw.edge_bound(pb)), dtype=torch.int32, device="cuda")
    jobs = [csaw.BatchJob(pa, sa, oa.shape[1], oa, with_depth=False),
            csaw.BatchJob(pb, sb, ob.shape[1], ob, with_depth=False)]
    for _ in range(args.warmup):
        G.sample_batch(jobs)
    torch.cuda.synchronize()
    r = G.sample_batch(jobs)
    torch.cuda.synchronize()
    G.profile(True)
    G.sample_batch(jobs)
    ks = {k: v for k, v in ((k, G.kernel_stats(k)) for k in KINDS) if v["launches"]}
    G.profile(False)
    print(json.dumps({"profile_step": {"workload": wl["name"], "edges": r[0][0].numel() + r[1][0].numel(),
                                       "kernels": {kernel_name(k, True): v for k, v in ks.items()}}}))
    G.close()


def profile_kernels(args):
    """Every kernel family once, on a graph far above L2, for per-kernel ncu
    captures (bench.py --profile-kernels under ncu --metrics): R-MAT
    (.6/.2/.15) scale 22, edge factor 16, int64 row offsets, Pareto(1.5)
    weights.  Runs, in order: the graph's prefix cache and neighbor records
    (first batched biased job), a batched F8 N10 D3 step with walks of 40
    (take-all, warp-list, pair, retry, thread-per-walk passes), a batched
    N 20 job (hub list), the plain schedule (warp expansion, CTA expansion,
    warp walks), batched warp walks, MDRW, per-sample dedup, profile
    recording and training of the learned scheduler, streaming through a
    512 MiB partition budget, and the allocation-free entry.  Prints the
    per-kind kernel statistics of each part."""
    import torch
    import csaw
    from csaw import _lib, graphgen
    torch.cuda.set_device(0)
    g = graphgen.rmat_device(scale=22, edge_factor=16, a=0.6, b=0.2, c=0.15, seed=25, symmetrize=False,
                             weight="pareto:1.5")
    torch.cuda.empty_cache()
    G = csaw.Graph(g, rowptr64=True)
    G.set_option(_lib.OPT_CUDA_GRAPHS, 0)
    out = {}

    def part(name, fn):
        G.profile(True)
        fn()
        torch.cuda.synchronize()
        out[name] = {k: v for k, v in ((k, G.kernel_stats(k)) for k in KINDS + ("mdrw", "persist")) if v["launches"]}
        G.profile(False)

    def job(mode, bias, n, F, N, D, fan=None, sched=csaw.SCHED_BATCHED, dedup=False, seed=1):
        p = csaw.make_params(mode, bias, n, F, N, D, fan, seed=seed, schedule=sched, dedup=dedup)
        seeds = G.make_seeds(n * (1 if mode == 1 else F), seed)
        o = torch.empty((3, csaw.edge_bound(p)), dtype=torch.int32, device="cuda")
        return csaw.BatchJob(p, seeds, o.shape[1], o, with_depth=False)

    step = [job(0, 2, 8192, 8, 10, 3, seed=2), job(1, 2, 131072, 1, 1, 40, seed=3)]
    part("cache_build_and_first_step", lambda: G.sample_batch(step))
    part("batched_step", lambda: G.sample_batch(step))
    part("batched_n20_hubs", lambda: G.sample_batch([job(0, 2, 2048, 4, 20, 2, seed=4)]))
    part("plain", lambda: G.sample_batch([job(0, 2, 256, 8, 10, 3, sched=csaw.SCHED_PLAIN, seed=5),
                                          job(1, 2, 2048, 1, 1, 40, sched=csaw.SCHED_PLAIN, seed=6)]))
    part("batched_warp_walks", lambda: G.sample_batch([job(1, 2, 4096, 1, 1, 40, seed=7)]))
    part("mdrw", lambda: G.sample_batch([job(2, 1, 8192, 8, 1, 20, seed=8)]))
    part("dedup", lambda: G.sample_batch([job(0, 2, 4096, 4, 10, 3, dedup=True, seed=9)]))
    learn = [job(0, 2, 4096, 8, 10, 3, sched=csaw.SCHED_LEARNED, seed=10)]
    G.sched_record(100_000)

    def learned():
        G.sample_batch(learn)
        G.sched_train(epochs=20, lr=3e-3, seed=1)
        G.sample_batch(learn)
    part("learned_record_train", learned)
    S = csaw.StreamGraph(g, partition_bits=16, slot_budget_bytes=512 << 20, rowptr64=True)
    ps = csaw.make_params(0, 2, 2048, 1, 10, 2, seed=11)
    pw = csaw.make_params(1, 2, 8192, 1, 1, 20, seed=12)
    ss, sw = G.make_seeds(2048, 11), G.make_seeds(8192, 12)
    S.sample(ps, ss)
    S.sample(pw, sw)
    torch.cuda.synchronize()
    out["stream"] = {"partition_loads": S.info()["partition_loads"], "kernel_launches": S.info()["kernel_launches"]}
    S.close()
    pn = csaw.make_params(0, 0, 2048, 2, 10, 3, seed=13)
    on = torch.empty((4, csaw.edge_bound(pn)), dtype=torch.int32, device="cuda")
    G.sample_noalloc(pn, G.make_seeds(4096, 13), on)
    torch.cuda.synchronize()
    G.close()
    print(json.dumps({"profile_kernels": out}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="csaw", choices=["csaw", "reference"])
    ap.add_argument("--workload", default="rmat25", choices=sorted(WORKLOADS))
    ap.add_argument("--scale", type=int, default=25,
                    help="R-MAT scale of the rmat25 workload (samples and walks scale with 2^scale)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the power-law, serving and streaming extra keys")
    ap.add_argument("--plain-budget-s", type=float, default=20.0,
                    help="device time the plain form's timed steps may take (at least 2 steps)")
    ap.add_argument("--profile-step", action="store_true",
                    help="run W warm-up steps and one step of the batched form only (for ncu captures)")
    ap.add_argument("--profile-kernels", action="store_true",
                    help="run every kernel family once on R-MAT scale 22 (for per-kernel ncu captures)")
    ap.add_argument("--learned-gain", action="store_true",
                    help="time the degree rule vs the learned scheduler on a heavy-tailed R-MAT graph instead")
    ap.add_argument("--serve", action="store_true", help="run only the serving (request loop) workload")
    ap.add_argument("--stream", action="store_true", help="run only the streaming (out-of-budget) workload")
    ap.add_argument("--stream-scale", type=int, default=26)
    ap.add_argument("--stream-budget-gb", type=float, default=4.0)
    ap.add_argument("--stream-pbits", type=int, default=17)
    ap.add_argument("--stream-walks", type=int, default=1 << 17)
    ap.add_argument("--stream-samples", type=int, default=1 << 15)
    ap.add_argument("--stream-warmup", type=int, default=1, help="untimed streaming steps before timing")
    ap.add_argument("--stream-cache", type=int, default=1,
                    help="1: build the streaming graph's weight-bias prefix cache (streamed in place of weights)")
    ap.add_argument("--stream-read-in-place", type=int, default=1,
                    help="1: partitions outside the device arena are read in place from page-locked host memory; "
                         "0: copied in and evicted by sweeps")
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
    if args.profile_step:
        profile_step(args)
        return
    if args.profile_kernels:
        profile_kernels(args)
        return
    if args.serve:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps({"serving": serving(args)}))
        return

    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    wl = workload(args.workload, args.scale)
    res, g = measure(args, wl, rank, world, local, headline=True)
    if rank == 0:
        line = {"metric": "sampled_edges_per_sec", "value": res["value"], "unit": "edges/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+int32",
                "data": "synthetic (seeded generators; no dataset)", "config": res["config"],
                "e2e": res["e2e"], "gpu_launches": res["gpu_launches"], "clocks": res["clocks"],
                "roofline": res["roofline"]}
        line.update({k: v for k, v in res.items() if k not in line})
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline(wl, g)
        del g
        if world == 1 and not args.no_extras:
            if args.workload != "powerlaw":
                extra, _ = measure(args, workload("powerlaw"), rank, world, local, headline=False)
                line["powerlaw"] = {k: extra[k] for k in ("value", "ms_per_step", "edges_per_step", "config", "e2e",
                                                          "e2e_detail", "roofline", "kernels", "forms", "mdrw",
                                                          "gpu_launches")}
            line["serving"] = serving(args)
            # streaming at a size the default run affords (the full sizes
            # are --stream options): R-MAT scale 24, 1 GiB of partition
            # slots for about 2.2 GB of host adjacency, 2^16-vertex partitions
            sa = argparse.Namespace(**vars(args))
            sa.stream_scale, sa.stream_budget_gb, sa.stream_pbits = EXTRA_STREAM_SHAPE
            line["streaming"] = streaming(sa)
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
