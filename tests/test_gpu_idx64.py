"""GPU parity of the 64-bit row-offset graph layout (the layout graphs of
2^31 or more edges use) against the CPU oracle: every kernel instantiation
for I = int64_t -- plain, batched and learned schedules, the per-vertex prefix
cache on and off, neighbor sampling, walks, MDRW, per-sample dedup, a
trained learned scheduler and the streaming path -- bit-exact on the
multiset of (sample, depth, src, dst) after a canonical sort.  The graphs are
small (64-bit offsets are forced), so the oracle finishes in seconds."""
import numpy as np
import pytest

import oracle
from conftest import sort_edges

pytestmark = pytest.mark.gpu

SCHEDULES = [0, 1, 2]   # plain, batched, learned (untrained: the degree rule)
CACHES = [None, False, True]   # default (batched schedules build it), never, always


@pytest.fixture(scope="module")
def csaw():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test without a CUDA device")
    import csaw as c
    c.lib()
    return c


_GRAPHS = {}


def graph64(csaw, csr, cache):
    key = (id(csr), cache)
    if key not in _GRAPHS:
        _GRAPHS[key] = csaw.Graph(csr, rowptr64=True, cdf_cache=cache)
    return _GRAPHS[key]


def run_gpu(csaw, G, mode, bias, n, F, depth, fan, seed, seeds, sched, dedup=False):
    import torch
    p = csaw.make_params(mode, bias, n, F, (fan or [1])[0], depth, fan, seed, schedule=sched, dedup=dedup)
    return [x.cpu().numpy() for x in G.sample(p, torch.from_numpy(np.ascontiguousarray(seeds, np.int32)).cuda())]


def run_oracle(csr, mode, bias, n, F, depth, fan, seed, seeds, dedup=False):
    return oracle.run(csr.rowptr, csr.col, csr.weight, seeds, mode, bias, n, F, depth, fan, seed=seed,
                      n_threads=8, flags=oracle.DEDUP if dedup else 0)


def same(a, b):
    sa, sb = sort_edges(*a), sort_edges(*b)
    assert sa.shape == sb.shape, (sa.shape, sb.shape)
    assert np.array_equal(sa, sb)


def hub_seeds(csr, n, seed, k=8):
    deg = np.diff(csr.rowptr)
    hubs = np.argsort(deg)[-k:].astype(np.int32)
    return np.concatenate([hubs, oracle.make_seeds(csr.rowptr, n - k, seed)]).astype(np.int32)


def test_graph_reports_64bit_offsets(csaw, rmat12_pareto):
    G = graph64(csaw, rmat12_pareto, None)
    assert G.rowptr_host.dtype == np.int64


@pytest.mark.parametrize("which", ["rmat12_pareto", "skewed_hubs"])
@pytest.mark.parametrize("cache", CACHES)
@pytest.mark.parametrize("sched", SCHEDULES)
@pytest.mark.parametrize("bias", [0, 1, 2])
def test_neighbor_int64(csaw, request, which, cache, sched, bias):
    g = request.getfixturevalue(which)
    G = graph64(csaw, g, cache)
    n, F, fan = 120, 2, [12, 6, 3]
    seeds = hub_seeds(g, n * F, 5 + bias)
    a = run_gpu(csaw, G, 0, bias, n, F, 3, fan, 0x64 + bias, seeds, sched)
    b = run_oracle(g, 0, bias, n, F, 3, fan, 0x64 + bias, seeds)
    assert len(b[0]) > 0
    same(a, b)


@pytest.mark.parametrize("which", ["rmat12_pareto", "skewed_hubs"])
@pytest.mark.parametrize("cache", CACHES)
@pytest.mark.parametrize("sched", SCHEDULES)
@pytest.mark.parametrize("bias", [0, 1, 2])
def test_walk_int64(csaw, request, which, cache, sched, bias):
    g = request.getfixturevalue(which)
    G = graph64(csaw, g, cache)
    seeds = hub_seeds(g, 400, 9 + bias)
    a = run_gpu(csaw, G, 1, bias, 400, 1, 30, None, 0x65 + bias, seeds, sched)
    b = run_oracle(g, 1, bias, 400, 1, 30, None, 0x65 + bias, seeds)
    same(a, b)


def test_many_walks_thread_per_walk_int64(csaw, skewed_hubs):
    """Enough biased walks over a cached prefix for the one-thread-per-walk kernel."""
    g = skewed_hubs
    G = graph64(csaw, g, None)
    seeds = hub_seeds(g, 160_000, 21)
    for bias in (1, 2):
        a = run_gpu(csaw, G, 1, bias, seeds.size, 1, 12, None, 0x66 + bias, seeds, 1)
        b = run_oracle(g, 1, bias, seeds.size, 1, 12, None, 0x66 + bias, seeds)
        same(a, b)


@pytest.mark.parametrize("sched", [0, 1])
@pytest.mark.parametrize("bias,F", [(0, 4), (1, 4), (1, 33)])
def test_mdrw_int64(csaw, skewed_hubs, sched, bias, F):
    g = skewed_hubs
    G = graph64(csaw, g, None)
    seeds = hub_seeds(g, 60 * F, 13)
    a = run_gpu(csaw, G, 2, bias, 60, F, 40, None, 0x67, seeds, sched)
    b = run_oracle(g, 2, bias, 60, F, 40, None, 0x67, seeds)
    same(a, b)


@pytest.mark.parametrize("sched", [0, 1])
@pytest.mark.parametrize("bias", [0, 2])
def test_dedup_int64(csaw, skewed_hubs, sched, bias):
    g = skewed_hubs
    G = graph64(csaw, g, None)
    seeds = hub_seeds(g, 100 * 2, 14)
    a = run_gpu(csaw, G, 0, bias, 100, 2, 3, [10, 5, 3], 0x68, seeds, sched, dedup=True)
    b = run_oracle(g, 0, bias, 100, 2, 3, [10, 5, 3], 0x68, seeds, dedup=True)
    same(a, b)


@pytest.mark.parametrize("bias", [1, 2])
def test_trained_learned_schedule_int64(csaw, skewed_hubs, bias):
    """Record profiles, train, then run with the model routing items to CTA
    widths: the edges stay the oracle's on a 64-bit-offset graph."""
    g = skewed_hubs
    G = csaw.Graph(g, rowptr64=True, cdf_cache=False)   # no cache: hubs need CTA-width prefix scans
    seeds = hub_seeds(g, 200 * 2, 15, k=6)
    ref = run_oracle(g, 0, bias, 200, 2, 3, [12, 6, 3], 0x69, seeds)
    same(run_gpu(csaw, G, 0, bias, 200, 2, 3, [12, 6, 3], 0x69, seeds, 2), ref)
    G.sched_record(200_000)
    for _ in range(3):
        same(run_gpu(csaw, G, 0, bias, 200, 2, 3, [12, 6, 3], 0x69, seeds, 2), ref)
    G.sched_train(epochs=200, lr=3e-3, seed=2)
    assert G.sched_info()["trained"]
    for _ in range(8):   # trial runs (model and degree rule alternate), then the kept rule
        same(run_gpu(csaw, G, 0, bias, 200, 2, 3, [12, 6, 3], 0x69, seeds, 2), ref)
    G.close()


def test_batch_jobs_int64(csaw, skewed_hubs):
    """Concurrent batched jobs with CUDA-graph replay on a 64-bit-offset graph."""
    import torch
    g = skewed_hubs
    G = graph64(csaw, g, None)
    specs = [(0, 2, 80, 2, 3, [10, 5, 3]), (1, 2, 300, 1, 25, None), (0, 1, 60, 4, 2, [20, 4]),
             (1, 1, 200, 1, 30, None)]
    jobs, refs = [], []
    for i, (mode, bias, n, F, depth, fan) in enumerate(specs):
        seeds = hub_seeds(g, n * F, 30 + i)
        p = csaw.make_params(mode, bias, n, F, (fan or [1])[0], depth, fan, 200 + i, schedule=1)
        jobs.append(csaw.BatchJob(p, torch.from_numpy(seeds).cuda()))
        refs.append(run_oracle(g, mode, bias, n, F, depth, fan, 200 + i, seeds))
    for _ in range(3):   # eager, captured, replayed
        for r, ref in zip(G.sample_batch(jobs), refs):
            same([x.cpu().numpy() for x in r], ref)


@pytest.mark.parametrize("bias", [0, 1, 2])
def test_stream_int64(csaw, skewed_hubs, bias):
    """Streaming with 64-bit offsets: partitions paged through a small budget."""
    import torch
    g = skewed_hubs
    sg = csaw.StreamGraph(g, partition_bits=12, slot_budget_bytes=3 << 20, rowptr64=True)
    seeds = hub_seeds(g, 150 * 2, 16 + bias)
    p = csaw.make_params(0, bias, 150, 2, 10, 3, [10, 5, 3], seed=0x6A)
    a = [x.cpu().numpy() for x in sg.sample(p, torch.from_numpy(seeds).cuda())]
    same(a, run_oracle(g, 0, bias, 150, 2, 3, [10, 5, 3], 0x6A, seeds))
    sw = hub_seeds(g, 300, 17 + bias)
    pw = csaw.make_params(1, bias, 300, 1, 1, 25, None, seed=0x6B)
    a = [x.cpu().numpy() for x in sg.sample(pw, torch.from_numpy(sw).cuda())]
    same(a, run_oracle(g, 1, bias, 300, 1, 25, None, 0x6B, sw))
    info = sg.info()
    assert info["bytes_h2d"] > 0 and info["partition_loads"] >= 1
    sg.close()
