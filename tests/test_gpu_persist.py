"""The persistent job kernel (CSAW_OPT_PERSISTENT): every level of a batched
neighbor job in one cooperative launch must give exactly the oracle's edges --
every bias kind, 32- and 64-bit row offsets, hub rows that need CTA rebuilds,
concurrent batches with CUDA-graph replay, and host-buffer jobs that post
their edge count after every level."""
import numpy as np
import pytest

import oracle
from conftest import sort_edges

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def csaw():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test without a CUDA device")
    import csaw as c
    c.lib()
    return c


def same(a, b):
    sa, sb = sort_edges(*a), sort_edges(*b)
    assert sa.shape == sb.shape, (sa.shape, sb.shape)
    assert np.array_equal(sa, sb)


def persistent_graph(csaw, g, rowptr64=False):
    from csaw import _lib
    G = csaw.Graph(g, rowptr64=rowptr64)
    G.set_option(_lib.OPT_PERSISTENT, 1)
    return G


def hub_seeds(g, n, seed, k=8):
    deg = np.diff(g.rowptr)
    hubs = np.argsort(deg)[-k:].astype(np.int32)
    return np.concatenate([hubs, oracle.make_seeds(g.rowptr, n - k, seed)]).astype(np.int32)


@pytest.mark.parametrize("which", ["powerlaw_small", "skewed_hubs", "rmat12_pareto"])
@pytest.mark.parametrize("rowptr64", [False, True])
@pytest.mark.parametrize("bias", [0, 1, 2])
@pytest.mark.parametrize("fan", [[20, 20, 20], [12, 6, 3], [10, 10, 10, 2], [3, 32]])
def test_persistent_neighbor_parity(csaw, request, which, rowptr64, bias, fan):
    import torch
    g = request.getfixturevalue(which)
    G = persistent_graph(csaw, g, rowptr64)
    n, F = 100, 2
    seeds = hub_seeds(g, n * F, 7 + bias)
    p = csaw.make_params(0, bias, n, F, fan[0], len(fan), fan, seed=0x9E + bias, schedule=csaw.SCHED_BATCHED)
    a = [x.cpu().numpy() for x in G.sample(p, torch.from_numpy(seeds).cuda())]
    b = oracle.run(g.rowptr, g.col, g.weight, seeds, 0, bias, n, F, len(fan), fan, seed=0x9E + bias, n_threads=8)
    assert len(b[0]) > 0
    same(a, b)
    assert G.kernel_stats("persist")["launches"] == 0   # profiling is off: no per-kind events
    G.close()


def test_persistent_kernel_is_the_one_launched(csaw, skewed_hubs):
    """With profiling on, a three-level job is one persistent launch (plus
    the seed queue), not the per-level passes."""
    import torch
    g = skewed_hubs
    G = persistent_graph(csaw, g)
    seeds = hub_seeds(g, 200, 3)
    p = csaw.make_params(0, 2, 100, 2, 10, 3, [10, 5, 3], seed=5, schedule=csaw.SCHED_BATCHED)
    G.sample(p, torch.from_numpy(seeds).cuda())   # builds the cache and records
    G.profile(True)
    G.sample(p, torch.from_numpy(seeds).cuda())
    st = {k: G.kernel_stats(k)["launches"] for k in ("persist", "expand", "select", "pair", "heavy", "hub")}
    G.profile(False)
    assert st["persist"] == 1 and st["expand"] == st["select"] == st["pair"] == st["heavy"] == st["hub"] == 0, st
    G.close()


def test_persistent_batches_replay_and_host_jobs(csaw, skewed_hubs):
    """Concurrent jobs (persistent neighbor jobs beside walks), captured and
    replayed as CUDA graphs, and the same jobs through host buffers (edge
    counts posted after every level, copies overlapping the launch)."""
    import torch
    g = skewed_hubs
    G = persistent_graph(csaw, g, rowptr64=True)
    specs = [(0, 2, 80, 2, 3, [10, 5, 3]), (1, 2, 300, 1, 25, None), (0, 1, 60, 4, 3, [20, 4, 2]),
             (0, 0, 50, 2, 2, [6, 6])]
    jobs, refs, hseeds = [], [], []
    for i, (mode, bias, n, F, depth, fan) in enumerate(specs):
        seeds = hub_seeds(g, n * F, 30 + i)
        p = csaw.make_params(mode, bias, n, F, (fan or [1])[0], depth, fan, 300 + i, schedule=csaw.SCHED_BATCHED)
        jobs.append(csaw.BatchJob(p, torch.from_numpy(seeds).cuda()))
        hseeds.append(seeds)
        refs.append(oracle.run(g.rowptr, g.col, g.weight, seeds, mode, bias, n, F, depth, fan, seed=300 + i,
                               n_threads=8))
    for _ in range(3):   # eager, captured, replayed
        for r, ref in zip(G.sample_batch(jobs), refs):
            same([x.cpu().numpy() for x in r], ref)
    hjobs = [csaw.BatchJob(j.params, s, host=True) for j, s in zip(jobs, hseeds)]
    for _ in range(2):
        for r, ref in zip(G.sample_batch(hjobs), refs):
            same(r, ref)
    G.close()
