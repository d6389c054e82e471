"""GPU parity at the benchmark sizes: the full power-law workload (875,713
vertices, 5,105,039 edges; 4000 degree-biased samples F4 N20 D3 and 4000
degree-biased walks of 64) under every schedule, and seed subsamples of the
two R-MAT workloads on their full graphs -- scale 22 (the serving graph, int32
row offsets) and scale 25 (516 M edges, 64-bit row offsets) -- against the
CPU oracle, bit-exact after a canonical sort.  The R-MAT graphs are generated
on the GPU (torch), so these tests need a few GB of device and host memory."""
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


def gpu(csaw, G, p, seeds):
    import torch
    return [x.cpu().numpy() for x in G.sample(p, torch.from_numpy(np.ascontiguousarray(seeds, np.int32)).cuda())]


def ora(g, p, seeds):
    return oracle.run(g.rowptr, g.col, g.weight, seeds, p.mode, p.bias, p.n_samples, p.frontier_size, p.depth,
                      [p.fanout[i] or p.neighbor_size for i in range(p.depth)] if p.mode == 0 else None,
                      seed=p.seed, n_threads=16)


@pytest.fixture(scope="module")
def powerlaw_full():
    from csaw import graphgen
    return graphgen.powerlaw_directed(n_vertices=875_713, n_edges=5_105_039, gamma=2.1, max_degree=460, seed=20,
                                      weight="lognormal")


def test_powerlaw_full_workload_every_schedule(csaw, powerlaw_full):
    """The benchmark's power-law step, plain / batched / learned (untrained,
    recording, trained) and as one two-job batch with graph replay."""
    import torch
    g = powerlaw_full
    G = csaw.Graph(g)
    sa = oracle.make_seeds(g.rowptr, 4000 * 4, 0xC5A0)
    sb = oracle.make_seeds(g.rowptr, 4000, 0xC5A1)

    def params(sched):
        return (csaw.make_params(0, 1, 4000, 4, 20, 3, seed=0xC5A0, schedule=sched),
                csaw.make_params(1, 1, 4000, 1, 1, 64, seed=0xC5A1, schedule=sched))

    ra, rb = ora(g, params(0)[0], sa), ora(g, params(0)[1], sb)
    assert len(ra[0]) > 1_000_000 and len(rb[0]) == 4000 * 64
    for sched in (0, 1, 2):
        pa, pb = params(sched)
        same(gpu(csaw, G, pa, sa), ra)
        same(gpu(csaw, G, pb, sb), rb)
    pa, pb = params(2)
    jobs = [csaw.BatchJob(pa, torch.from_numpy(sa).cuda()), csaw.BatchJob(pb, torch.from_numpy(sb).cuda())]
    G.sched_record(200_000)
    for _ in range(2):
        r = G.sample_batch(jobs)
    same([x.cpu().numpy() for x in r[0]], ra)
    G.sched_train(epochs=200, lr=3e-3, seed=0)
    for _ in range(8):   # the model's timed trial, then the kept rule; captured and replayed
        r = G.sample_batch(jobs)
        same([x.cpu().numpy() for x in r[0]], ra)
        same([x.cpu().numpy() for x in r[1]], rb)
    G.close()


def _rmat_case(csaw, spec, rowptr64, jobs):
    import torch
    from csaw import graphgen
    g = graphgen.rmat_device(**spec)
    torch.cuda.empty_cache()
    G = csaw.Graph(g, rowptr64=rowptr64)
    try:
        for mode, bias, n, F, depth, fan, seed, scheds in jobs:
            seeds = oracle.make_seeds(g.rowptr, n * F, seed)
            ref = None
            for sched in scheds:
                p = csaw.make_params(mode, bias, n, F, (fan or [1])[0], depth, fan, seed=seed, schedule=sched)
                if ref is None:
                    ref = ora(g, p, seeds)
                    assert len(ref[0]) > 0
                same(gpu(csaw, G, p, seeds), ref)
    finally:
        G.close()
        del g
        torch.cuda.empty_cache()


def test_rmat22_serving_graph_subsample(csaw):
    """The serving graph (R-MAT scale 22, edge factor 16, symmetrised, U(0,1]
    weights; 128 M edges): 512 seeds of each request kind."""
    spec = dict(scale=22, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=22, weight="uniform")
    _rmat_case(csaw, spec, False, [
        (0, 2, 512, 1, 2, [25, 10], 0x2201, (0, 1)),
        (0, 2, 512, 1, 3, [15, 10, 5], 0x2202, (0, 1)),
        (1, 2, 4096, 1, 40, None, 0x2203, (0, 1)),
    ])


def test_rmat25_learned_config_subsample(csaw):
    """The scale-25 learned-scheduler graph (R-MAT .6/.2/.15, edge factor 16,
    directed, Pareto(1.5) weights; 516 M edges, max degree ~1 M) with 64-bit
    row offsets: 512 samples F8 N10 D3 and 4096 walks of 40, edge-weight bias,
    under the plain, batched and learned (degree-rule) schedules."""
    spec = dict(scale=25, edge_factor=16, a=0.6, b=0.2, c=0.15, seed=25, symmetrize=False, weight="pareto:1.5")
    _rmat_case(csaw, spec, True, [
        (0, 2, 512, 8, 3, [10, 10, 10], 0x25A, (0, 1, 2)),
        (1, 2, 4096, 1, 40, None, 0x25B, (0, 1, 2)),
    ])
