"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle,
bit-exact on the multiset of (sample, depth, src, dst) after a canonical sort."""
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


SCHEDULES = [0, 1]   # plain, batched: both must equal the oracle


def gpu_run(csaw, csr, mode, bias, n, F, depth, fanout, seed, seeds, degree_bias=False, graph=None, schedule=0):
    import torch
    g = graph or csaw.Graph(csr, degree_bias=degree_bias)
    p = csaw.make_params(mode, bias, n, F, (fanout or [1])[0], depth, fanout, seed, schedule=schedule)
    out = g.sample(p, torch.from_numpy(np.ascontiguousarray(seeds, dtype=np.int32)).cuda())
    return [x.cpu().numpy() for x in out]


def oracle_run(csr, mode, bias, n, F, depth, fanout, seed, seeds):
    return oracle.run(csr.rowptr, csr.col, csr.weight, seeds, mode, bias, n, F, depth, fanout, seed=seed,
                      n_threads=8)


def assert_parity(a, b):
    sa, sb = sort_edges(*a), sort_edges(*b)
    assert sa.shape == sb.shape, (sa.shape, sb.shape)
    assert np.array_equal(sa, sb)


@pytest.mark.parametrize("sched", SCHEDULES)
def test_rmat16_unbiased_small_config(csaw, rmat16, sched):
    """R-MAT scale 16 ef 8, unbiased, 1000 samples, F 1, N 2, D 2, Philox seed 0."""
    g = rmat16
    seeds = oracle.make_seeds(g.rowptr, 1000, 0)
    a = gpu_run(csaw, g, 0, 0, 1000, 1, 2, [2, 2], 0, seeds, schedule=sched)
    b = oracle_run(g, 0, 0, 1000, 1, 2, [2, 2], 0, seeds)
    assert len(a[0]) > 0
    assert_parity(a, b)


@pytest.mark.parametrize("sched", SCHEDULES)
@pytest.mark.parametrize("bias", [0, 1, 2])
@pytest.mark.parametrize("fan", [[20, 20, 20], [3, 7], [1, 1, 1, 1], [32, 2]])
def test_powerlaw_neighbor_parity(csaw, powerlaw_small, bias, fan, sched):
    g = powerlaw_small
    n, F = 150, 4
    seeds = oracle.make_seeds(g.rowptr, n * F, 17)
    a = gpu_run(csaw, g, 0, bias, n, F, len(fan), fan, 0x1234, seeds, schedule=sched)
    b = oracle_run(g, 0, bias, n, F, len(fan), fan, 0x1234, seeds)
    assert_parity(a, b)


@pytest.mark.parametrize("sched", SCHEDULES)
@pytest.mark.parametrize("bias", [0, 1, 2])
def test_rmat_pareto_heavy_vertices(csaw, rmat12_pareto, bias, sched):
    """Hub vertices above the per-warp shared capacity take the CTA path."""
    g = rmat12_pareto
    deg = np.diff(g.rowptr)
    assert deg.max() > 1024
    hubs = np.argsort(deg)[-8:].astype(np.int32)
    seeds = np.concatenate([hubs, oracle.make_seeds(g.rowptr, 192, 2)]).astype(np.int32)
    a = gpu_run(csaw, g, 0, bias, 200, 1, 2, [25, 10], 77, seeds, schedule=sched)
    b = oracle_run(g, 0, bias, 200, 1, 2, [25, 10], 77, seeds)
    assert_parity(a, b)


@pytest.mark.parametrize("sched", SCHEDULES)
@pytest.mark.parametrize("bias", [0, 1, 2])
def test_walk_parity(csaw, powerlaw_small, bias, sched):
    g = powerlaw_small
    seeds = oracle.make_seeds(g.rowptr, 500, 5)
    a = gpu_run(csaw, g, 1, bias, 500, 1, 64, None, 9, seeds, schedule=sched)
    b = oracle_run(g, 1, bias, 500, 1, 64, None, 9, seeds)
    assert_parity(a, b)


@pytest.mark.parametrize("sched", SCHEDULES)
@pytest.mark.parametrize("bias", [0, 1, 2])
def test_walk_parity_hubs(csaw, rmat12_pareto, bias, sched):
    g = rmat12_pareto
    seeds = oracle.make_seeds(g.rowptr, 300, 6)
    a = gpu_run(csaw, g, 1, bias, 300, 1, 40, None, 10, seeds, schedule=sched)
    b = oracle_run(g, 1, bias, 300, 1, 40, None, 10, seeds)
    assert_parity(a, b)


@pytest.mark.parametrize("bias,F", [(0, 4), (1, 4), (1, 33), (1, 1)])
def test_mdrw_parity(csaw, powerlaw_small, bias, F):
    g = powerlaw_small
    seeds = oracle.make_seeds(g.rowptr, 100 * F, 8)
    a = gpu_run(csaw, g, 2, bias, 100, F, 50, None, 11, seeds)
    b = oracle_run(g, 2, bias, 100, F, 50, None, 11, seeds)
    assert_parity(a, b)


def test_hook_bias_equals_degree_bias(csaw, powerlaw_small):
    g = powerlaw_small
    seeds = oracle.make_seeds(g.rowptr, 400, 3)
    a = gpu_run(csaw, g, 0, 3, 100, 4, 3, [10, 5, 3], 5, seeds)
    b = gpu_run(csaw, g, 0, 1, 100, 4, 3, [10, 5, 3], 5, seeds)
    assert_parity(a, b)


def test_materialised_degree_bias_same_output(csaw, powerlaw_small):
    g = powerlaw_small
    seeds = oracle.make_seeds(g.rowptr, 400, 4)
    a = gpu_run(csaw, g, 0, 1, 100, 4, 3, [20, 20, 20], 6, seeds, degree_bias=True)
    b = gpu_run(csaw, g, 0, 1, 100, 4, 3, [20, 20, 20], 6, seeds, degree_bias=False)
    assert_parity(a, b)


def test_make_seeds_matches_oracle(csaw, rmat16):
    g = csaw.Graph(rmat16)
    s = g.make_seeds(5000, 123).cpu().numpy()
    assert np.array_equal(s, oracle.make_seeds(rmat16.rowptr, 5000, 123))


def test_host_buffers_equal_device_buffers(csaw, powerlaw_small):
    g = csaw.Graph(powerlaw_small)
    seeds = oracle.make_seeds(powerlaw_small.rowptr, 200, 1)
    p = csaw.make_params(0, 1, 50, 4, 20, 3, [20, 20, 20], 3)
    h = g.sample_host(p, seeds)
    d = gpu_run(csaw, powerlaw_small, 0, 1, 50, 4, 3, [20, 20, 20], 3, seeds, graph=g)
    assert_parity(h, d)


def test_capacity_error_reports_needed(csaw, powerlaw_small):
    g = csaw.Graph(powerlaw_small)
    seeds = oracle.make_seeds(powerlaw_small.rowptr, 40, 1)
    import torch
    p = csaw.make_params(0, 0, 10, 4, 5, 2, [5, 5], 3)
    full = g.sample(p, torch.from_numpy(seeds).cuda())
    with pytest.raises(csaw.CsawError) as ei:
        g.sample(p, torch.from_numpy(seeds).cuda(), capacity=3)
    assert ei.value.code == 3
    assert len(full[0]) > 3


def test_bad_seed_is_rejected(csaw, powerlaw_small):
    import torch
    g = csaw.Graph(powerlaw_small)
    p = csaw.make_params(0, 0, 2, 1, 5, 2, [5, 5], 3)
    with pytest.raises(csaw.CsawError) as ei:
        g.sample(p, torch.tensor([0, powerlaw_small.n_vertices + 5], dtype=torch.int32).cuda())
    assert ei.value.code == 1


def test_reference_compatible_sampler(csaw, powerlaw_small, tmp_path):
    """Sampler() on int64 beg.bin/csr.bin files: its edge count equals the
    oracle's on the file-loaded graph (the entry draws make_seeds(n * F, 56)
    and samples with the default hooks, i.e. degree bias, seed 56), and the
    same call through the handle API gives the oracle's edges."""
    import torch
    from csaw import graphgen
    beg, csr = tmp_path / "beg.bin", tmp_path / "csr.bin"
    graphgen.write_reference_format(powerlaw_small, beg, csr)
    g = graphgen.read_reference_format(beg, csr)
    G = csaw.Graph(g, rowptr64=True, degree_bias=True)   # what the entry builds from the files
    for n, F, N, D in ((100, 1, 5, 3), (50, 4, 1, 30)):   # FrontierSize > 1: MDRW, as main.cu:281-288
        r = csaw.Sampler(beg, csr, 400, 128, n, F, N, D)
        mode = 2 if F > 1 else 0
        seeds = oracle.make_seeds(g.rowptr, n * F, 56)
        ref = oracle.run(g.rowptr, g.col, None, seeds, mode, 1, n, F, D, [N] * D if mode == 0 else None, seed=56,
                         n_threads=8)
        assert r.sampled_edges == len(ref[0]) > 0 and r.time > 0
        p = csaw.make_params(mode, 3, n, F, N, D, None, seed=56)
        out = [x.cpu().numpy() for x in G.sample(p, torch.from_numpy(seeds).cuda())]
        assert_parity(out, ref)


def test_repeat_runs_identical(csaw, rmat12_pareto):
    g = rmat12_pareto
    seeds = oracle.make_seeds(g.rowptr, 300, 2)
    a = gpu_run(csaw, g, 0, 2, 300, 1, 3, [10, 5, 2], 4, seeds)
    b = gpu_run(csaw, g, 0, 2, 300, 1, 3, [10, 5, 2], 4, seeds)
    assert_parity(a, b)


@pytest.mark.parametrize("bias", [0, 1, 2])
def test_schedules_agree_on_tight_fanout(csaw, rmat12_pareto, bias):
    """N close to d forces collisions, phase rebuilds and zero-mass fills."""
    g = rmat12_pareto
    deg = np.diff(g.rowptr)
    pick = np.flatnonzero((deg > 20) & (deg < 40))[:300].astype(np.int32)
    a = gpu_run(csaw, g, 0, bias, len(pick), 1, 2, [20, 3], 21, pick, schedule=0)
    b = gpu_run(csaw, g, 0, bias, len(pick), 1, 2, [20, 3], 21, pick, schedule=1)
    c = oracle_run(g, 0, bias, len(pick), 1, 2, [20, 3], 21, pick)
    assert_parity(a, b)
    assert_parity(a, c)


def test_batch_jobs_equal_solo_runs(csaw, powerlaw_small, rmat12_pareto):
    """Concurrent jobs (neighbor, walk, MDRW, mixed biases) give exactly the
    edges each gives alone; host-buffer jobs too."""
    import torch
    g = csaw.Graph(powerlaw_small)
    specs = [(0, 1, 60, 4, 3, [20, 20, 20]), (1, 1, 200, 1, 64, None), (1, 2, 150, 1, 30, None),
             (0, 0, 80, 2, 2, [5, 5]), (2, 1, 40, 8, 20, None), (0, 2, 50, 1, 3, [10, 5, 2])]
    jobs, solo = [], []
    for i, (mode, bias, n, F, depth, fan) in enumerate(specs):
        seeds = oracle.make_seeds(powerlaw_small.rowptr, n * (1 if mode == 1 else F), 40 + i)
        p = csaw.make_params(mode, bias, n, F, (fan or [1])[0], depth, fan, 100 + i, schedule=1)
        jobs.append(csaw.BatchJob(p, torch.from_numpy(seeds).cuda(), host=(i % 2 == 1) and False))
        solo.append(gpu_run(csaw, powerlaw_small, mode, bias, n, F, depth, fan, 100 + i, seeds, graph=g,
                            schedule=1))
    res = g.sample_batch(jobs)
    for r, s in zip(res, solo):
        assert_parity([x.cpu().numpy() for x in r], s)
    hjobs = [csaw.BatchJob(j.params, j.seeds.cpu().numpy(), host=True) for j in jobs]
    for r, s in zip(g.sample_batch(hjobs), solo):
        assert_parity(r, s)


@pytest.mark.parametrize("mode,fan", [(0, [6, 4, 2]), (1, None), (2, None)])
def test_shards_union_equals_full_run(csaw, powerlaw_small, mode, fan):
    """Three shards (global sample ids via sample_base) give the full job's edges."""
    import torch
    from csaw import dist as cdist
    g = csaw.Graph(powerlaw_small)
    F = 1 if mode == 1 else 3
    n, depth = 120, (3 if mode == 0 else 25)
    seeds = oracle.make_seeds(powerlaw_small.rowptr, n * F, 9)
    full = csaw.make_params(mode, 1, n, F, (fan or [1])[0], depth, fan, seed=31, schedule=1)
    ref = g.sample(full, torch.from_numpy(seeds).cuda())
    parts = []
    for r in range(3):
        p, sl = cdist.shard_params(full, r, 3)
        parts.append([x.cpu().numpy() for x in g.sample(p, torch.from_numpy(seeds[sl]).cuda())])
    union = [np.concatenate([pp[i] for pp in parts]) for i in range(4)]
    assert_parity(union, [x.cpu().numpy() for x in ref])


@pytest.mark.parametrize("graphs", [1, 0])
def test_repeated_batches_replay_identically(csaw, powerlaw_small, graphs):
    """The second identical batch is captured into a CUDA graph, later ones
    replay it; every repetition returns the same edges (and the same as with
    graphs off)."""
    import torch
    from csaw import _lib
    g = csaw.Graph(powerlaw_small)
    g.set_option(_lib.OPT_CUDA_GRAPHS, graphs)
    sa = torch.from_numpy(oracle.make_seeds(powerlaw_small.rowptr, 400, 1)).cuda()
    sb = torch.from_numpy(oracle.make_seeds(powerlaw_small.rowptr, 300, 2)).cuda()
    jobs = [csaw.BatchJob(csaw.make_params(0, 1, 100, 4, 20, 3, [20, 20, 20], seed=5, schedule=1), sa),
            csaw.BatchJob(csaw.make_params(1, 1, 300, 1, 1, 40, None, seed=6, schedule=1), sb)]
    outs = []
    for _ in range(4):
        outs.append([[x.cpu().numpy() for x in r] for r in g.sample_batch(jobs)])
    for o in outs[1:]:
        for a, b in zip(o, outs[0]):
            assert_parity(a, b)
    ref = oracle_run(powerlaw_small, 0, 1, 100, 4, 3, [20, 20, 20], 5, sa.cpu().numpy())
    assert_parity(outs[-1][0], ref)


@pytest.mark.parametrize("sched", SCHEDULES)
def test_pinned_and_pageable_host_outputs(csaw, rmat12_pareto, sched):
    """Host-buffer jobs give the same edges into page-locked and pageable
    output arrays, for neighbor sampling and walks, alone and in a batch, and
    a too-small capacity fails."""
    import torch
    g = rmat12_pareto
    G = csaw.Graph(g)
    seeds = oracle.make_seeds(g.rowptr, 400, 4)
    for mode, fan, depth in ((0, [10, 5, 3], 3), (1, None, 30)):
        p = csaw.make_params(mode, 2, 400 if mode else 100, 1 if mode else 4, (fan or [1])[0], depth, fan, 11,
                             schedule=sched)
        cap = csaw.edge_bound(p)
        pinned = torch.empty((4, cap), dtype=torch.int32).pin_memory().numpy()
        a = G.sample_host(p, seeds, out=pinned)
        b = G.sample_host(p, seeds)
        assert len(a[0]) > 0
        assert_parity(a, b)
        jobs = [csaw.BatchJob(p, seeds, cap, torch.empty((4, cap), dtype=torch.int32).pin_memory().numpy(),
                              host=True), csaw.BatchJob(p, seeds, cap, host=True)]
        r = G.sample_batch(jobs)
        assert_parity(r[0], b)
        assert_parity(r[1], b)
    p = csaw.make_params(0, 2, 100, 4, 10, 2, [10, 5], 11, schedule=sched)
    small = torch.empty((4, 16), dtype=torch.int32).pin_memory().numpy()
    with pytest.raises(csaw.CsawError):
        G.sample_host(p, seeds, capacity=16, out=small)
