"""GPU tests of host-buffer jobs that copy edges back while they sample
(CSAW_OPT_HOST_PARTS): a job run as P consecutive sample ranges, its edges
posted after every hop and range, gives exactly the edges of the one-range
run and of the oracle, for all three modes and schedules, ragged splits,
page-locked and pageable outputs, alone and in a batch (eager, captured,
replayed); a capacity below the output still fails."""
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


# (mode, bias, samples, frontier size, fanout, depth): sample counts that no
# part count divides evenly
CASES = [
    (0, 2, 997, 2, [10, 5, 3], 3),
    (0, 1, 1000, 1, [25, 10], 2),
    (1, 2, 1003, 1, None, 40),
    (2, 1, 601, 4, None, 6),
]


def params(csaw, case, sched):
    mode, bias, n, F, fan, depth = case
    return csaw.make_params(mode, bias, n, F, (fan or [1])[0], depth, fan, seed=13, schedule=sched)


def seeds_for(g, case, shift=0):
    mode, _, n, F, _, _ = case
    return oracle.make_seeds(g.rowptr, n * (1 if mode == 1 else F), 7 + shift)


@pytest.mark.parametrize("sched", [0, 1, 2])
def test_parts_equal_one_part_and_oracle(csaw, rmat12_pareto, sched):
    import torch
    from csaw import _lib
    g = rmat12_pareto
    G = csaw.Graph(g)
    try:
        for case in CASES:
            mode, bias, n, F, fan, depth = case
            seeds = seeds_for(g, case)
            p = params(csaw, case, sched)
            G.set_option(_lib.OPT_HOST_PARTS, 1)
            one = sort_edges(*G.sample_host(p, seeds))
            ref = oracle.run(g.rowptr, g.col, g.weight, seeds, mode, bias, n, F, depth, fan, seed=13, n_threads=8)
            assert one.shape[1] > 0
            assert np.array_equal(one, sort_edges(*ref)), case
            cap = csaw.edge_bound(p)
            for P in (-1, 2, 3, 8):
                G.set_option(_lib.OPT_HOST_PARTS, P)
                pinned = torch.empty((4, cap), dtype=torch.int32).pin_memory().numpy()
                a = sort_edges(*G.sample_host(p, seeds, out=pinned))
                b = sort_edges(*G.sample_host(p, seeds))
                assert np.array_equal(a, one), (case, P)
                assert np.array_equal(b, one), (case, P)
    finally:
        G.close()


def test_parts_in_a_batch(csaw, rmat12_pareto):
    """Several multi-part host jobs and a device job in one batch, run
    eagerly, captured and replayed as a CUDA graph; then new seed values in
    the same host arrays (the replayed graph must see them)."""
    import torch
    from csaw import _lib
    g = rmat12_pareto
    G = csaw.Graph(g)
    try:
        def expected(seed_shift):
            G.set_option(_lib.OPT_HOST_PARTS, 1)
            out = []
            for case in CASES:
                seeds = seeds_for(g, case, seed_shift)
                out.append(sort_edges(*G.sample_host(params(csaw, case, 1), seeds)))
            out.append(out[1])
            return out

        first, second = expected(0), expected(1)
        jobs = []
        for case in CASES:
            p = params(csaw, case, 1)
            seeds = seeds_for(g, case, 0)
            cap = csaw.edge_bound(p)
            jobs.append(csaw.BatchJob(p, seeds, cap, torch.empty((4, cap), dtype=torch.int32).pin_memory().numpy(),
                                      host=True))
        pd = params(csaw, CASES[1], 1)
        sd = torch.from_numpy(seeds_for(g, CASES[1], 0)).cuda()
        jobs.append(csaw.BatchJob(pd, sd, csaw.edge_bound(pd)))
        G.set_option(_lib.OPT_HOST_PARTS, 4)
        st = torch.cuda.current_stream().cuda_stream

        def check(expect):
            res = G.sample_batch(jobs, stream=st)
            for r, e in zip(res, expect):
                got = sort_edges(*[x.cpu().numpy() if hasattr(x, "cpu") else x for x in r])
                assert np.array_equal(got, e)

        for _ in range(4):   # eager, capture, replay, replay
            check(first)
        for job, case in zip(jobs, CASES):
            job.seeds[:] = seeds_for(g, case, 1)   # same host arrays, new values
        jobs[-1].seeds.copy_(torch.from_numpy(seeds_for(g, CASES[1], 1)))
        second[-1] = second[1]
        check(second)
    finally:
        G.close()


def test_parts_capacity_error(csaw, rmat12_pareto):
    from csaw import _lib
    g = rmat12_pareto
    G = csaw.Graph(g)
    try:
        case = CASES[0]
        p = params(csaw, case, 1)
        seeds = seeds_for(g, case)
        G.set_option(_lib.OPT_HOST_PARTS, 1)
        n = G.sample_host(p, seeds)[0].size
        G.set_option(_lib.OPT_HOST_PARTS, 4)
        with pytest.raises(csaw.CsawError) as e:
            G.sample_host(p, seeds, capacity=n - 1)
        assert e.value.code == 3
        assert sort_edges(*G.sample_host(p, seeds, capacity=n)).shape[1] == n   # exactly enough
        for bad in (9, -2):
            with pytest.raises(csaw.CsawError):
                G.set_option(_lib.OPT_HOST_PARTS, bad)
    finally:
        G.close()
