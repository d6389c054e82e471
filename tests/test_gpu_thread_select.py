"""GPU parity of the thread class of the batched schedule (one thread per
biased item with N < d <= 32, the row's prefix in registers): forced on
every such item (CSAW_OPT_THREAD_SELECT = 2) it must give the oracle's edges
bit for bit on every bias, both row-offset widths, with and without the
prefix cache; the degree rule's use of it (large levels only) and turning it
off must not change the output; recording mode explores it as class 6."""
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


def run_gpu(csaw, G, bias, n, F, fan, seed, seeds, sched=1):
    import torch
    p = csaw.make_params(0, bias, n, F, fan[0], len(fan), fan, seed, schedule=sched)
    return [x.cpu().numpy() for x in G.sample(p, torch.from_numpy(np.ascontiguousarray(seeds, np.int32)).cuda())]


def same(a, b):
    sa, sb = sort_edges(*a), sort_edges(*b)
    assert sa.shape == sb.shape, (sa.shape, sb.shape)
    assert np.array_equal(sa, sb)


@pytest.mark.parametrize("which", ["rmat12_pareto", "skewed_hubs", "powerlaw_small"])
@pytest.mark.parametrize("rowptr64", [False, True])
@pytest.mark.parametrize("cache", [None, False])
@pytest.mark.parametrize("bias", [1, 2, 3])
def test_forced_thread_class_equals_oracle(csaw, request, which, rowptr64, cache, bias):
    from csaw import _lib
    g = request.getfixturevalue(which)
    G = csaw.Graph(g, rowptr64=rowptr64, cdf_cache=cache)
    G.set_option(_lib.OPT_THREAD_SELECT, 2)
    n, F = 150, 2
    for fan, seed in (([12, 6, 3], 0x7A1 + bias), ([4, 20], 0x7B1 + bias), ([2, 2, 2, 2], 0x7C1 + bias)):
        seeds = oracle.make_seeds(g.rowptr, n * F, seed)
        G.profile(True)
        a = run_gpu(csaw, G, bias, n, F, fan, seed, seeds)
        st = G.kernel_stats("select_thread")
        G.profile(False)
        b = oracle.run(g.rowptr, g.col, g.weight, seeds, 0, bias, n, F, len(fan), fan, seed=seed, n_threads=8)
        assert len(b[0]) > 0
        same(a, b)
        if fan[0] < 12:
            assert st["items"] > 0, "no item ran as a thread"
    G.close()


def test_rule_forced_and_off_agree_on_large_levels(csaw, rmat16):
    """8192 samples F8: the first level has 65,536 items, so the degree rule
    sends its N < d <= 32 items to the thread list (N <= 16)."""
    import torch
    from csaw import _lib
    g = rmat16
    G = csaw.Graph(g)
    seeds = oracle.make_seeds(g.rowptr, 8192 * 8, 0x7D)
    outs, items = {}, {}
    for mode in (1, 2, 0):
        G.set_option(_lib.OPT_THREAD_SELECT, mode)
        G.profile(True)
        outs[mode] = run_gpu(csaw, G, 2, 8192, 8, [5, 3], 0x7D1, seeds)
        items[mode] = G.kernel_stats("select_thread")["items"]
        G.profile(False)
    assert items[1] > 0 and items[2] >= items[1] and items[0] == 0
    same(outs[1], outs[0])
    same(outs[2], outs[0])
    # a sample of the samples against the oracle (sample ids are global, so
    # the first 64 samples of the job are the job of 64 samples)
    b = oracle.run(g.rowptr, g.col, g.weight, seeds[:64 * 8], 0, 2, 64, 8, 2, [5, 3], seed=0x7D1, n_threads=8)
    smp = outs[1][2]
    keep = smp < 64
    same([x[keep] for x in outs[1]], b)
    with pytest.raises(Exception):
        G.set_option(_lib.OPT_THREAD_SELECT, 3)
    G.close()
    del torch


def test_recording_explores_thread_class(csaw, rmat12_pareto):
    import torch
    g = rmat12_pareto
    G = csaw.Graph(g)
    seeds = oracle.make_seeds(g.rowptr, 400 * 2, 0x7E)
    ref = oracle.run(g.rowptr, g.col, g.weight, seeds, 0, 2, 400, 2, 3, [8, 4, 3], seed=0x7E1, n_threads=8)
    G.sched_record(100_000)
    for _ in range(3):
        same(run_gpu(csaw, G, 2, 400, 2, [8, 4, 3], 0x7E1, seeds, sched=2), ref)
    rec = G.sched_records()
    cls = set(np.unique(rec["cls"]).tolist())
    assert {0, 6} <= cls, cls
    small = rec["x"][:, 0] <= 5.0 + 1e-6     # log2 d <= 5: the thread class is valid
    assert set(np.unique(rec["cls"][rec["cls"] == 6])) == {6}
    assert np.all(small[rec["cls"] == 6])
    G.close()
    del torch
