"""GPU parity of per-sample vertex dedup (CSAW_PARAM_DEDUP): every schedule
equals the oracle bit for bit, with repeated seeds and revisits frequent."""
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


def gpu(csaw, G, bias, n, F, fan, seed, seeds, schedule, dedup=True):
    import torch
    p = csaw.make_params(0, bias, n, F, fan[0], len(fan), fan, seed, schedule=schedule, dedup=dedup)
    out = G.sample(p, torch.from_numpy(np.ascontiguousarray(seeds, dtype=np.int32)).cuda())
    return [x.cpu().numpy() for x in out]


def ref(g, bias, n, F, fan, seed, seeds):
    return oracle.run(g.rowptr, g.col, g.weight, seeds, 0, bias, n, F, len(fan), fan, seed=seed, n_threads=8,
                      flags=oracle.DEDUP)


@pytest.mark.parametrize("schedule", [0, 1, 2])
@pytest.mark.parametrize("bias", [0, 1, 2])
@pytest.mark.parametrize("fan", [[10, 5, 3], [25, 10], [4, 4, 4, 4]])
def test_dedup_parity(csaw, rmat12_pareto, schedule, bias, fan):
    g = rmat12_pareto
    G = csaw.Graph(g)
    n, F = 300, 3
    base = oracle.make_seeds(g.rowptr, 40, 3)
    rng = np.random.default_rng(1)
    seeds = base[rng.integers(0, base.size, n * F)]          # repeated seeds within samples
    a = gpu(csaw, G, bias, n, F, fan, 0x5EED, seeds, schedule)
    b = ref(g, bias, n, F, fan, 0x5EED, seeds)
    assert np.array_equal(sort_edges(*a), sort_edges(*b))
    full = gpu(csaw, G, bias, n, F, fan, 0x5EED, seeds, schedule, dedup=False)
    assert len(a[0]) < len(full[0])
    G.close()


def test_dedup_on_cached_hubs_and_batches(csaw, rmat12_pareto):
    """Dedup jobs in a concurrent batch (graph replay on the repeat) equal
    their solo runs and the oracle."""
    import torch
    jobs, refs = [], []
    G = csaw.Graph(rmat12_pareto)
    for i, (bias, fan) in enumerate(((2, [10, 10, 4]), (1, [6, 6, 6]))):
        g = rmat12_pareto
        seeds = oracle.make_seeds(g.rowptr, 200 * 2, 50 + i)
        p = csaw.make_params(0, bias, 200, 2, fan[0], len(fan), fan, 9 + i, schedule=1, dedup=True)
        jobs.append(csaw.BatchJob(p, torch.from_numpy(seeds).cuda()))
        refs.append(sort_edges(*ref(g, bias, 200, 2, fan, 9 + i, seeds)))
    for _ in range(3):
        res = G.sample_batch(jobs)
        for r, e in zip(res, refs):
            assert np.array_equal(sort_edges(*[x.cpu().numpy() for x in r]), e)
    G.close()


def test_dedup_rejections(csaw, powerlaw_small):
    import torch
    g = powerlaw_small
    G = csaw.Graph(g)
    seeds = torch.from_numpy(oracle.make_seeds(g.rowptr, 50, 1)).cuda()
    walk = csaw.make_params(1, 1, 50, 1, 1, 10, seed=1, schedule=1, dedup=True)
    with pytest.raises(csaw.CsawError):
        G.sample(walk, seeds)
    nb = csaw.make_params(0, 1, 50, 1, 5, 2, seed=1, schedule=0, dedup=True)
    out = torch.empty((4, csaw.edge_bound(nb)), dtype=torch.int32, device="cuda")
    with pytest.raises(csaw.CsawError):
        G.sample_noalloc(nb, seeds, out)
    G.close()
