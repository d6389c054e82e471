"""GPU parity of the per-vertex CDF cache (the canonical bias prefix built once
per graph and bias): every schedule with the cache off, built on demand and
forced on must equal the oracle bit for bit, including hub expansions whose
draws exhaust the heavy edges, so that the cached search gives up and the
item is rebuilt (with its selected edges zeroed) by the CTA pass."""
import numpy as np
import pytest

import oracle
from conftest import sort_edges

pytestmark = pytest.mark.gpu

HUB_DEGREES = [600, 700, 1500, 3000, 4100, 5000, 9000, 20000]


@pytest.fixture(scope="module")
def csaw():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test without a CUDA device")
    import csaw as c
    c.lib()
    return c


@pytest.fixture(scope="module")
def skewed_hubs():
    """Hubs 0..7 (degrees 600..20000, two above 4096 for the one-CTA-per-vertex
    build) whose first 24 edges point at other hubs with weight 1000 and whose
    other edges point at leaves with weight ~0.01; leaves have 1..3 edges."""
    from csaw import graphgen
    rng = np.random.default_rng(11)
    V = 30_000
    n_h = len(HUB_DEGREES)
    rows, cols, ws = [], [], []
    for h, d in enumerate(HUB_DEGREES):
        heavy = rng.integers(0, n_h, 24)
        light = rng.integers(1000, V, d - 24)
        rows.append(np.full(d, h))
        cols.append(np.concatenate([heavy, light]))
        ws.append(np.concatenate([np.full(24, 1000.0), rng.lognormal(-4.6, 0.5, d - 24)]))
    for v in range(n_h, V):
        d = int(rng.integers(1, 4))
        rows.append(np.full(d, v))
        cols.append(rng.integers(0, V, d))
        ws.append(rng.lognormal(0.0, 1.0, d))
    src = np.concatenate(rows)
    dst = np.concatenate(cols).astype(np.int32)
    w = np.concatenate(ws).astype(np.float32)
    o = np.argsort(src, kind="stable")
    rowptr = np.zeros(V + 1, dtype=np.int64)
    np.add.at(rowptr, src + 1, 1)
    rowptr = np.cumsum(rowptr)
    return graphgen.CSR(rowptr, dst[o], w[o], name="skewed_hubs")


def run_gpu(csaw, G, mode, bias, n, F, fan, seed, seeds, schedule):
    import torch
    p = csaw.make_params(mode, bias, n, F, fan[0], len(fan), fan, seed, schedule=schedule)
    out = G.sample(p, torch.from_numpy(np.ascontiguousarray(seeds, dtype=np.int32)).cuda())
    return [x.cpu().numpy() for x in out]


def run_oracle(g, mode, bias, n, F, fan, seed, seeds):
    return oracle.run(g.rowptr, g.col, g.weight, seeds, mode, bias, n, F, len(fan), fan, seed=seed, n_threads=8)


def assert_parity(a, b):
    sa, sb = sort_edges(*a), sort_edges(*b)
    assert sa.shape == sb.shape, (sa.shape, sb.shape)
    assert np.array_equal(sa, sb)


@pytest.mark.parametrize("cache", [None, True, False])
@pytest.mark.parametrize("schedule", [0, 1, 2])
@pytest.mark.parametrize("bias", [1, 2])
def test_hub_neighbor_parity(csaw, skewed_hubs, cache, schedule, bias):
    g = skewed_hubs
    G = csaw.Graph(g, cdf_cache=cache)
    hubs = np.repeat(np.arange(len(HUB_DEGREES), dtype=np.int32), 24)
    seeds = np.concatenate([hubs, oracle.make_seeds(g.rowptr, 400 - hubs.size, 5)]).astype(np.int32)
    fan = [32, 32, 4]
    a = run_gpu(csaw, G, 0, bias, 400, 1, fan, 0xC0FFEE, seeds, schedule)
    b = run_oracle(g, 0, bias, 400, 1, fan, 0xC0FFEE, seeds)
    assert len(a[0]) > 0
    assert_parity(a, b)
    G.close()


@pytest.mark.parametrize("cache", [None, True, False])
@pytest.mark.parametrize("schedule", [0, 1])
@pytest.mark.parametrize("bias", [1, 2])
def test_hub_walk_parity(csaw, skewed_hubs, cache, schedule, bias):
    g = skewed_hubs
    G = csaw.Graph(g, cdf_cache=cache)
    seeds = np.concatenate([np.arange(len(HUB_DEGREES), dtype=np.int32),
                            oracle.make_seeds(g.rowptr, 2000 - len(HUB_DEGREES), 9)]).astype(np.int32)
    a = run_gpu(csaw, G, 1, bias, 2000, 1, [1] * 40, 99, seeds, schedule)
    b = run_oracle(g, 1, bias, 2000, 1, [1] * 40, 99, seeds)
    assert_parity(a, b)
    G.close()


def test_cache_residency_policy(csaw, skewed_hubs):
    """The batched schedule builds the cache (4.13E bytes, plus the hub rows'
    tile summaries, 8 (E/32 + V + 1) bytes) on first biased use of a graph
    with hubs; the plain schedule does not unless asked; the opt-out flag
    keeps it off; an unbiased job never builds it."""
    g = skewed_hubs
    E = g.n_edges
    seeds = oracle.make_seeds(g.rowptr, 64, 1)

    def grows(cache, schedule, bias):
        G = csaw.Graph(g, cdf_cache=cache)
        before = G.stats()["device_bytes"]
        run_gpu(csaw, G, 0, bias, 64, 1, [8, 8], 1, seeds, schedule)
        after = G.stats()["device_bytes"]
        G.close()
        return after - before

    cache = 4 * (E + (E + 31) // 32 + (E + 1023) // 1024)   # prefix and its two search-index levels
    assert np.diff(g.rowptr).max() > 512
    cache += 8 * ((E >> 5) + g.n_vertices + 1)                 # tile summaries (rows above 512 edges)
    assert grows(None, 1, 2) - grows(False, 1, 2) == cache   # batched also adds neighbor records
    assert grows(None, 0, 2) == 0
    assert grows(True, 0, 2) == cache
    assert grows(None, 1, 0) == grows(False, 1, 0)


def test_cache_rebuilt_for_other_bias(csaw, skewed_hubs):
    """One graph alternating degree and edge-weight jobs rebuilds the cache for
    each bias and stays equal to the oracle."""
    g = skewed_hubs
    G = csaw.Graph(g)
    seeds = np.concatenate([np.arange(8, dtype=np.int32), oracle.make_seeds(g.rowptr, 120, 3)]).astype(np.int32)
    for bias in (1, 2, 1, 2):
        a = run_gpu(csaw, G, 0, bias, 128, 1, [32, 6], 7 + bias, seeds, 1)
        b = run_oracle(g, 0, bias, 128, 1, [32, 6], 7 + bias, seeds)
        assert_parity(a, b)
    G.close()


def test_plain_schedule_after_cache_built(csaw, skewed_hubs):
    """A batched job builds the cache; plain jobs on the same graph (which do
    not see it unless asked) still equal the oracle, walks and neighbors."""
    g = skewed_hubs
    G = csaw.Graph(g)
    seeds = np.concatenate([np.arange(8, dtype=np.int32), oracle.make_seeds(g.rowptr, 120, 4)]).astype(np.int32)
    for mode, fan, sched in ((0, [32, 6], 1), (1, [1] * 20, 0), (0, [32, 6], 0), (1, [1] * 20, 1)):
        a = run_gpu(csaw, G, mode, 2, 128, 1, fan, 5, seeds, sched)
        b = run_oracle(g, mode, 2, 128, 1, fan, 5, seeds)
        assert_parity(a, b)
    G.close()


@pytest.mark.parametrize("bias", [1, 2])
def test_many_biased_walks_thread_per_walk(csaw, rmat12_pareto, powerlaw_small, bias):
    """Enough biased walks on a cached prefix take the one-thread-per-walk
    kernel; its edges equal the oracle's (hub graph, and a small-degree graph
    with the cache forced on)."""
    for g, cache, n, length in ((rmat12_pareto, None, 120_000, 8), (powerlaw_small, True, 100_000, 20)):
        G = csaw.Graph(g, cdf_cache=cache)
        seeds = oracle.make_seeds(g.rowptr, n, 21)
        a = run_gpu(csaw, G, 1, bias, n, 1, [1] * length, 0xABC, seeds, 1)
        b = run_oracle(g, 1, bias, n, 1, [1] * length, 0xABC, seeds)
        assert len(a[0]) > n
        assert_parity(a, b)
        G.close()


@pytest.mark.parametrize("retry_smem", [16384, 98304])
@pytest.mark.parametrize("bias", [1, 2])
def test_retry_rebuild_in_shared_memory(csaw, skewed_hubs, retry_smem, bias):
    """The cached-hub retry pass rebuilding prefixes in shared memory
    (CSAW_OPT_RETRY_SMEM) gives the oracle's edges, for rows that fit and
    rows that do not."""
    from csaw import _lib
    g = skewed_hubs
    G = csaw.Graph(g)
    G.set_option(_lib.OPT_RETRY_SMEM, retry_smem)
    hubs = np.repeat(np.arange(len(HUB_DEGREES), dtype=np.int32), 24)
    seeds = np.concatenate([hubs, oracle.make_seeds(g.rowptr, 400 - hubs.size, 5)]).astype(np.int32)
    fan = [32, 32, 4]
    a = run_gpu(csaw, G, 0, bias, 400, 1, fan, 0xC0FFEE, seeds, 1)
    b = run_oracle(g, 0, bias, 400, 1, fan, 0xC0FFEE, seeds)
    assert_parity(a, b)
    G.close()
