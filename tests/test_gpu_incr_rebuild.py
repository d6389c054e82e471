"""GPU parity of the incremental hub rebuild (CTA retries of cached hubs
rebuild the zeroed prefix from per-tile summaries instead of rescanning the
row): on hub rows whose mass sits on a few neighbors spread over tiles and
groups, so retries rebuild several times and some run out of mass, the
edges equal the oracle's bit for bit with the incremental rebuild on and off,
on both row-offset widths."""
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


def make_concentrated_hubs():
    """A power-law graph (80k vertices) plus hub rows of 600 to 70,000
    neighbors whose weights put almost all the mass on a few neighbors:
    k heavy neighbors (weights 1e6 * 2^-i, i < k) at random positions, the
    rest weight 1, or 0 on the rows marked sparse (there, once the heavy
    neighbors are taken, no mass is left)."""
    from csaw import graphgen
    base = graphgen.powerlaw_directed(n_vertices=80_000, n_edges=320_000, gamma=2.1, max_degree=200, seed=31,
                                      weight="none")
    V = base.n_vertices
    src = np.repeat(np.arange(V, dtype=np.int64), np.diff(base.rowptr))
    dst = base.col.astype(np.int64)
    w = np.random.default_rng(32).pareto(1.5, dst.size).astype(np.float32) + 0.01
    rng = np.random.default_rng(33)
    hubs = rng.choice(V, 7, replace=False)
    spec = [(70_000, 6, False), (20_000, 3, False), (9_000, 12, False), (3_000, 5, True),
            (1_500, 2, False), (700, 8, True), (600, 20, False)]
    hs, hd, hw = [src], [dst], [w]
    for h, (d, k, sparse) in zip(hubs, spec):
        nb = np.sort(rng.choice(np.setdiff1d(np.arange(V), [h]), d, replace=False))
        ww = np.full(nb.size, 0.0 if sparse else 1.0, dtype=np.float32)
        heavy = rng.choice(nb.size, k, replace=False)
        ww[heavy] = (1e6 * 2.0 ** -np.arange(k)).astype(np.float32)
        hs.append(np.full(nb.size, h, dtype=np.int64))
        hd.append(nb.astype(np.int64))
        hw.append(ww)
    s, d, ww = np.concatenate(hs), np.concatenate(hd), np.concatenate(hw)
    key = s * V + d
    order = np.argsort(key, kind="stable")
    key, ww = key[order], ww[order]
    keep = np.ones(key.size, dtype=bool)
    keep[1:] = key[1:] != key[:-1]
    key, ww = key[keep], ww[keep]
    rowptr, col = graphgen._csr_from_edges(key // V, key % V, V)
    return graphgen.CSR(rowptr, col, ww.astype(np.float32), name="concentrated_hubs"), hubs


@pytest.fixture(scope="module")
def concentrated():
    return make_concentrated_hubs()


@pytest.mark.parametrize("rowptr64", [False, True])
@pytest.mark.parametrize("fan", [[10, 4], [16, 2], [6, 6]])
def test_incremental_rebuild_equals_oracle(csaw, concentrated, rowptr64, fan):
    import torch
    from csaw import _lib
    g, hubs = concentrated
    n, F = 600, 2
    seeds = np.concatenate([np.tile(hubs.astype(np.int32), (n * F) // (2 * hubs.size) + 1)[: n * F // 2],
                            oracle.make_seeds(g.rowptr, n * F - n * F // 2, 0x1C)]).astype(np.int32)
    seed = 0x1C0 + fan[0]
    ref = oracle.run(g.rowptr, g.col, g.weight, seeds, 0, 2, n, F, len(fan), fan, seed=seed, n_threads=8)
    G = csaw.Graph(g, rowptr64=rowptr64)
    p = csaw.make_params(0, 2, n, F, fan[0], len(fan), fan, seed, schedule=csaw.SCHED_BATCHED)
    sd = torch.from_numpy(seeds).cuda()
    retries = {}
    for incr in (1, 0, 1):
        G.set_option(_lib.OPT_INCR_REBUILD, incr)
        G.profile(True)
        out = [x.cpu().numpy() for x in G.sample(p, sd)]
        retries[incr] = G.kernel_stats("heavy")["items"]
        G.profile(False)
        a, b = sort_edges(*out), sort_edges(*ref)
        assert a.shape == b.shape and np.array_equal(a, b), f"incr={incr}"
    assert retries[1] > 0 and retries[0] == retries[1], retries
    G.close()


@pytest.mark.parametrize("bias", [1, 3])
def test_incremental_rebuild_other_biases(csaw, concentrated, bias):
    import torch
    from csaw import _lib
    g, hubs = concentrated
    n, F, fan = 400, 2, [12, 3]
    seeds = np.concatenate([np.tile(hubs.astype(np.int32), 60)[: n],
                            oracle.make_seeds(g.rowptr, n * F - n, 0x2C)]).astype(np.int32)
    ref = oracle.run(g.rowptr, g.col, g.weight, seeds, 0, bias, n, F, 2, fan, seed=0x2C1, n_threads=8)
    G = csaw.Graph(g)
    p = csaw.make_params(0, bias, n, F, fan[0], 2, fan, 0x2C1, schedule=csaw.SCHED_BATCHED)
    for incr in (1, 0):
        G.set_option(_lib.OPT_INCR_REBUILD, incr)
        out = [x.cpu().numpy() for x in G.sample(p, torch.from_numpy(seeds).cuda())]
        a, b = sort_edges(*out), sort_edges(*ref)
        assert a.shape == b.shape and np.array_equal(a, b), f"incr={incr}"
    G.close()
