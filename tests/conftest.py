import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("", "c-saw_b200", "oracle", "tests", "tests/golden"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libcsaw_b200.so")


@pytest.fixture(scope="session")
def rmat16():
    from csaw import graphgen
    return graphgen.rmat(16, 8, a=0.57, b=0.19, c=0.19, seed=0, symmetrize=True, weight="uniform")


@pytest.fixture(scope="session")
def rmat12_pareto():
    from csaw import graphgen
    return graphgen.rmat(12, 16, a=0.6, b=0.2, c=0.15, seed=3, symmetrize=True, weight="pareto:1.5")


@pytest.fixture(scope="session")
def powerlaw_small():
    from csaw import graphgen
    return graphgen.powerlaw_directed(n_vertices=20_000, n_edges=116_000, gamma=2.1, max_degree=460, seed=5,
                                      weight="lognormal")


def make_skewed_hubs():
    """Power-law graph (60k vertices) plus six hub rows of 600 to 50,000
    distinct neighbors: rows above 4096 edges (one-CTA prefix build), above
    1024 (both prefix index levels) and above 512 (hub and pair paths)."""
    from csaw import graphgen
    base = graphgen.powerlaw_directed(n_vertices=60_000, n_edges=300_000, gamma=2.1, max_degree=300, seed=11,
                                      weight="none")
    V = base.n_vertices
    src = np.repeat(np.arange(V, dtype=np.int64), np.diff(base.rowptr))
    dst = base.col.astype(np.int64)
    rng = np.random.default_rng(12)
    hubs = rng.choice(V, 6, replace=False)
    hs, hd = [src], [dst]
    for h, d in zip(hubs, (50_000, 12_000, 5_000, 2_100, 1_100, 600)):
        nb = rng.choice(V, d, replace=False)
        nb = nb[nb != h]
        hs.append(np.full(nb.size, h, dtype=np.int64))
        hd.append(nb.astype(np.int64))
    key = np.unique(np.concatenate(hs) * V + np.concatenate(hd))
    rowptr, col = graphgen._csr_from_edges(key // V, key % V, V)
    return graphgen.CSR(rowptr, col, graphgen.weights("pareto:1.5", col.size, 13), name="skewed_hubs")


@pytest.fixture(scope="session")
def skewed_hubs():
    return make_skewed_hubs()


def sort_edges(src, dst, smp, dep):
    src, dst, smp, dep = (np.asarray(x, dtype=np.int64) for x in (src, dst, smp, dep))
    o = np.lexsort((dst, src, dep, smp))
    return np.stack([smp[o], dep[o], src[o], dst[o]])
