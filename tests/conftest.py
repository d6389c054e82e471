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


def sort_edges(src, dst, smp, dep):
    src, dst, smp, dep = (np.asarray(x, dtype=np.int64) for x in (src, dst, smp, dep))
    o = np.lexsort((dst, src, dep, smp))
    return np.stack([smp[o], dep[o], src[o], dst[o]])
