"""csaw_sample_noalloc: neighbor sampling that allocates no device memory.

Callers such as a serving loop that reserved its memory budget up front, or
code running inside another framework's memory pool, cannot call cudaMalloc
while they sample; this entry point keeps its frontier queues and counters in
a fixed 32 MiB device array instead.  Its output must equal the regular entry
point's, on repeated calls (the shared array keeps the previous call's
contents, so the second call checks that the state is reset properly).
This file is collected last on purpose.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("c-saw_b200", "oracle", "tests"):
    if os.path.join(ROOT, sub) not in sys.path:
        sys.path.insert(0, os.path.join(ROOT, sub))

pytestmark = pytest.mark.gpu


def canon(src, dst, smp, dep):
    a = [np.asarray(x.cpu().numpy() if hasattr(x, "cpu") else x, dtype=np.int64) for x in (src, dst, smp, dep)]
    o = np.lexsort((a[1], a[0], a[3], a[2]))
    return np.stack([a[2][o], a[3][o], a[0][o], a[1][o]])


@pytest.fixture(scope="module")
def setup():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test without a CUDA device")
    import csaw
    from csaw import graphgen
    g = graphgen.powerlaw_directed(n_vertices=30_000, n_edges=175_000, max_degree=460, seed=9, weight="lognormal")
    G = csaw.Graph(g)     # residency is set-up work; the sampling call below allocates nothing
    return csaw, torch, g, G


@pytest.mark.parametrize("bias,fan", [(0, [10, 5, 3]), (1, [20, 20, 20]), (2, [8, 4])])
def test_noalloc_matches_regular_entry_twice(setup, bias, fan):
    csaw, torch, g, G = setup
    n, F = 300, 2
    seeds = torch.from_numpy(G.make_seeds(n * F, 17 + bias).cpu().numpy()).cuda()
    p = csaw.make_params(0, bias, n, F, fan[0], len(fan), fan, seed=1234 + bias, schedule=csaw.SCHED_PLAIN)
    ref = canon(*G.sample(p, seeds))
    cap = csaw.edge_bound(p)
    out = torch.empty((4, cap), dtype=torch.int32, device="cuda")   # caller-owned outputs
    for _ in range(2):
        got = canon(*G.sample_noalloc(p, seeds, out))
        assert got.shape == ref.shape and np.array_equal(got, ref)


def test_noalloc_rejects_jobs_beyond_its_scratch(setup):
    csaw, torch, g, G = setup
    p = csaw.make_params(0, 0, 20000, 4, 32, 3, [32, 32, 32], seed=1)   # largest level 81.9 M items
    seeds = torch.zeros(20000 * 4, dtype=torch.int32, device="cuda")
    out = torch.empty((2, 16), dtype=torch.int32, device="cuda")
    with pytest.raises(csaw.CsawError) as ei:
        G.sample_noalloc(p, seeds, out, with_sample=False, with_depth=False)
    assert ei.value.code == 1 and b"32 MiB" in csaw.lib().csaw_last_error()
