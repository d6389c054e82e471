"""csaw_sample_noalloc: neighbor sampling that allocates no device memory.

Callers such as a serving loop that reserved its memory budget up front, or
code running inside another framework's memory pool, cannot call cudaMalloc
while they sample; this entry point keeps its frontier queues and counters in
a fixed 32 MiB device array instead.  Its output must equal the regular entry
point's, on repeated calls (the shared array keeps the previous call's
contents, so the second call checks that the state is reset properly), for
every bias kind, 64-bit row offsets and a graph with a cached bias prefix;
and a graph that only ever ran it holds no workspace.
This file is collected last on purpose.
"""
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
    return csaw, torch, g


def _params(csaw, bias, fan):
    return csaw.make_params(0, bias, 300, 2, fan[0], len(fan), fan, seed=1234 + bias, schedule=csaw.SCHED_PLAIN)


def test_noalloc_first_on_a_fresh_graph_holds_no_workspace(setup):
    """The no-allocation call runs before any regular call on a new graph:
    the graph's workspace stays empty and a second (warm) call leaves the
    device's free memory unchanged."""
    csaw, torch, g = setup
    G = csaw.Graph(g)     # residency is set-up work; the sampling calls below allocate nothing
    p = _params(csaw, 1, [20, 20, 20])
    seeds = G.make_seeds(300 * 2, 5)
    out = torch.empty((4, csaw.edge_bound(p)), dtype=torch.int32, device="cuda")   # caller-owned outputs
    torch.cuda.synchronize()
    first = canon(*G.sample_noalloc(p, seeds, out))
    assert G.stats()["workspace_bytes"] == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    again = canon(*G.sample_noalloc(p, seeds, out))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert G.stats()["workspace_bytes"] == 0
    assert np.array_equal(first, again)
    ref = canon(*G.sample(p, seeds))   # the regular entry point (allocates its workspace)
    assert first.shape == ref.shape and np.array_equal(first, ref)
    G.close()


@pytest.mark.parametrize("layout", ["int32", "int64", "cdf_cache"])
@pytest.mark.parametrize("bias,fan", [(0, [10, 5, 3]), (1, [20, 20, 20]), (2, [8, 4]), (3, [6, 6])])
def test_noalloc_matches_regular_entry_twice(setup, layout, bias, fan):
    csaw, torch, g = setup
    G = csaw.Graph(g, rowptr64=(layout == "int64"), cdf_cache=True if layout == "cdf_cache" else None)
    n, F = 300, 2
    seeds = G.make_seeds(n * F, 17 + bias)
    p = _params(csaw, bias, fan)
    ref = canon(*G.sample(p, seeds))   # with cdf_cache, this builds the cached prefix first
    out = torch.empty((4, csaw.edge_bound(p)), dtype=torch.int32, device="cuda")
    for _ in range(2):
        got = canon(*G.sample_noalloc(p, seeds, out))
        assert got.shape == ref.shape and np.array_equal(got, ref)
    G.close()


def test_noalloc_rejects_jobs_beyond_its_scratch(setup):
    csaw, torch, g = setup
    G = csaw.Graph(g)
    p = csaw.make_params(0, 0, 20000, 4, 32, 3, [32, 32, 32], seed=1)   # largest level 81.9 M items
    seeds = torch.zeros(20000 * 4, dtype=torch.int32, device="cuda")
    out = torch.empty((2, 16), dtype=torch.int32, device="cuda")
    with pytest.raises(csaw.CsawError) as ei:
        G.sample_noalloc(p, seeds, out, with_sample=False, with_depth=False)
    assert ei.value.code == 1 and b"32 MiB" in csaw.lib().csaw_last_error()
    G.close()
