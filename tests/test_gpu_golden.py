"""GPU parity against the committed golden fixtures: every case of
tests/golden/oracle_edges.npz (oracle edge lists in canonical order: all
three modes and bias kinds, per-sample dedup, shards with a sample base) run
through the C ABI under the plain and batched schedules gives exactly the
fixture."""
import os

import numpy as np
import pytest

from conftest import sort_edges

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def csaw():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test without a CUDA device")
    import csaw as c
    c.lib()
    return c


def case_inputs(csaw, case, schedule):
    """(graph name, params, seeds) of a golden case, as its generator made them."""
    import oracle
    from make_oracle_golden import graph
    gname, mode, bias, n, F, depth, fan, seed, *rest = case
    extra = rest[0] if rest else {}
    g = graph(gname)
    seeds = oracle.make_seeds(g.rowptr, n * (1 if mode == 1 else F), seed + 1000)
    if extra.get("flags"):   # few distinct seeds, as generated
        seeds = seeds[np.arange(seeds.size) % 7]
    p = csaw.make_params(mode, bias, n, F, (fan or [1])[0], depth, fan, seed, schedule=schedule,
                         sample_base=extra.get("sample_base", 0), dedup=bool(extra.get("flags")))
    return gname, g, p, np.ascontiguousarray(seeds, dtype=np.int32)


@pytest.mark.parametrize("schedule", [0, 1])
def test_golden_cases_on_gpu(csaw, schedule):
    import torch
    from make_oracle_golden import CASES
    data = np.load(os.path.join(GOLDEN, "oracle_edges.npz"))
    graphs = {}
    try:
        for name, case in CASES.items():
            gname, g, p, seeds = case_inputs(csaw, case, schedule)
            if gname not in graphs:
                graphs[gname] = csaw.Graph(g)
            out = [x.cpu().numpy() for x in graphs[gname].sample(p, torch.from_numpy(seeds).cuda())]
            assert np.array_equal(sort_edges(*out), data[name].astype(np.int64)), name
    finally:
        for G in graphs.values():
            G.close()
