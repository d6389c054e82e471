"""GPU tests of the request loop (csaw_server_*): every request's result in a
concurrent mix equals the same request run alone (and the oracle), under a
device budget small enough that admission has to wait for memory."""
import threading

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


def mixed_requests(csaw, g, n, seed):
    """Mix of 2-hop [25,10] and 3-hop [15,10,5] edge-weight-biased neighbor
    sampling and edge-weight-biased walks of length 10..80; 8..300 seeds."""
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        kind = i % 3
        k = int(rng.integers(8, 300))
        seeds = oracle.make_seeds(g.rowptr, k, 1000 + i)
        sched = int(rng.integers(0, 2))
        if kind == 0:
            p = csaw.make_params(0, 2, k, 1, 25, 2, [25, 10], seed=77 + i, schedule=sched)
        elif kind == 1:
            p = csaw.make_params(0, 2, k, 1, 15, 3, [15, 10, 5], seed=77 + i, schedule=sched)
        else:
            p = csaw.make_params(1, 2, k, 1, 1, int(rng.integers(10, 81)), seed=77 + i, schedule=sched)
        reqs.append((p, seeds))
    return reqs


def alone(csaw, G, p, seeds):
    import torch
    out = G.sample(p, torch.from_numpy(seeds).cuda())
    return sort_edges(*[x.cpu().numpy() for x in out])


def test_mix_equals_alone(csaw, rmat12_pareto):
    g = rmat12_pareto
    G = csaw.Graph(g)
    reqs = mixed_requests(csaw, g, 60, 1)
    expect = [alone(csaw, G, p, s) for p, s in reqs]
    # budget for a few requests at a time: admission waits for memory
    S = csaw.Server(G, n_slots=6, device_budget=24 << 20)
    tickets = [S.submit(p, s) for p, s in reqs]
    for t, e in zip(tickets, expect):
        n, lat, res = S.wait(t)
        assert lat > 0
        assert np.array_equal(sort_edges(*res), e)
    st = S.stats()
    assert st["completed"] == 60 and st["failed"] == 0
    assert 0 < st["peak_device_bytes"] <= 24 << 20
    assert st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    S.close()
    G.close()


def test_server_matches_oracle(csaw, powerlaw_small):
    g = powerlaw_small
    G = csaw.Graph(g)
    S = csaw.Server(G, n_slots=4)
    seeds = oracle.make_seeds(g.rowptr, 200, 5)
    cases = [(0, 1, [20, 20, 20]), (0, 2, [25, 10]), (1, 1, None), (1, 0, None)]
    tickets = []
    for mode, bias, fan in cases:
        if mode == 0:
            p = csaw.make_params(0, bias, 200, 1, fan[0], len(fan), fan, seed=9, schedule=1)
        else:
            p = csaw.make_params(1, bias, 200, 1, 1, 30, seed=9, schedule=1)
        tickets.append((S.submit(p, seeds), mode, bias, fan))
    for t, mode, bias, fan in tickets:
        n, _, res = S.wait(t)
        depth = len(fan) if fan else 30
        b = oracle.run(g.rowptr, g.col, g.weight, seeds, mode, bias, 200, 1, depth, fan or [1] * 30, seed=9,
                       n_threads=8)
        assert np.array_equal(sort_edges(*res), sort_edges(*b))
    S.close()
    G.close()


def test_pinned_and_pageable_outputs_agree(csaw, powerlaw_small):
    import torch
    g = powerlaw_small
    G = csaw.Graph(g)
    S = csaw.Server(G, n_slots=2)
    seeds = oracle.make_seeds(g.rowptr, 300, 8)
    p = csaw.make_params(0, 2, 300, 1, 25, 2, [25, 10], seed=4, schedule=1)
    cap = csaw.edge_bound(p)
    pinned = torch.empty((4, cap), dtype=torch.int32).pin_memory()
    t1 = S.submit(p, seeds, out=pinned)
    t2 = S.submit(p, seeds)
    n1, _, r1 = S.wait(t1)
    n2, _, r2 = S.wait(t2)
    assert n1 == n2 > 0
    a = sort_edges(*[x.numpy() for x in r1])
    assert np.array_equal(a, sort_edges(*r2))
    S.close()
    G.close()


def test_errors(csaw, powerlaw_small):
    g = powerlaw_small
    G = csaw.Graph(g)
    S = csaw.Server(G, n_slots=2, device_budget=1 << 20)
    seeds = oracle.make_seeds(g.rowptr, 4000, 8)
    big = csaw.make_params(0, 1, 4000, 1, 20, 3, seed=1, schedule=1)   # bound 33.6M edges: above the budget
    with pytest.raises(csaw.CsawError) as e:
        S.submit(big, seeds)
    assert e.value.code == 3
    small = csaw.make_params(0, 1, 100, 1, 20, 2, seed=1, schedule=1)
    t = S.submit(small, seeds[:100], capacity=10)                       # host capacity too small
    with pytest.raises(csaw.CsawError) as e:
        S.wait(t)
    assert e.value.code == 3
    bad = seeds[:100].copy()
    bad[7] = g.n_vertices + 5
    t = S.submit(small, bad)
    with pytest.raises(csaw.CsawError) as e:
        S.wait(t)
    assert e.value.code == 1
    ok = S.submit(small, seeds[:100])                                   # the server keeps serving
    assert S.wait(ok)[0] > 0
    with pytest.raises(csaw.CsawError):
        S.wait(ok)                                                      # a reported ticket is released
    st = S.stats()
    assert st["failed"] == 2 and st["completed"] == 1
    S.close()
    G.close()


def test_concurrent_submitters(csaw, rmat12_pareto):
    g = rmat12_pareto
    G = csaw.Graph(g)
    reqs = mixed_requests(csaw, g, 40, 2)
    expect = [alone(csaw, G, p, s) for p, s in reqs]
    S = csaw.Server(G, n_slots=8, device_budget=64 << 20)
    got = [None] * len(reqs)

    def client(idx):
        for i in idx:
            p, s = reqs[i]
            t = S.submit(p, s)
            got[i] = sort_edges(*S.wait(t)[2])

    th = [threading.Thread(target=client, args=(range(k, len(reqs), 4),)) for k in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for a, e in zip(got, expect):
        assert np.array_equal(a, e)
    assert S.stats()["completed"] == len(reqs)
    S.close()
    G.close()
