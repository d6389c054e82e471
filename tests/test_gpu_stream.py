"""Streaming (partitioned) sampling: adjacency in page-locked host memory,
paged into a few device slots; the output must equal the in-memory path and
the oracle exactly, whatever the partition order and evictions."""
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


def _same(a, b):
    sa, sb = sort_edges(*a), sort_edges(*b)
    assert sa.shape == sb.shape and np.array_equal(sa, sb)


@pytest.mark.parametrize("rip", [0, 1])
@pytest.mark.parametrize("bias", [0, 1, 2, 3])
@pytest.mark.parametrize("pbits,slots", [(8, 2), (6, 3), (10, 100)])
def test_stream_neighbor_equals_in_memory(csaw, rmat12_pareto, bias, pbits, slots, rip):
    """rip 0: partitions copied in and evicted by sweeps; rip 1: partitions
    outside the arena read in place from page-locked host memory."""
    import torch
    from csaw import _lib
    g = rmat12_pareto
    per_slot = int(np.max(g.rowptr[np.minimum(np.arange(0, g.n_vertices + (1 << pbits), 1 << pbits), g.n_vertices)][1:]
                          - g.rowptr[np.minimum(np.arange(0, g.n_vertices + (1 << pbits), 1 << pbits), g.n_vertices)][:-1]))
    budget = slots * per_slot * 8
    sg = csaw.StreamGraph(g, partition_bits=pbits, slot_budget_bytes=budget)
    sg.set_option(_lib.STREAM_OPT_READ_IN_PLACE, rip)
    G = csaw.Graph(g)
    seeds = oracle.make_seeds(g.rowptr, 200 * 2, 3 + bias)
    p = csaw.make_params(0, bias, 200, 2, 10, 3, [10, 5, 3], seed=41 + bias)
    a = [x.cpu().numpy() for x in sg.sample(p, torch.from_numpy(seeds).cuda())]
    b = [x.cpu().numpy() for x in G.sample(p, torch.from_numpy(seeds).cuda())]
    _same(a, b)
    info = sg.info()
    assert info["n_slots"] == min(slots, info["n_partitions"])
    if info["n_slots"] < info["n_partitions"] and not rip:
        assert info["partition_loads"] > info["n_slots"]     # evictions and reloads happened
    if info["n_slots"] < info["n_partitions"] and rip:
        assert info["items_read_in_place"] > 0                # the arena holds only some partitions
    if not rip:
        assert info["items_read_in_place"] == 0
    assert info["bytes_h2d"] > 0 and info["host_pinned_in_place"] & 1
    if bias in (0, 1, 2):
        _same(a, oracle.run(g.rowptr, g.col, g.weight, seeds, 0, bias, 200, 2, 3, [10, 5, 3], seed=41 + bias,
                            n_threads=8))


@pytest.mark.parametrize("rip", [0, 1])
@pytest.mark.parametrize("bias", [0, 1, 2])
def test_stream_walk_equals_in_memory(csaw, powerlaw_small, bias, rip):
    import torch
    from csaw import _lib
    g = powerlaw_small
    sg = csaw.StreamGraph(g, partition_bits=11, slot_budget_bytes=4 * 8 * int(np.diff(g.rowptr[::2048]).max() + 2048))
    sg.set_option(_lib.STREAM_OPT_READ_IN_PLACE, rip)
    seeds = oracle.make_seeds(g.rowptr, 300, 6)
    p = csaw.make_params(1, bias, 300, 1, 1, 40, None, seed=9)
    a = [x.cpu().numpy() for x in sg.sample(p, torch.from_numpy(seeds).cuda())]
    b = oracle.run(g.rowptr, g.col, g.weight, seeds, 1, bias, 300, 1, 40, seed=9, n_threads=8)
    _same(a, b)


def test_stream_rejects_mdrw_and_tiny_budget(csaw, powerlaw_small):
    import torch
    g = powerlaw_small
    with pytest.raises(csaw.CsawError):
        csaw.StreamGraph(g, partition_bits=11, slot_budget_bytes=16)
    sg = csaw.StreamGraph(g, partition_bits=11, slot_budget_bytes=1 << 26)
    p = csaw.make_params(2, 1, 10, 4, 1, 5, None, seed=1)
    with pytest.raises(csaw.CsawError):
        sg.sample(p, torch.zeros(40, dtype=torch.int32, device="cuda"))


@pytest.mark.parametrize("rip", [0, 1])
def test_stream_weights_added_to_resident_partitions(csaw, powerlaw_small, rip):
    """A degree-biased job leaves partitions resident without their weights;
    an edge-weight job on the same streaming graph must still see them."""
    import torch
    from csaw import _lib
    g = powerlaw_small
    sg = csaw.StreamGraph(g, partition_bits=11, slot_budget_bytes=64 << 20)
    sg.set_option(_lib.STREAM_OPT_READ_IN_PLACE, rip)
    seeds = oracle.make_seeds(g.rowptr, 300, 7)
    sd = torch.from_numpy(seeds).cuda()
    for bias in (1, 2, 1, 2):
        p = csaw.make_params(0, bias, 300, 1, 10, 2, [10, 5], seed=3)
        a = [x.cpu().numpy() for x in sg.sample(p, sd)]
        b = oracle.run(g.rowptr, g.col, g.weight, seeds, 0, bias, 300, 1, 2, [10, 5], seed=3, n_threads=8)
        _same(a, b)


@pytest.mark.parametrize("rip", [0, 1])
@pytest.mark.parametrize("rowptr64", [False, True])
@pytest.mark.parametrize("bias", [1, 2, 3])
def test_stream_prefix_cache_equals_oracle(csaw, rmat12_pareto, rowptr64, bias, rip):
    """With the streaming prefix cache (csaw_stream_graph_cache) each
    partition's canonical prefix is streamed instead of its weights and
    searched: the edges stay the in-memory run's (and the oracle's), for
    neighbor sampling with rebuilds and for walks, through a budget of a few
    partitions."""
    import torch
    g = rmat12_pareto
    pbits = 8
    edges = np.diff(g.rowptr[np.minimum(np.arange(0, g.n_vertices + (1 << pbits), 1 << pbits), g.n_vertices)])
    sg = csaw.StreamGraph(g, partition_bits=pbits, slot_budget_bytes=3 * int(edges.max()) * 8, rowptr64=rowptr64)
    from csaw import _lib
    sg.set_option(_lib.STREAM_OPT_READ_IN_PLACE, rip)
    sg.cache(bias)
    G = csaw.Graph(g, rowptr64=rowptr64)
    deg = np.diff(g.rowptr)
    hubs = np.argsort(deg)[-8:].astype(np.int32)
    seeds = np.concatenate([hubs, oracle.make_seeds(g.rowptr, 2 * 200 - 8, 31 + bias)]).astype(np.int32)
    for mode, fan, depth, n, F in ((0, [12, 6, 3], 3, 200, 2), (0, [30, 4], 2, 200, 2), (1, None, 30, 400, 1)):
        sd = seeds[:n * F]
        p = csaw.make_params(mode, bias, n, F, (fan or [1])[0], depth, fan, seed=0x51 + bias)
        a = [x.cpu().numpy() for x in sg.sample(p, torch.from_numpy(sd).cuda())]
        b = [x.cpu().numpy() for x in G.sample(p, torch.from_numpy(sd).cuda())]
        _same(a, b)
        if bias in (1, 2):
            _same(a, oracle.run(g.rowptr, g.col, g.weight, sd, mode, bias, n, F, depth, fan, seed=0x51 + bias,
                                n_threads=8))
    info = sg.info()
    assert info["bytes_h2d"] > 0
    if rip:
        assert info["items_read_in_place"] > 0
    else:
        assert info["partition_loads"] > info["n_slots"]
    sg.close()


@pytest.mark.parametrize("rip", [0, 1])
def test_stream_cached_and_uncached_biases_mix(csaw, rmat12_pareto, rip):
    """A streaming graph with a weight-bias prefix cache runs degree-biased
    (uncached: weights not needed), weight-biased (cached) and unbiased jobs
    in turn; resident partitions are reloaded with the array each job needs
    (or read in place)."""
    import torch
    from csaw import _lib
    g = rmat12_pareto
    sg = csaw.StreamGraph(g, partition_bits=9, slot_budget_bytes=1 << 20)
    sg.set_option(_lib.STREAM_OPT_READ_IN_PLACE, rip)
    sg.cache(2)
    seeds = oracle.make_seeds(g.rowptr, 300, 5)
    sd = torch.from_numpy(seeds).cuda()
    for bias in (2, 1, 0, 2, 1):
        p = csaw.make_params(0, bias, 300, 1, 10, 2, [10, 5], seed=7 + bias)
        a = [x.cpu().numpy() for x in sg.sample(p, sd)]
        _same(a, oracle.run(g.rowptr, g.col, g.weight, seeds, 0, bias, 300, 1, 2, [10, 5], seed=7 + bias,
                            n_threads=8))
    sg.close()
