"""Multi-rank placement on CPU (gloo, world size 2): shards of a job, keyed
by global sample ids, reproduce the single-rank output exactly; replicas
never share sample ids; the totals reduction sums edges and takes the max
time.  The oracle stands in for the GPU compute."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import sort_edges


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for sub in ("c-saw_b200", "oracle", "tests"):
        sys.path.insert(0, os.path.join(root, sub))
    import torch
    import torch.distributed as dist
    import oracle
    import csaw
    from csaw import dist as cdist, graphgen
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    g = graphgen.rmat(10, 8, seed=3, weight="uniform")
    seeds = oracle.make_seeds(g.rowptr, 101 * 2, 5)
    full = csaw.make_params(0, 2, 101, 2, 4, 3, [4, 3, 2], seed=77)
    p, sl = cdist.shard_params(full, rank, world)
    e = oracle.run(g.rowptr, g.col, g.weight, seeds[sl], 0, 2, p.n_samples, 2, 3, [4, 3, 2], seed=77,
                   sample_base=p.sample_base)
    mine = torch.from_numpy(sort_edges(*e))
    sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(sizes, torch.tensor([mine.shape[1]]))
    width = int(max(s.item() for s in sizes))
    padded = torch.full((4, width), -1, dtype=torch.int64)
    padded[:, :mine.shape[1]] = mine
    parts = [torch.zeros((4, width), dtype=torch.int64) for _ in sizes]
    dist.all_gather(parts, padded)
    parts = [x[:, :int(n.item())] for x, n in zip(parts, sizes)]
    tot_e, tot_t = cdist.reduce_totals(mine.shape[1], 1.0 + rank)
    r = cdist.replica_params(full, rank)
    ids = torch.tensor([r.sample_base, r.sample_base + r.n_samples])
    all_ids = [torch.zeros(2, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(all_ids, ids)
    if rank == 0:
        ref = sort_edges(*oracle.run(g.rowptr, g.col, g.weight, seeds, 0, 2, 101, 2, 3, [4, 3, 2], seed=77))
        union = np.concatenate([x.numpy() for x in parts], axis=1)
        o = np.lexsort(union[::-1])
        q.put((np.array_equal(union[:, o], ref), tot_e == ref.shape[1], tot_t == float(world),
               [x.tolist() for x in all_ids]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_shards_equal_single_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    import queue
    res = None
    for _ in range(120):
        try:
            res = q.get(timeout=1)
            break
        except queue.Empty:
            if any(p.exitcode not in (None, 0) for p in procs):
                break
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
        assert p.exitcode == 0
    assert res is not None
    same, edges_ok, time_ok, ids = res
    assert same and edges_ok and time_ok
    (a0, a1), (b0, b1) = ids
    assert a1 <= b0 or b1 <= a0       # replica sample ids do not overlap


def test_shard_range_covers_exactly():
    from csaw import dist as cdist
    for n in (0, 1, 7, 100):
        for w in (1, 2, 3, 8):
            r = [cdist.shard_range(n, k, w) for k in range(w)]
            assert r[0][0] == 0 and r[-1][1] == n
            assert all(r[k][1] == r[k + 1][0] for k in range(w - 1))
    with pytest.raises(ValueError):
        cdist.shard_range(5, 2, 2)
