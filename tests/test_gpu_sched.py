"""Learned granularity scheduler: the MLP's GPU gradient against a float64
NumPy backward, training reduces the loss, and the learned schedule (while
recording, and with the trained model) never changes the output."""
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


def np_loss_grad(w, norm, rec):
    """Reference forward/backward in float64 (same layout and loss)."""
    w = w.astype(np.float64)
    W1 = w[0:256].reshape(32, 8); b1 = w[256:288]
    W2 = w[288:1312].reshape(32, 32); b2 = w[1312:1344]
    W3 = w[1344:1568].reshape(7, 32); b3 = w[1568:1575]
    x = (rec["x"].astype(np.float64) - norm[:8]) / norm[8:16]
    a1 = x @ W1.T + b1; h1 = np.maximum(a1, 0)
    a2 = h1 @ W2.T + b2; h2 = np.maximum(a2, 0)
    y = h2 @ W3.T + b3
    c = rec["cls"]
    t = (np.log2(np.maximum(rec["cycles"], 1.0)) - norm[16]) / norm[17]
    n = len(rec)
    e = y[np.arange(n), c] - t
    dy = np.zeros_like(y); dy[np.arange(n), c] = e
    gW3 = dy.T @ h2; gb3 = dy.sum(0)
    dh2 = (dy @ W3) * (a2 > 0)
    gW2 = dh2.T @ h1; gb2 = dh2.sum(0)
    dh1 = (dh2 @ W2) * (a1 > 0)
    gW1 = dh1.T @ x; gb1 = dh1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3]) / n
    return 0.5 * np.mean(e * e), g


def test_mlp_gradient_matches_numpy(csaw):
    from csaw.sampler import PROF_DTYPE, mlp_grad
    rng = np.random.default_rng(0)
    w = (rng.standard_normal(1575) * 0.3).astype(np.float32)
    norm = np.concatenate([rng.standard_normal(8), 0.5 + rng.random(8), [10.0, 2.0]]).astype(np.float32)
    rec = np.zeros(777, dtype=PROF_DTYPE)
    rec["x"] = rng.standard_normal((777, 8)) * 2
    rec["cls"] = rng.integers(0, 7, 777)
    rec["cycles"] = 2.0 ** rng.uniform(8, 14, 777)
    loss, g = mlp_grad(w, norm, rec)
    rl, rg = np_loss_grad(w, norm, rec)
    assert abs(loss - rl) <= 1e-4 * max(1.0, abs(rl))
    np.testing.assert_allclose(g, rg, rtol=2e-3, atol=2e-5 * np.abs(rg).max())


@pytest.mark.parametrize("bias", [1, 2])
def test_learned_schedule_keeps_output_and_trains(csaw, rmat12_pareto, bias):
    import torch
    g = rmat12_pareto
    deg = np.diff(g.rowptr)
    hubs = np.argsort(deg)[-16:].astype(np.int32)
    seeds = np.concatenate([hubs, oracle.make_seeds(g.rowptr, 2 * 300 - 16, 4)]).astype(np.int32)
    ref = oracle.run(g.rowptr, g.col, g.weight, seeds, 0, bias, 300, 2, 3, [12, 6, 3], seed=23, n_threads=8)
    G = csaw.Graph(g)
    p = csaw.make_params(0, bias, 300, 2, 12, 3, [12, 6, 3], seed=23, schedule=csaw.SCHED_LEARNED)
    sd = torch.from_numpy(seeds).cuda()

    def run():
        out = [x.cpu().numpy() for x in G.sample(p, sd)]
        assert np.array_equal(sort_edges(*out), sort_edges(*ref))

    run()                                  # untrained: degree rule
    G.sched_record(200_000)
    for _ in range(3):
        run()                              # recording: random granularities
    info = G.sched_info()
    assert info["records"] > 300
    rec = G.sched_records()
    assert set(np.unique(rec["cls"])) >= {1, 2, 3, 4, 5}      # every granularity was explored
    loss = G.sched_train(epochs=400, lr=3e-3, seed=1)
    w, nrm = G.sched_model()
    assert np.isfinite(loss) and G.sched_info()["trained"]
    # the trained network explains a large part of the variance of the
    # recorded latencies (a zero network predicts the mean: loss ~ variance)
    zero_loss, _ = np_loss_grad(np.zeros_like(w), nrm.astype(np.float64), rec)
    assert loss < 0.7 * zero_loss
    ref_loss, _ = np_loss_grad(w, nrm.astype(np.float64), rec)
    assert abs(ref_loss - loss) < 1e-3 * max(1.0, loss)
    mask = G.sched_info()["class_mask"]
    assert mask & 0x3 == 0x3                   # the warp classes are always kept
    for _ in range(8):
        run()                              # trained (and timed against the degree rule): same edges
    # after the trial the model is kept, or dropped for the degree rule
    assert G.sched_info()["class_mask"] in (mask, 0x3)
