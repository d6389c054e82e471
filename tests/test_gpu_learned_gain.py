"""What the trained granularity scheduler gains over the degree rule, measured
on the device: R-MAT (a=.6, b=.2, c=.15) scale 20, edge factor 16, Pareto(1.5)
weights, without the per-vertex prefix cache (hubs then need CTA-width prefix
scans, where the width choice matters), 8192 edge-weight-biased samples F8
N10 D3.  The model is trained on the GPU on profiles recorded on three
steps, must survive its own timed trial, and must then run the step faster
than the degree rule by more than run-to-run noise, with the same edges."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_trained_scheduler_beats_degree_rule():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test without a CUDA device")
    import csaw
    from csaw import graphgen
    g = graphgen.rmat_device(scale=20, edge_factor=16, a=0.6, b=0.2, c=0.15, seed=25, symmetrize=False,
                             weight="pareto:1.5")
    G = csaw.Graph(g, cdf_cache=False)
    seeds = G.make_seeds(8192 * 8, 0x25)
    out = torch.empty((3, 8192 * 8 * (10 + 100 + 1000)), dtype=torch.int32, device="cuda")

    def job(schedule):
        p = csaw.make_params(0, 2, 8192, 8, 10, 3, seed=0x25, schedule=schedule)
        return [csaw.BatchJob(p, seeds, out.shape[1], out, with_depth=False)]

    rule, learned = job(csaw.SCHED_BATCHED), job(csaw.SCHED_LEARNED)

    def edges(res):
        r = res[0]
        key = (r[2].to(torch.int64) << 42) | (r[0].to(torch.int64) << 21) | r[1].to(torch.int64)
        return torch.sort(key).values.cpu().numpy()

    ref = edges(G.sample_batch(rule))
    G.sched_record(400_000)
    for _ in range(3):
        G.sample_batch(learned)
    G.sched_train(epochs=400, lr=3e-3, seed=1)
    for _ in range(6):   # the model's own timed trial against the degree rule
        G.sample_batch(learned)
    info = G.sched_info()
    assert info["class_mask"] != 0x3, "the trained model lost its trial against the degree rule"
    assert np.array_equal(edges(G.sample_batch(learned)), ref)

    def timed(jobs):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        G.sample_batch(jobs)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    for _ in range(2):
        timed(rule)
        timed(learned)
    t_rule, t_learned = [], []
    for _ in range(9):   # interleaved, so clock or thermal drift hits both alike
        t_rule.append(timed(rule))
        t_learned.append(timed(learned))
    m_rule, m_learned = float(np.median(t_rule)), float(np.median(t_learned))
    spread = float(np.percentile(t_rule, 75) - np.percentile(t_rule, 25)) / m_rule
    print(f"degree rule {m_rule:.2f} ms, learned {m_learned:.2f} ms, gain {m_rule / m_learned:.3f}, "
          f"rule IQR {spread:.3f}")
    assert m_learned < m_rule * (1.0 - max(0.03, 2 * spread)), (m_rule, m_learned, spread)
    G.close()
