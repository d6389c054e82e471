"""CPU tests of the oracle: Philox pinned to cuRAND's host generator, the
canonical prefix and the full sampling semantics cross-checked against an
independent pure-Python restatement, committed golden edge lists, and
distributional checks against the ideal normalised bias."""
import os

import numpy as np
import pytest
from scipy import stats

import oracle
import pyspec
from conftest import sort_edges

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_philox_matches_curand_host_generator():
    cases = np.load(os.path.join(GOLDEN, "philox_curand.npz"))["cases"]
    assert len(cases) >= 30
    for row in cases:
        assert np.array_equal(oracle.philox(row[:4], row[4:6]), row[6:10])


def test_philox_python_restatement_agrees():
    rng = np.random.default_rng(1)
    for _ in range(200):
        ctr = rng.integers(0, 2**32, 4, dtype=np.uint64)
        key = rng.integers(0, 2**32, 2, dtype=np.uint64)
        assert list(oracle.philox(ctr, key)) == pyspec.philox(ctr, key)


@pytest.mark.parametrize("d", [1, 2, 31, 32, 33, 100, 1023, 1024, 1025, 3000, 40000])
def test_canonical_prefix_matches_python(d):
    rng = np.random.default_rng(d)
    w = rng.lognormal(0, 2, d).astype(np.float32)
    w[rng.random(d) < 0.1] = 0.0
    P = oracle.canon_prefix(w)
    if d <= 3000:
        assert np.array_equal(P, np.array(pyspec.canon_prefix(list(w)), dtype=np.float32))
    assert np.all(np.diff(P) >= 0)
    ref = np.cumsum(w.astype(np.float64))
    np.testing.assert_allclose(P, ref, rtol=2e-5 * max(1.0, np.log2(d)), atol=1e-30)


def test_canonical_prefix_exact_on_integer_biases():
    rng = np.random.default_rng(7)
    w = rng.integers(0, 460, 5000).astype(np.float32)
    P = oracle.canon_prefix(w)
    assert np.array_equal(P.astype(np.int64), np.cumsum(w.astype(np.int64)))


def _graph_small(seed, V=300, avgdeg=12, weight=True):
    from csaw import graphgen
    rng = np.random.default_rng(seed)
    deg = np.minimum(rng.zipf(1.8, V), V - 1)
    deg[rng.random(V) < 0.05] = 0
    src = np.repeat(np.arange(V), deg)
    dst = np.concatenate([rng.choice(V, size=d, replace=False) for d in deg]) if deg.sum() else np.zeros(0, int)
    keep = src != dst
    rp, col = graphgen._csr_from_edges(src[keep], dst[keep], V)
    w = rng.lognormal(0, 1.5, col.size).astype(np.float32) if weight else None
    if w is not None:
        w[rng.random(col.size) < 0.05] = 0.0
    return graphgen.CSR(rp, col, w)


CASES = [
    # mode, bias, n, F, depth, fanout
    (0, 0, 12, 1, 3, [2, 3, 2]),
    (0, 1, 10, 2, 2, [5, 4]),
    (0, 2, 10, 2, 2, [8, 3]),
    (0, 2, 6, 1, 2, [30, 2]),
    (1, 0, 20, 1, 15, None),
    (1, 1, 20, 1, 15, None),
    (1, 2, 20, 1, 15, None),
    (2, 0, 10, 5, 12, None),
    (2, 1, 10, 5, 12, None),
]


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_python_restatement(case):
    mode, bias, n, F, depth, fan = case
    g = _graph_small(11 + mode * 3 + bias)
    nz = np.flatnonzero(np.diff(g.rowptr) > 0)
    rng = np.random.default_rng(5)
    per = 1 if mode == 1 else F
    seeds = rng.choice(nz, n * per).astype(np.int32)
    seed = 0xABCDEF0123 + mode
    a = oracle.run(g.rowptr, g.col, g.weight, seeds, mode, bias, n, F, depth, fan, seed=seed)
    b = pyspec.run(g, seeds, mode, bias, n, F, depth, fan, seed)
    assert np.array_equal(sort_edges(*a), sort_edges(*b))


def test_oracle_threads_do_not_change_output(rmat16):
    g = rmat16
    seeds = oracle.make_seeds(g.rowptr, 300, 9)
    a = oracle.run(g.rowptr, g.col, g.weight, seeds, 0, 2, 300, 1, 3, [5, 4, 3], seed=4, n_threads=1)
    b = oracle.run(g.rowptr, g.col, g.weight, seeds, 0, 2, 300, 1, 3, [5, 4, 3], seed=4, n_threads=7)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_walk_is_neighbor_sampling_with_one_neighbor(powerlaw_small):
    g = powerlaw_small
    seeds = oracle.make_seeds(g.rowptr, 200, 3)
    for bias in (0, 1, 2):
        w = oracle.run(g.rowptr, g.col, g.weight, seeds, 1, bias, 200, 1, 30, seed=8)
        s = oracle.run(g.rowptr, g.col, g.weight, seeds, 0, bias, 200, 1, 30, [1] * 30, seed=8)
        assert np.array_equal(sort_edges(*w), sort_edges(*s))


def test_selection_properties(rmat12_pareto):
    g = rmat12_pareto
    seeds = oracle.make_seeds(g.rowptr, 400, 1)
    src, dst, smp, dep = oracle.run(g.rowptr, g.col, g.weight, seeds, 0, 2, 400, 1, 2, [10, 4], seed=2)
    deg = np.diff(g.rowptr)
    # every edge exists in the graph
    for u, v in zip(src[:2000], dst[:2000]):
        assert v in g.col[g.rowptr[u]:g.rowptr[u + 1]]
    # depth 0: each seed expansion selects min(N, d) distinct neighbors
    for s in range(400):
        m = (smp == s) & (dep == 0)
        assert m.sum() == min(10, deg[seeds[s]])
        assert len(set(dst[m].tolist())) == m.sum()


def test_make_seeds_uniform_over_nonisolated(rmat16):
    g = rmat16
    s = oracle.make_seeds(g.rowptr, 20000, 0)
    deg = np.diff(g.rowptr)
    assert np.all(deg[s] > 0)
    nz = np.flatnonzero(deg > 0)
    counts = np.bincount(np.searchsorted(nz, s) * 16 // nz.size, minlength=16)
    assert stats.chisquare(counts).pvalue > 1e-4


def _first_slot_frequencies(g, v, bias, trials, N=1):
    seeds = np.full(trials, v, dtype=np.int32)
    src, dst, smp, dep = oracle.run(g.rowptr, g.col, g.weight, seeds, 0, bias, trials, 1, 1, [N], seed=12,
                                    n_threads=4)
    beg, end = g.rowptr[v], g.rowptr[v + 1]
    pos = {int(u): i for i, u in enumerate(g.col[beg:end])}
    return np.bincount([pos[int(u)] for u in dst], minlength=end - beg)


@pytest.mark.parametrize("bias", [0, 1, 2])
def test_distribution_matches_normalised_bias(rmat12_pareto, bias):
    g = rmat12_pareto
    deg = np.diff(g.rowptr)
    v = int(np.flatnonzero((deg > 40) & (deg < 80))[0])
    beg, end = g.rowptr[v], g.rowptr[v + 1]
    if bias == 0:
        p = np.ones(end - beg)
    elif bias == 1:
        p = deg[g.col[beg:end]].astype(np.float64)
    else:
        p = g.weight[beg:end].astype(np.float64)
    p /= p.sum()
    trials = 40000
    obs = _first_slot_frequencies(g, v, bias, trials)
    exp = p * trials
    big = exp >= 5
    o = np.append(obs[big], obs[~big].sum())
    e = np.append(exp[big], exp[~big].sum())
    if e[-1] == 0:
        o, e = o[:-1], e[:-1]
    assert stats.chisquare(o, e * o.sum() / e.sum()).pvalue > 1e-4


def test_without_replacement_inclusion_probabilities(rmat12_pareto):
    """Successive sampling: P(item in sample) for k=3 of a skewed distribution
    matches the exact successive-sampling inclusion probabilities."""
    from itertools import permutations
    g = rmat12_pareto
    deg = np.diff(g.rowptr)
    v = int(np.flatnonzero(deg == 6)[0])
    beg = g.rowptr[v]
    w = g.weight[beg:beg + 6].astype(np.float64)
    incl = np.zeros(6)
    for perm in permutations(range(6), 3):
        pr, rem = 1.0, w.sum()
        for i in perm:
            pr *= w[i] / rem
            rem -= w[i]
        incl[list(perm)] += pr
    trials = 30000
    seeds = np.full(trials, v, dtype=np.int32)
    src, dst, smp, dep = oracle.run(g.rowptr, g.col, g.weight, seeds, 0, 2, trials, 1, 1, [3], seed=99,
                                    n_threads=4)
    pos = {int(u): i for i, u in enumerate(g.col[beg:beg + 6])}
    cnt = np.bincount([pos[int(u)] for u in dst], minlength=6)
    np.testing.assert_allclose(cnt / trials, incl, atol=0.015)


def test_golden_edge_lists():
    from make_oracle_golden import CASES as GCASES, build_case
    data = np.load(os.path.join(GOLDEN, "oracle_edges.npz"))
    for name in GCASES:
        got = build_case(name)
        assert np.array_equal(got, data[name]), name


@pytest.mark.parametrize("bias", [0, 1, 2])
@pytest.mark.parametrize("F,fan", [(1, [6, 5, 4]), (3, [3, 3, 3, 3]), (2, [8, 8])])
def test_dedup_matches_python_restatement(bias, F, fan):
    """Per-sample vertex dedup: the oracle equals the Python restatement, on a
    small dense graph where repeats are frequent (and seeds repeat too)."""
    g = _graph_small(41 + bias)
    nz = np.flatnonzero(np.diff(g.rowptr) > 0)
    rng = np.random.default_rng(8)
    n = 40
    seeds = rng.choice(nz[:12], n * F).astype(np.int32)   # few distinct seeds: repeats within a sample
    a = oracle.run(g.rowptr, g.col, g.weight, seeds, 0, bias, n, F, len(fan), fan, seed=77, flags=oracle.DEDUP)
    b = pyspec.run(g, seeds, 0, bias, n, F, len(fan), fan, 77, dedup=True)
    assert np.array_equal(sort_edges(*a), sort_edges(*b))
    full = oracle.run(g.rowptr, g.col, g.weight, seeds, 0, bias, n, F, len(fan), fan, seed=77)
    assert 0 < len(a[0]) <= len(full[0])
    if F > 1:
        assert len(a[0]) < len(full[0])             # repeated seeds are expanded once
    # depth-0 edges only lose repeated seeds; each sample expands a vertex at most once per level set
    for s in range(n):
        m = (a[2] == s)
        src_levels = {}
        for u, l in zip(a[0][m], a[3][m]):
            src_levels.setdefault(int(u), set()).add(int(l))
        assert all(len(ls) == 1 for ls in src_levels.values())
