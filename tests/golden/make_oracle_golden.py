"""Generate tests/golden/oracle_edges.npz: canonical (sorted) edge lists of the
oracle on small fixed cases.  They pin the sampling semantics against
accidental change; the GPU parity tests compare against the oracle itself.

Run:  python tests/golden/make_oracle_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for sub in ("c-saw_b200", "oracle", "tests"):
    sys.path.insert(0, os.path.join(ROOT, sub))

import oracle  # noqa: E402
from csaw import graphgen  # noqa: E402

CASES = {
    # name: (graph, mode, bias, n_samples, F, depth, fanout, seed[, {flags, sample_base}])
    "rmat10_unbiased_n2d2": ("rmat10", 0, 0, 200, 1, 2, [2, 2], 0),
    "rmat10_weight_n5d3": ("rmat10", 0, 2, 100, 1, 3, [5, 3, 2], 7),
    "rmat10_degree_f4": ("rmat10", 0, 1, 50, 4, 2, [6, 3], 11),
    "pl_degree_walk": ("pl", 1, 1, 100, 1, 20, None, 3),
    "pl_weight_walk": ("pl", 1, 2, 100, 1, 20, None, 4),
    "pl_unbiased_walk": ("pl", 1, 0, 100, 1, 20, None, 5),
    "pl_mdrw_degree": ("pl", 2, 1, 40, 6, 25, None, 6),
    "pl_weight_tight": ("pl", 0, 2, 60, 1, 2, [12, 12], 8),
    # per-sample vertex dedup (few distinct seeds, so repeats are common)
    "rmat10_weight_dedup": ("rmat10", 0, 2, 80, 2, 3, [6, 4, 3], 9, {"flags": oracle.DEDUP}),
    "rmat10_degree_dedup_f3": ("rmat10", 0, 1, 60, 3, 2, [8, 5], 10, {"flags": oracle.DEDUP}),
    # a shard of a larger job: sample ids (and every draw) start at sample_base
    "pl_weight_base": ("pl", 0, 2, 50, 2, 2, [7, 4], 12, {"sample_base": 123456}),
    "pl_walk_base": ("pl", 1, 2, 64, 1, 16, None, 13, {"sample_base": 1 << 20}),
}


def graph(name):
    if name == "rmat10":
        return graphgen.rmat(10, 8, seed=1, weight="pareto:1.5")
    return graphgen.powerlaw_directed(n_vertices=3000, n_edges=18000, gamma=2.1, max_degree=200, seed=2,
                                      weight="lognormal")


def build_case(name):
    gname, mode, bias, n, F, depth, fan, seed, *rest = CASES[name]
    extra = rest[0] if rest else {}
    g = graph(gname)
    per = 1 if mode == 1 else F
    seeds = oracle.make_seeds(g.rowptr, n * per, seed + 1000)
    if extra.get("flags"):   # few distinct seeds
        seeds = seeds[np.arange(seeds.size) % 7]
    src, dst, smp, dep = oracle.run(g.rowptr, g.col, g.weight, seeds, mode, bias, n, F, depth, fan, seed=seed,
                                    flags=extra.get("flags", 0), sample_base=extra.get("sample_base", 0))
    src, dst, smp, dep = (np.asarray(x, dtype=np.int64) for x in (src, dst, smp, dep))
    o = np.lexsort((dst, src, dep, smp))
    return np.stack([smp[o], dep[o], src[o], dst[o]]).astype(np.int32)


def main():
    out = {name: build_case(name) for name in CASES}
    path = os.path.join(HERE, "oracle_edges.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, {k: v.shape[1] for k, v in out.items()})


if __name__ == "__main__":
    main()
