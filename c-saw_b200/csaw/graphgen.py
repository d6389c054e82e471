"""Deterministic synthetic graph generators (CSR, int32 col, float32 weights).

The reference's example graph (web-Google, SNAP) is not shipped with it, so
the workloads use seeded synthetic graphs with the stated shapes:
  - R-MAT (Chakrabarti, Zhan, Faloutsos, SDM 2004) with (a, b, c, d), scale
    and edge factor, optionally symmetrised, self-loops and duplicate edges
    removed;
  - a directed graph with a power-law out-degree sequence (exponent gamma,
    capped at max_degree, summing exactly to n_edges) whose destinations follow
    a Zipf popularity, so in-degrees are skewed too.
Weights: uniform (0, 1], lognormal(0, 1) or Pareto(alpha) (numpy PCG64).
"""
import numpy as np


class CSR:
    """Host CSR: rowptr int64[V+1], col int32[E], weight float32[E] or None."""

    def __init__(self, rowptr, col, weight=None, name=""):
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.int64)
        self.col = np.ascontiguousarray(col, dtype=np.int32)
        self.weight = None if weight is None else np.ascontiguousarray(weight, dtype=np.float32)
        self.name = name

    @property
    def n_vertices(self):
        return self.rowptr.size - 1

    @property
    def n_edges(self):
        return self.col.size

    def degrees(self):
        return np.diff(self.rowptr)

    def rowptr32(self):
        if self.n_edges >= 2**31:
            raise ValueError("E >= 2^31 needs int64 rowptr")
        return self.rowptr.astype(np.int32)


def _csr_from_edges(src, dst, V):
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]
    counts = np.bincount(src, minlength=V).astype(np.int64)
    rowptr = np.zeros(V + 1, dtype=np.int64)
    np.cumsum(counts, out=rowptr[1:])
    return rowptr, dst.astype(np.int32)


def weights(kind, n, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    if kind == "uniform":
        return (1.0 - rng.random(n, dtype=np.float32)).astype(np.float32)  # (0, 1]
    if kind == "lognormal":
        return rng.lognormal(0.0, 1.0, n).astype(np.float32)
    if kind.startswith("pareto"):
        alpha = float(kind.split(":")[1]) if ":" in kind else 1.5
        return (1.0 + rng.pareto(alpha, n)).astype(np.float32)
    if kind == "none":
        return None
    raise ValueError(kind)


def rmat(scale, edge_factor, a=0.57, b=0.19, c=0.19, seed=0, symmetrize=True, weight="uniform",
         chunk=1 << 22):
    """R-MAT graph with 2^scale vertices and edge_factor * 2^scale generated edges."""
    V = 1 << scale
    E = edge_factor * V
    rng = np.random.Generator(np.random.PCG64(seed))
    ab, abc = a + b, a + b + c
    srcs, dsts = [], []
    for off in range(0, E, chunk):
        n = min(chunk, E - off)
        s = np.zeros(n, dtype=np.int64)
        d = np.zeros(n, dtype=np.int64)
        for bit in range(scale):
            r = rng.random(n, dtype=np.float32)
            sbit = r >= ab                      # quadrants c, d
            dbit = ((r >= a) & (r < ab)) | (r >= abc)  # quadrants b, d
            s |= sbit.astype(np.int64) << bit
            d |= dbit.astype(np.int64) << bit
        srcs.append(s)
        dsts.append(d)
    s = np.concatenate(srcs)
    d = np.concatenate(dsts)
    if symmetrize:
        s, d = np.concatenate([s, d]), np.concatenate([d, s])
    keep = s != d
    s, d = s[keep], d[keep]
    key = np.unique(s * V + d)
    s, d = key // V, key % V
    rowptr, col = _csr_from_edges(s, d, V)
    w = weights(weight, col.size, seed + 1)
    return CSR(rowptr, col, w, name=f"rmat{scale}_ef{edge_factor}")


def rmat_device(scale, edge_factor, a=0.57, b=0.19, c=0.19, seed=0, symmetrize=True, weight="uniform",
                device="cuda", chunk=1 << 26):
    """R-MAT as rmat() (same quadrant rule, self-loops and duplicates removed),
    generated with torch on a CUDA device, so scales 22-25 take seconds rather
    than minutes.  Draws come from a torch Philox generator seeded with `seed`:
    the same distribution as rmat(), not the same graph."""
    import torch
    V = 1 << scale
    E = edge_factor * V
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    ab, abc = a + b, a + b + c
    keys = []
    for off in range(0, E, chunk):
        n = min(chunk, E - off)
        s = torch.zeros(n, dtype=torch.int64, device=device)
        d = torch.zeros(n, dtype=torch.int64, device=device)
        for bit in range(scale):
            r = torch.rand(n, generator=gen, device=device)
            s |= (r >= ab).to(torch.int64) << bit
            d |= (((r >= a) & (r < ab)) | (r >= abc)).to(torch.int64) << bit
            del r
        keep = s != d
        s, d = s[keep], d[keep]
        keys.append(torch.unique(s * V + d))
        if symmetrize:
            keys.append(torch.unique(d * V + s))
        del s, d, keep
    key = torch.unique(torch.cat(keys))
    del keys
    src = key // V
    col = (key % V).to(torch.int32)
    del key
    rowptr = torch.zeros(V + 1, dtype=torch.int64, device=device)
    rowptr[1:] = torch.cumsum(torch.bincount(src, minlength=V), 0)
    del src
    m = col.numel()
    wgen = torch.Generator(device=device)
    wgen.manual_seed(seed + 1)
    if weight == "uniform":
        w = 1.0 - torch.rand(m, generator=wgen, device=device)                      # (0, 1]
    elif weight == "lognormal":
        w = torch.exp(torch.randn(m, generator=wgen, device=device))
    elif weight.startswith("pareto"):
        alpha = float(weight.split(":")[1]) if ":" in weight else 1.5
        w = torch.pow(1.0 - torch.rand(m, generator=wgen, device=device), -1.0 / alpha)   # Pareto, x_m = 1
    elif weight == "none":
        w = None
    else:
        raise ValueError(weight)
    out = CSR(rowptr.cpu().numpy(), col.cpu().numpy(), None if w is None else w.float().cpu().numpy(),
              name=f"rmat{scale}_ef{edge_factor}_dev")
    return out


def rmat_device_bucketed(scale, edge_factor, a=0.57, b=0.19, c=0.19, seed=0, weight="uniform",
                         max_bucket_edges=1 << 30, device="cuda", chunk=1 << 26):
    """Directed R-MAT as rmat_device() for graphs whose edge keys do not fit
    one on-device sort (scales 27-29): the edge stream (same quadrant rule,
    one torch Philox generator seeded with `seed`) is replayed once to count
    edges per coarse source range, the ranges are merged into buckets of at
    most max_bucket_edges generated edges (R-MAT puts most edges on low
    source ids, so equal ranges would not do), then replayed once per bucket,
    keeping that bucket's edges, which are deduplicated and turned into its
    CSR rows in host memory.  Self-loops and duplicates are removed.
    Weights come from a generator seeded with seed + 1 + bucket."""
    import torch
    V = 1 << scale
    E = edge_factor * V
    ab, abc = a + b, a + b + c

    def stream():
        gen = torch.Generator(device=device)
        gen.manual_seed(seed)
        for off in range(0, E, chunk):
            n = min(chunk, E - off)
            s = torch.zeros(n, dtype=torch.int64, device=device)
            d = torch.zeros(n, dtype=torch.int64, device=device)
            for bit in range(scale):
                r = torch.rand(n, generator=gen, device=device)
                s |= (r >= ab).to(torch.int64) << bit
                d |= (((r >= a) & (r < ab)) | (r >= abc)).to(torch.int64) << bit
                del r
            yield s, d
            del s, d

    cbits = min(16, scale - 1)
    cshift = scale - cbits
    counts = torch.zeros(1 << cbits, dtype=torch.int64, device=device)
    for s, d in stream():
        counts += torch.bincount(s >> cshift, minlength=1 << cbits)
    counts = counts.cpu().numpy()
    bounds = [0]   # coarse range boundaries of the buckets
    acc = 0
    for k, n in enumerate(counts):
        if acc and acc + n > max_bucket_edges:
            bounds.append(k)
            acc = 0
        acc += int(n)
    bounds.append(1 << cbits)
    rowptr = np.zeros(V + 1, dtype=np.int64)
    # filled in place (the generated edge count bounds the deduplicated one),
    # so host memory peaks near the final graph size
    col_all = np.empty(E, dtype=np.int32)
    w_all = None if weight == "none" else np.empty(E, dtype=np.float32)
    total = 0
    for bk in range(len(bounds) - 1):
        lo, hi = bounds[bk] << cshift, bounds[bk + 1] << cshift
        keys = []
        for s, d in stream():
            keep = (s >= lo) & (s < hi) & (s != d)
            keys.append(torch.unique(s[keep] * V + d[keep]))
            del keep
        key = torch.unique(torch.cat(keys))
        del keys
        src = key // V
        col = (key % V).to(torch.int32)
        del key
        cnt = torch.bincount(src - lo, minlength=hi - lo)
        del src
        rowptr[lo + 1:hi + 1] = total + torch.cumsum(cnt, 0).cpu().numpy()
        m = col.numel()
        col_all[total:total + m] = col.cpu().numpy()
        del col
        wgen = torch.Generator(device=device)
        wgen.manual_seed(seed + 1 + bk)
        if weight == "uniform":
            w = 1.0 - torch.rand(m, generator=wgen, device=device)
        elif weight.startswith("pareto"):
            alpha = float(weight.split(":")[1]) if ":" in weight else 1.5
            w = torch.pow(1.0 - torch.rand(m, generator=wgen, device=device), -1.0 / alpha)
        elif weight == "none":
            w = None
        else:
            raise ValueError(weight)
        if w is not None:
            w_all[total:total + m] = w.float().cpu().numpy()
        total += m
        del w
        if device != "cpu":
            torch.cuda.empty_cache()
    return CSR(rowptr, col_all[:total], None if w_all is None else w_all[:total],
               name=f"rmat{scale}_ef{edge_factor}_dev")


def powerlaw_directed(n_vertices=875_713, n_edges=5_105_039, gamma=2.1, max_degree=460, zipf=0.6,
                      seed=0, weight="lognormal"):
    """Directed graph whose out-degrees follow P(d) ~ d^-gamma on [1, max_degree]."""
    V, E = n_vertices, n_edges
    rng = np.random.Generator(np.random.PCG64(seed))
    ds = np.arange(1, max_degree + 1, dtype=np.float64)
    pmf = ds ** (-gamma)
    pmf /= pmf.sum()
    deg = rng.choice(ds.astype(np.int64), size=V, p=pmf)
    # rescale the sequence to sum to E (keeps the power-law shape), cap, then fix the remainder
    deg = np.minimum(np.floor(deg * (E / deg.sum())).astype(np.int64), max_degree)
    deg[np.argmax(deg)] = max_degree
    diff = E - int(deg.sum())
    while diff != 0:
        idx = rng.integers(0, V, size=abs(diff) * 2)
        for v in idx:
            if diff > 0 and deg[v] < max_degree:
                deg[v] += 1
                diff -= 1
            elif diff < 0 and deg[v] > 0 and deg[v] != max_degree:
                deg[v] -= 1
                diff += 1
            if diff == 0:
                break
    # destinations: Zipf popularity over a random permutation of the vertices
    perm = rng.permutation(V)
    pop = (np.arange(1, V + 1, dtype=np.float64)) ** (-zipf)
    cdf = np.cumsum(pop)
    cdf /= cdf[-1]
    src = np.repeat(np.arange(V, dtype=np.int64), deg)
    dst = perm[np.searchsorted(cdf, rng.random(src.size))]
    for _ in range(64):  # redraw self loops and duplicate (src, dst) pairs
        key = src * V + dst
        order = np.argsort(key, kind="stable")
        ks = key[order]
        dup = np.zeros(ks.size, dtype=bool)
        dup[1:] = ks[1:] == ks[:-1]
        bad = np.zeros(src.size, dtype=bool)
        bad[order[dup]] = True
        bad |= src == dst
        nb = int(bad.sum())
        if nb == 0:
            break
        dst[bad] = perm[np.searchsorted(cdf, rng.random(nb))]
    else:
        raise RuntimeError("could not remove duplicate edges")
    rowptr, col = _csr_from_edges(src, dst, V)
    w = weights(weight, col.size, seed + 1)
    return CSR(rowptr, col, w, name=f"powerlaw_v{V}_e{E}")


def write_reference_format(g, beg_path, csr_path):
    """beg.bin = int64[V+1], csr.bin = int64[E] (reference graph.hpp:18-34)."""
    g.rowptr.astype(np.int64).tofile(beg_path)
    g.col.astype(np.int64).tofile(csr_path)


def read_reference_format(beg_path, csr_path):
    rowptr = np.fromfile(beg_path, dtype=np.int64)
    col = np.fromfile(csr_path, dtype=np.int64)[: rowptr[-1]]
    return CSR(rowptr, col.astype(np.int32), None, name="file")
