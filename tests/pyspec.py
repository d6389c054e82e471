"""Second, independent restatement of the sampling semantics in pure Python.

Used only by CPU tests, on small cases, to cross-check the C oracle
(oracle/csaw_oracle.c): two restatements written separately from the same
specification must agree bit for bit.  float32 arithmetic is done on numpy
float32 scalars (one IEEE rounding per operation).
"""
import numpy as np

M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85
MASK = 0xFFFFFFFF
TAG_SAMPLE, TAG_MDRW, TAG_SEED = 1, 2, 3
R = 4
MAX_DRAWS = 16
f32 = np.float32


def philox(ctr, key):
    c0, c1, c2, c3 = (int(x) for x in ctr)
    k0, k1 = (int(x) for x in key)
    for _ in range(10):
        p0, p1 = M0 * c0, M1 * c2
        c0, c1, c2, c3 = ((p1 >> 32) ^ c1 ^ k0) & MASK, p1 & MASK, ((p0 >> 32) ^ c3 ^ k1) & MASK, p0 & MASK
        k0, k1 = (k0 + W0) & MASK, (k1 + W1) & MASK
    return [c0, c1, c2, c3]


def word(seed, s, l, p, j, a):
    b = philox([p, s, (TAG_SAMPLE << 24) | l, (j << 16) | (a >> 2)], [seed & MASK, seed >> 32])
    return b[a & 3]


def unit(x):
    return f32(x >> 8) * f32(2.0 ** -24)


def mulhi(x, n):
    return (x * n) >> 32


def below(T):
    return np.array([T], dtype=np.float32).view(np.uint32).__sub__(1).view(np.float32)[0]


def ks(a):
    a = list(a)
    off = 1
    while off < 32:
        prev = list(a)
        for l in range(off, 32):
            a[l] = f32(prev[l] + prev[l - off])
        off *= 2
    return a


def canon_prefix(w):
    d = len(w)
    nt = (d + 31) // 32
    P = [f32(0)] * d
    ts = []
    for t in range(nt):
        a = ks([f32(w[32 * t + l]) if 32 * t + l < d else f32(0) for l in range(32)])
        for l in range(32):
            if 32 * t + l < d:
                P[32 * t + l] = a[l]
        ts.append(a[31])
    C = f32(0)
    for g in range((nt + 31) // 32):
        q = ks([ts[32 * g + l] if 32 * g + l < nt else f32(0) for l in range(32)])
        for l in range(32):
            t = 32 * g + l
            if t >= nt:
                break
            qex = q[l - 1] if l else f32(0)
            for m in range(32):
                i = 32 * t + m
                if i >= d:
                    break
                P[i] = f32(C + f32(qex + P[i]))
        C = f32(C + q[31])
    mx = P[0]
    for i in range(d):
        P[i] = max(mx, P[i])
        mx = P[i]
    return P


def search(P, t):
    for i, v in enumerate(P):
        if v > t:
            return i
    raise AssertionError("no index above target")


def target(x, T):
    t = f32(unit(x) * T)
    return t if t < T else below(T)


def select(wfun, d, N, seed, s, l, p, biased):
    if d <= N:
        return list(range(d))
    S, Z = [], []

    def prefix():
        return canon_prefix([f32(0) if i in Z else f32(wfun(i)) for i in range(d)])

    P = prefix() if biased else None
    T = P[-1] if biased else None
    for j in range(N):
        A = a = 0
        while True:
            if (biased and not T > 0) or A == MAX_DRAWS:
                idx = min(i for i in range(d) if i not in S)
                break
            if a == R:
                Z = sorted(S)
                if biased:
                    P = prefix()
                    T = P[-1]
                a = 0
                continue
            x = word(seed, s, l, p, j, A)
            A += 1
            a += 1
            if biased:
                idx = search(P, target(x, T))
            else:
                t = mulhi(x, d - len(Z))
                for z in Z:
                    if z <= t:
                        t += 1
                idx = t
            if idx not in S:
                break
        S.append(idx)
    return S


def run(csr, seeds, mode, bias, n_samples, F, depth, fanout, seed, dedup=False):
    rp, col, w = csr.rowptr, csr.col, csr.weight
    out = []

    def bias_of(e):
        if bias == 2:
            return w[e]
        u = col[e]
        return float(rp[u + 1] - rp[u])

    for s in range(n_samples):
        if mode == 0:
            cur = [(int(seeds[s * F + f]), f) for f in range(F)]
            seen = set()

            def fresh(items):   # per-sample dedup: first occurrence in lineage order
                keep = []
                for v, p in items:
                    if v not in seen:
                        seen.add(v)
                        keep.append((v, p))
                return keep

            if dedup:
                cur = fresh(cur)
            for l in range(depth):
                N = fanout[l]
                nxt = []
                for v, p in cur:
                    beg, d = int(rp[v]), int(rp[v + 1] - rp[v])
                    if d <= 0:
                        continue
                    sel = select(lambda i: bias_of(beg + i), d, N, seed, s, l, p, bias != 0)
                    for j, idx in enumerate(sel):
                        u = int(col[beg + idx])
                        out.append((v, u, s, l))
                        if l + 1 < depth:
                            nxt.append((u, (p * N + j) & MASK))
                cur = fresh(nxt) if dedup else nxt
        elif mode == 1:
            v = int(seeds[s])
            for t in range(depth):
                beg, d = int(rp[v]), int(rp[v + 1] - rp[v])
                if d <= 0:
                    break
                idx = select(lambda i: bias_of(beg + i), d, 1, seed, s, t, 0, bias != 0)[0]
                u = int(col[beg + idx])
                out.append((v, u, s, t))
                v = u
        else:
            f = [int(x) for x in seeds[s * F:(s + 1) * F]]
            for t in range(depth):
                b = philox([0, s, (TAG_MDRW << 24) | t, 0], [seed & MASK, seed >> 32])
                slot = 0
                if F > 1:
                    P = canon_prefix([f32(1.0) if bias == 0 else f32(rp[v + 1] - rp[v]) for v in f])
                    if P[-1] > 0:
                        slot = search(P, target(b[0], P[-1]))
                v = f[slot]
                beg, d = int(rp[v]), int(rp[v + 1] - rp[v])
                if d <= 0:
                    continue
                u = int(col[beg + mulhi(b[1], d)])
                out.append((v, u, s, t))
                f[slot] = u
    if not out:
        return [np.zeros(0, dtype=np.int32)] * 4
    a = np.array(out, dtype=np.int64)
    return a[:, 0], a[:, 1], a[:, 2], a[:, 3]
