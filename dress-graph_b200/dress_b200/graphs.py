"""Seeded synthetic graphs for the DRESS workloads.

Every generator returns ``(N, U, V)`` with int32 ``U``/``V`` listing each
undirected edge exactly once (the convention of the reference's tests,
e.g. ``tests/c/test_delta_dress.c:71-72``), no self-loops and no parallel
edges.  The same seed always gives the same graph.
"""
import numpy as np


def _dedupe_pairs(a, b, n):
    lo = np.minimum(a, b).astype(np.int64)
    hi = np.maximum(a, b).astype(np.int64)
    keep = lo != hi
    key = lo[keep] * n + hi[keep]
    _, first = np.unique(key, return_index=True)
    first.sort()                       # keep the order of first appearance
    return key[first]


def erdos_renyi(n, m, seed=42):
    """G(n, m): m distinct unordered pairs drawn uniformly by rejection."""
    rng = np.random.default_rng(seed)
    if m > n * (n - 1) // 2:
        raise ValueError("too many edges")
    keys = np.zeros(0, dtype=np.int64)
    while keys.size < m:
        need = int((m - keys.size) * 1.2) + 16
        a = rng.integers(0, n, need)
        b = rng.integers(0, n, need)
        keys = _dedupe_pairs(np.concatenate([keys // n, a]),
                             np.concatenate([keys % n, b]), n)
    keys = keys[:m]
    U = (keys // n).astype(np.int32)
    V = (keys % n).astype(np.int32)
    return n, U, V


def chung_lu(n, m, gamma=2.3, max_degree=20000, seed=42):
    """Chung-Lu power-law graph with exactly m distinct undirected edges.

    Expected degrees follow w_i ~ i^(-1/(gamma-1)), scaled to mean 2m/n and
    capped at ``max_degree``; endpoints are drawn proportionally to w,
    loops and duplicates are rejected, and vertex ids are shuffled.
    """
    rng = np.random.default_rng(seed)
    i = np.arange(1, n + 1, dtype=np.float64)
    w = i ** (-1.0 / (gamma - 1.0))
    w *= (2.0 * m / n) / w.mean()
    for _ in range(50):                # cap, then rescale the rest to keep the mean
        over = w > max_degree
        if not over.any():
            break
        w[over] = max_degree
        rest = ~over
        w[rest] *= (2.0 * m - w[over].sum()) / w[rest].sum()
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    keys = np.zeros(0, dtype=np.int64)
    while keys.size < m:
        need = int((m - keys.size) * 1.3) + 1024
        a = np.searchsorted(cdf, rng.random(need), side="right").clip(0, n - 1)
        b = np.searchsorted(cdf, rng.random(need), side="right").clip(0, n - 1)
        keys = _dedupe_pairs(np.concatenate([keys // n, a]),
                             np.concatenate([keys % n, b]), n)
    keys = keys[:m]
    perm = rng.permutation(n).astype(np.int64)
    U = perm[keys // n].astype(np.int32)
    V = perm[keys % n].astype(np.int32)
    order = rng.permutation(m)
    return n, U[order], V[order]


def random_regular(n, d, seed=42, max_rounds=100000):
    """Random d-regular simple graph from the configuration model.

    A random stub pairing is drawn, then every loop or repeated pair is
    rejected and re-paired by a degree-preserving switch with a random other
    pair ({a,b},{c,e} -> {a,c},{b,e}), accepted only when it creates no new
    loop or repeat; this is the usual switching repair of the pairing model.
    """
    if (n * d) % 2 or d >= n:
        raise ValueError("n*d must be even and d < n")
    rng = np.random.default_rng(seed)
    stubs = rng.permutation(np.repeat(np.arange(n, dtype=np.int64), d))
    pairs = [[int(a), int(b)] for a, b in zip(stubs[0::2], stubs[1::2])]
    m = len(pairs)
    count = {}
    for a, b in pairs:
        k = (min(a, b), max(a, b))
        count[k] = count.get(k, 0) + 1

    def bad(i):
        a, b = pairs[i]
        return a == b or count[(min(a, b), max(a, b))] > 1

    def ok(a, b):
        return a != b and (min(a, b), max(a, b)) not in count

    for _ in range(max_rounds):
        bads = [i for i in range(m) if bad(i)]
        if not bads:
            lo = np.array([min(p) for p in pairs], dtype=np.int32)
            hi = np.array([max(p) for p in pairs], dtype=np.int32)
            return n, lo, hi
        for i in bads:
            if not bad(i):
                continue
            j = int(rng.integers(m))
            if j == i:
                continue
            a, b = pairs[i]
            c, e = pairs[j]
            if rng.random() < 0.5:
                c, e = e, c
            for key in ((min(a, b), max(a, b)), (min(c, e), max(c, e))):
                count[key] -= 1
                if count[key] == 0:
                    del count[key]
            if ok(a, c) and ok(b, e) and (min(a, c), max(a, c)) != (min(b, e), max(b, e)):
                pairs[i], pairs[j] = [a, c], [b, e]
            for x, y in pairs[i], pairs[j]:
                key = (min(x, y), max(x, y))
                count[key] = count.get(key, 0) + 1
    raise RuntimeError("switching repair did not converge")


def regular_batch(count, n_range=(16, 100), d_range=(3, 12), seed=42):
    """``count`` random d-regular graphs with n ~ U[n_range] and
    d ~ U{d_range}, d resampled until n*d is even (one seed per graph)."""
    rng = np.random.default_rng(seed)
    out = []
    for gi in range(count):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        while True:
            d = int(rng.integers(d_range[0], d_range[1] + 1))
            if (n * d) % 2 == 0 and d < n:
                break
        out.append(random_regular(n, d, seed=int(rng.integers(1 << 31)) ^ gi))
    return out


def uniform_weights(m, lo=0.5, hi=2.0, seed=7):
    return np.random.default_rng(seed).uniform(lo, hi, m)


def serving_stream(count, seed=5, fit_edges=(10, 1_000_000), delta_edges=(10, 5000), delta_frac=0.3,
                   weighted_frac=0.3, regular_below=5000):
    """Requests of a serving workload: ``count`` tuples (kind, n, U, V, W)
    with kind 2 (fit) or 0 (Delta^1) (a ``delta_frac`` share), edge counts
    log-uniform in ``fit_edges`` / ``delta_edges``, random d-regular graphs
    (d ~ U{3..12}) below ``regular_below`` edges and Chung-Lu power-law
    graphs (mean degree 14, gamma 2.3) above, a ``weighted_frac`` share with
    U[0.5, 2.0] edge weights."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        kind = 0 if rng.random() < delta_frac else 2
        lo, hi = delta_edges if kind == 0 else fit_edges
        m = int(round(np.exp(rng.uniform(np.log(lo), np.log(hi)))))
        s = int(rng.integers(1 << 31))
        if m < regular_below:
            d = int(rng.integers(3, 13))
            n = max(d + 1, (2 * m) // d)
            if (n * d) % 2:
                n += 1
            n, U, V = random_regular(n, d, seed=s)
        else:
            n = max(16, m // 7)
            n, U, V = chung_lu(n, m, 2.3, min(20000, n // 2), seed=s)
        W = uniform_weights(len(U), seed=s + 1) if rng.random() < weighted_frac else None
        out.append((kind, n, U, V, W))
    return out
