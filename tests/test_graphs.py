"""The seeded synthetic inputs of the benchmarks and tests (CPU only): every
generator lists each undirected edge once, without loops or parallel edges,
with the shapes the workloads are defined by, and the same seed gives the
same graph."""
import numpy as np

from dress_b200 import graphs


def simple(n, U, V):
    assert U.dtype == np.int32 and V.dtype == np.int32 and U.shape == V.shape
    assert ((U >= 0) & (U < n) & (V >= 0) & (V < n)).all()
    assert (U != V).all()
    lo, hi = np.minimum(U, V).astype(np.int64), np.maximum(U, V).astype(np.int64)
    assert np.unique(lo * n + hi).size == U.size


def degrees(n, U, V):
    return np.bincount(U, minlength=n) + np.bincount(V, minlength=n)


def test_erdos_renyi_exact_edge_count():
    n, U, V = graphs.erdos_renyi(2000, 10000, seed=42)
    assert n == 2000 and U.size == 10000
    simple(n, U, V)
    again = graphs.erdos_renyi(2000, 10000, seed=42)
    assert np.array_equal(again[1], U) and np.array_equal(again[2], V)


def test_random_regular_is_regular_and_simple():
    for n, d in ((16, 3), (50, 7), (100, 12), (200, 10)):
        n2, U, V = graphs.random_regular(n, d, seed=3)
        assert n2 == n and U.size == n * d // 2
        simple(n, U, V)
        assert (degrees(n, U, V) == d).all()


def test_regular_batch_shapes():
    gs = graphs.regular_batch(200, (16, 100), (3, 12), seed=42)
    assert len(gs) == 200
    for n, U, V in gs:
        assert 16 <= n <= 100
        deg = degrees(n, U, V)
        d = int(deg[0])
        assert 3 <= d <= 12 and (deg == d).all() and (n * d) % 2 == 0
        simple(n, U, V)


def test_chung_lu_power_law_and_cap():
    n, U, V = graphs.chung_lu(20000, 140000, 2.3, 3000, seed=5)
    assert U.size == 140000
    simple(n, U, V)
    deg = degrees(n, U, V)
    assert deg.max() <= 3000 * 2          # capped expectation, sampled
    assert deg.max() > 20 * deg.mean()    # heavy tail


def test_serving_stream_mix():
    reqs = graphs.serving_stream(60, seed=5)
    assert len(reqs) == 60
    kinds = {k for k, *_ in reqs}
    assert kinds <= {0, 2}
    for kind, n, U, V, W in reqs:
        simple(n, U, V)
        if kind == 0:
            assert U.size <= 5000 + 12
        if W is not None:
            assert W.shape == U.shape and (W >= 0.5).all() and (W <= 2.0).all()
