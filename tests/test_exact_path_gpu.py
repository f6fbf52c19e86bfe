"""The sorted path behind the certified sums, on the GPU.

Every sum of the engine is a certified sum in gathering order; an item whose
certificate fails is summed the reference's way (sort ascending, then
sequential KBN, libdress/src/dress.c:51-66).  Real inputs almost never fail
the certificate, so these tests configure the engine with exact_sums=1,
which sends EVERY item down that sorted path, and require the same bits as
the oracle: the single-graph fit (shared-memory sorts and, for a hub beyond
shared memory, the global-scratch sort), the one-launch fits and the
batched Delta/Nabla kernel (its in-place selection order).
"""
import numpy as np
import pytest

import dress_b200 as db
from dress_b200 import graphs

pytestmark = pytest.mark.gpu


def bits(a):
    return np.asarray(a, dtype=np.float64).view(np.int64)


@pytest.fixture
def exact_sums():
    db.configure(exact_sums=1)
    try:
        yield
    finally:
        db.configure()


def gpu_fit(n, U, V, W=None, NW=None, variant=0, max_iterations=100, epsilon=1e-6):
    with db.Graph(n, U, V, W, NW, variant, 0) as g:
        it, dl = db.fit_graph(g, max_iterations, epsilon)
        return dict(edge_dress=g.edge_dress, vertex_dress=g.vertex_dress, iterations=it, delta=dl)


def assert_same(a, b):
    assert a["iterations"] == b["iterations"]
    assert bits([a["delta"]])[0] == bits([b["delta"]])[0]
    np.testing.assert_array_equal(bits(a["edge_dress"]), bits(b["edge_dress"]))
    np.testing.assert_array_equal(bits(a["vertex_dress"]), bits(b["vertex_dress"]))


def test_single_fit_sorted_path(oracle_port, exact_sums):
    # thread, warp and block items of a power-law graph, weighted, vertex weights
    n, U, V = graphs.chung_lu(20000, 120000, 2.3, 3000, seed=3)
    W = graphs.uniform_weights(len(U), seed=2)
    NW = np.random.default_rng(1).uniform(0.5, 2.0, n)
    assert_same(gpu_fit(n, U, V, W, NW, max_iterations=12), oracle_port.fit(n, U, V, W, NW, max_iterations=12))
    for variant in (1, 2):
        nn, U2, V2 = graphs.erdos_renyi(3000, 12000, seed=variant)
        assert_same(gpu_fit(nn, U2, V2, variant=variant), oracle_port.fit(nn, U2, V2, variant=variant))


def test_hub_beyond_shared_memory_sorted_path(oracle_port, exact_sums):
    # a 40000-leaf star: the hub's 40001 terms are sorted in global scratch
    n = 40001
    U = np.zeros(40000, np.int32)
    V = np.arange(1, 40001, dtype=np.int32)
    assert_same(gpu_fit(n, U, V, max_iterations=5), oracle_port.fit(n, U, V, max_iterations=5))


def test_one_launch_fits_sorted_path(oracle_port, exact_sums):
    for n, m in ((300, 1200), (1500, 6000)):
        n, U, V = graphs.erdos_renyi(n, m, seed=9)
        W = graphs.uniform_weights(m, seed=5)
        assert_same(gpu_fit(n, U, V, W), oracle_port.fit(n, U, V, W))


def test_batched_delta_nabla_sorted_path(oracle_port, exact_sums):
    gs = graphs.regular_batch(12, (16, 40), (3, 9), seed=4)
    objs = [db.Graph(n, U, V) for n, U, V in gs]
    for kind, fn in ((db.DELTA, oracle_port.delta_fit), (db.NABLA, oracle_port.nabla_fit)):
        flats = [r[0] for r in db.hist_requests(objs, kind, 1)]
        for (n, U, V), flat in zip(gs, flats):
            np.testing.assert_array_equal(flat, fn(n, U, V, k=1)["hist"])
    for g in objs:
        g.close()


def test_large_graph_layout_sorted_path(oracle_port, exact_sums):
    # the renumbered layout of a graph above 2^20 edges, every item sorted
    n, U, V = graphs.chung_lu(200_000, 1_200_000, 2.3, 3000, seed=5)
    W = graphs.uniform_weights(len(U), seed=6)
    assert_same(gpu_fit(n, U, V, W, max_iterations=4), oracle_port.fit(n, U, V, W, precompute=1, max_iterations=4))
