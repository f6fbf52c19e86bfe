"""GPU parity of dress_fit_cuda against the oracle and the golden fixtures.

Bar: bit-identical edge and vertex values, identical iteration count and
final delta (the reference's own CUDA test accepts 1e-12,
tests/c/cuda/test_dress_cuda.c:180; this engine is exact).
"""
import ctypes
import gzip
import json
import os
import subprocess

import numpy as np
import pytest

import dress_b200 as db
from dress_b200 import graphs

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def bits(a):
    return np.asarray(a, dtype=np.float64).view(np.int64)


def gpu_fit(n, U, V, W=None, NW=None, variant=0, pre=0, max_iterations=100, epsilon=1e-6):
    with db.Graph(n, U, V, W, NW, variant, pre) as g:
        it, dl = db.fit_graph(g, max_iterations, epsilon)
        return dict(edge_dress=g.edge_dress, vertex_dress=g.vertex_dress, iterations=it, delta=dl)


def assert_same(a, b, name=""):
    assert a["iterations"] == b["iterations"], (name, a["iterations"], b["iterations"])
    assert bits([a["delta"]])[0] == bits([b["delta"]])[0], (name, a["delta"], b["delta"])
    np.testing.assert_array_equal(bits(a["edge_dress"]), bits(b["edge_dress"]), err_msg=name)
    np.testing.assert_array_equal(bits(a["vertex_dress"]), bits(b["vertex_dress"]), err_msg=name)


def test_golden_fits():
    with gzip.open(os.path.join(ROOT, "tests", "golden", "fit_cases.json.gz"), "rt") as f:
        cases = json.load(f)
    for c in cases:
        r = gpu_fit(c["N"], c["U"], c["V"], c["W"], None, c["variant"], c["precompute"],
                    c["max_iterations"], c["eps"])
        assert r["iterations"] == c["iterations"], c["name"]
        assert bits([r["delta"]])[0] == c["delta"], c["name"]
        np.testing.assert_array_equal(bits(r["edge_dress"]), c["edge_dress"], err_msg=c["name"])
        np.testing.assert_array_equal(bits(r["vertex_dress"]), c["vertex_dress"], err_msg=c["name"])


@pytest.mark.parametrize("variant", [0, 1, 2, 3])
@pytest.mark.parametrize("weighted", [False, True])
def test_er2000_all_variants(oracle_port, variant, weighted):
    """The plain-fit workload: G(2000, 10000)."""
    n, U, V = graphs.erdos_renyi(2000, 10000, seed=42)
    W = graphs.uniform_weights(10000, seed=1) if weighted else None
    a = gpu_fit(n, U, V, W, variant=variant)
    b = oracle_port.fit(n, U, V, W, variant=variant)
    assert_same(a, b)


@pytest.mark.parametrize("variant", [0, 1, 2, 3])
@pytest.mark.parametrize("n,m", [(300, 1200), (1500, 6000)])
def test_one_launch_fits(oracle_port, variant, n, m):
    """Graphs fitted in one launch: up to 2048 edges by one CTA with the
    graph in shared memory, up to 8192 by a cluster of CTAs whose
    distributed shared memory holds the state."""
    n, U, V = graphs.erdos_renyi(n, m, seed=9)
    W = graphs.uniform_weights(m, seed=5)
    NW = np.random.default_rng(2).uniform(0.5, 2.0, n)
    a = gpu_fit(n, U, V, W, NW, variant=variant)
    b = oracle_port.fit(n, U, V, W, NW, variant=variant)
    assert_same(a, b)


@pytest.mark.parametrize("pre", [0, 1])
def test_powerlaw_bins(oracle_port, pre):
    """Chung-Lu graph whose rows and triangle counts fill every bin
    (thread, warp and block items)."""
    n, U, V = graphs.chung_lu(20000, 120000, 2.3, 3000, seed=3)
    W = graphs.uniform_weights(len(U), seed=2)
    NW = np.random.default_rng(1).uniform(0.5, 2.0, n)
    a = gpu_fit(n, U, V, W, NW, pre=pre)
    b = oracle_port.fit(n, U, V, W, NW, precompute=1)
    assert_same(a, b)


def test_hub_row_larger_than_shared_memory(oracle_port):
    """A star with 40000 leaves: the hub's 40001-term norm spills to global."""
    n = 40001
    U = np.zeros(40000, np.int32)
    V = np.arange(1, 40001, dtype=np.int32)
    a = gpu_fit(n, U, V)
    b = oracle_port.fit(n, U, V)
    assert_same(a, b)


def test_hub_edge_with_many_common_neighbours(oracle_port):
    """Two hubs sharing 5000 neighbours and joined by an edge: that edge's
    5001-term sum is a hub-edge item, streamed by a whole warp."""
    k = 5000
    leaves = np.arange(2, k + 2, dtype=np.int32)
    U = np.concatenate([[0], np.zeros(k, np.int32), np.ones(k, np.int32)]).astype(np.int32)
    V = np.concatenate([[1], leaves, leaves]).astype(np.int32)
    W = graphs.uniform_weights(len(U), seed=4)
    a = gpu_fit(k + 2, U, V, W)
    b = oracle_port.fit(k + 2, U, V, W)
    assert_same(a, b)


def test_multigraph_and_self_loops(oracle_port):
    rng = np.random.default_rng(9)
    n = 30
    U = rng.integers(0, n, 200).astype(np.int32)
    V = rng.integers(0, n, 200).astype(np.int32)
    W = rng.uniform(0.5, 2.0, 200)
    for variant in range(4):
        assert_same(gpu_fit(n, U, V, W, variant=variant), oracle_port.fit(n, U, V, W, variant=variant), str(variant))


def test_degenerate_inputs(oracle_port):
    # no edges, no vertices, zero iterations, epsilon 0 (all sweeps run)
    assert_same(gpu_fit(5, [], []), oracle_port.fit(5, [], []))
    assert_same(gpu_fit(0, [], []), oracle_port.fit(0, [], []))
    n, U, V = graphs.erdos_renyi(50, 120, seed=4)
    assert_same(gpu_fit(n, U, V, epsilon=0.0, max_iterations=7),
                oracle_port.fit(n, U, V, epsilon=0.0, max_iterations=7))
    with db.Graph(n, U, V) as g:
        it, _ = db.fit_graph(g, 0, 1e-6)
        assert it == 0
        np.testing.assert_array_equal(g.edge_dress, 1.0)


def test_fit_continues_from_current_values(oracle_port):
    """A second call starts from edge_dress, like the reference's dress_fit."""
    n, U, V = graphs.erdos_renyi(300, 1200, seed=8)
    with db.Graph(n, U, V) as g:
        db.fit_graph(g, 3, 1e-6)
        it, dl = db.fit_graph(g, 100, 1e-9)
        ed = g.edge_dress
    gb = oracle_port.build(n, U, V)
    it0, d0 = ctypes.c_int(), ctypes.c_double()
    oracle_port.fit_fn(gb, 3, 1e-6, ctypes.byref(it0), ctypes.byref(d0))
    oracle_port.fit_fn(gb, 100, 1e-9, ctypes.byref(it0), ctypes.byref(d0))
    ref = np.ctypeslib.as_array(gb.contents.edge_dress, (len(U),)).copy()
    oracle_port.free_graph(gb)
    assert it == it0.value and dl == d0.value
    np.testing.assert_array_equal(bits(ed), bits(ref))


def test_python_api_mirror(oracle_port):
    n, U, V = graphs.erdos_renyi(100, 400, seed=6)
    r = db.fit(n, U.tolist(), V.tolist(), epsilon=1e-8)
    b = oracle_port.fit(n, U, V, epsilon=1e-8)
    assert r.iterations == b["iterations"]
    np.testing.assert_array_equal(bits(r.edge_dress), bits(b["edge_dress"]))
    ed, vd, ew, it, dl = db.dress_cuda(n, len(U), U, V, epsilon=1e-8)
    np.testing.assert_array_equal(bits(ed), bits(b["edge_dress"]))


def test_malformed_graph_is_rejected_without_crash():
    n, U, V = graphs.erdos_renyi(20, 40, seed=1)
    with db.Graph(n, U, V) as g:
        g.ptr.contents.adj_edge_idx[3] = 10_000          # out of range edge id
        with pytest.raises(db.DressError) as e:
            db.fit_graph(g, 10, 1e-6)
        assert e.value.code == 1
    # the engine is still usable afterwards
    with db.Graph(n, U, V) as g:
        db.fit_graph(g, 10, 1e-6)


def test_null_vertex_weights_mean_unit_weights(oracle_port):
    """NW == NULL is all-1.0 vertex weights (libdress/include/dress/dress.h:65);
    the reference's CUDA test relies on it when it deep-copies a graph
    (tests/c/cuda/test_dress_cuda.c:25-86 copies no NW)."""
    n, U, V = graphs.erdos_renyi(200, 800, seed=12)
    with db.Graph(n, U, V) as g:
        db._libc.free(ctypes.cast(g.ptr.contents.NW, ctypes.c_void_p))
        g.ptr.contents.NW = ctypes.POINTER(ctypes.c_double)()
        it, dl = db.fit_graph(g, 100, 1e-6)
        ed = g.edge_dress
        g.ptr.contents.NW = db._malloc_copy(np.ones(n), ctypes.c_double)   # for dress_free_graph
    ref = oracle_port.fit(n, U, V)
    assert it == ref["iterations"]
    np.testing.assert_array_equal(bits(ed), bits(ref["edge_dress"]))


def test_reference_c_tests_through_redirect():
    """The reference's tests/c/test_dress.c, compiled from its sources with the
    reference's include-redirect header (dress_fit -> dress_fit_cuda) and
    linked against this library."""
    exe = os.path.join(ROOT, "oracle", "_ref", "test_dress_redirect")
    if not os.path.exists(exe):
        pytest.skip("reference test binary not built")
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout[-3000:] + out.stderr[-2000:]
    assert " 0 failed" in out.stdout


@pytest.mark.parametrize("variant", [0, 1, 2, 3])
def test_virtual_edge_queries_match_oracle(oracle_port, variant):
    """dressx_get_batch against the oracle's dress_get (pinned to the
    reference): existing edges, non-edges with few and with many common
    neighbours (register and sorted-slot paths), per-pair weights."""
    rng = np.random.default_rng(7 + variant)
    n, U, V = graphs.chung_lu(400, 3000, 2.3, 150, seed=11)
    W = graphs.uniform_weights(len(U), seed=5)
    NW = rng.uniform(0.5, 2.0, n)
    deg = np.bincount(np.concatenate([U, V]), minlength=n)
    hubs = np.argsort(-deg)[:12]
    q = [(int(a), int(b)) for a, b in rng.integers(0, n, (600, 2))]
    q += [(int(a), int(b)) for a in hubs for b in hubs if a != b]          # many common neighbours
    q += [(int(U[i]), int(V[i])) for i in range(0, len(U), 37)]           # existing edges
    qu = np.array([a for a, _ in q], np.int32)
    qv = np.array([b for _, b in q], np.int32)
    with db.Graph(n, U, V, W, NW, variant) as g:
        db.fit_graph(g, 100, 1e-6)
        got = db.get(g, qu, qv, 100, 1e-6, 0.8)
        ews = rng.uniform(0.5, 2.0, len(q))
        got_w = db.get(g, qu, qv, 50, 1e-9, ews)
    ref = oracle_port.get_many(n, U, V, W, q, NW=NW, variant=variant, edge_weight=0.8)
    np.testing.assert_array_equal(bits(got), bits(ref))
    gb = oracle_port.build(n, U, V, W, NW, variant, 0)
    it, dl = ctypes.c_int(), ctypes.c_double()
    oracle_port.fit_fn(gb, 100, 1e-6, ctypes.byref(it), ctypes.byref(dl))
    ref_w = np.array([oracle_port.get_fn(gb, a, b, 50, 1e-9, float(w)) for (a, b), w in zip(q, ews)])
    oracle_port.free_graph(gb)
    np.testing.assert_array_equal(bits(got_w), bits(ref_w))
    assert max(int(deg[a]) for a in hubs) > 40


def test_virtual_edge_query_rejects_bad_vertices():
    n, U, V = graphs.erdos_renyi(50, 100, seed=2)
    with db.Graph(n, U, V) as g:
        db.fit_graph(g, 10, 1e-6)
        with pytest.raises(db.DressError) as e:
            db.get(g, [0, 60], [1, 2])
        assert e.value.code == 1


def _graph_arrays(g):
    c = g.ptr.contents
    S = c.adj_offset[c.N] if c.N > 0 else 0
    out = dict(adj_offset=db._arr(c.adj_offset, c.N + 1, np.int32), adj_target=db._arr(c.adj_target, S, np.int32),
               adj_edge_idx=db._arr(c.adj_edge_idx, S, np.int32), edge_weight=bits(db._arr(c.edge_weight, c.E, np.float64)),
               edge_dress=bits(db._arr(c.edge_dress, c.E, np.float64)), NW=bits(db._arr(c.NW, c.N, np.float64)),
               max_degree=c.max_degree)
    if c.precompute_intercepts:
        T = c.intercept_offset[c.E]
        out.update(intercept_offset=db._arr(c.intercept_offset, c.E + 1, np.int32),
                   intercept_edge_ux=db._arr(c.intercept_edge_ux, T, np.int32),
                   intercept_edge_vx=db._arr(c.intercept_edge_vx, T, np.int32))
    return out


@pytest.mark.parametrize("variant", [0, 1, 2, 3])
def test_device_graph_build_matches_host(variant):
    """dressx_init_graph (GPU) equals dress_init_graph (host, pinned to the
    reference's construction by test_abi) array for array: simple graphs with
    hubs, multigraphs with self loops and reciprocal edges, with and without
    weights, vertex weights and intercept tables."""
    rng = np.random.default_rng(variant)
    cases = [graphs.chung_lu(3000, 20000, 2.3, 400, seed=5), graphs.erdos_renyi(500, 3000, seed=2)]
    m = 4000
    cases.append((300, rng.integers(0, 300, m).astype(np.int32), rng.integers(0, 300, m).astype(np.int32)))
    cases.append((10, np.zeros(0, np.int32), np.zeros(0, np.int32)))
    for n, U, V in cases:
        for W, NW, pre in ((None, None, 0), (graphs.uniform_weights(len(U), seed=3), rng.uniform(0.5, 2, n), 1)):
            with db.Graph(n, U, V, W, NW, variant, pre) as a, db.Graph(n, U, V, W, NW, variant, pre, device_build=True) as b:
                x, y = _graph_arrays(a), _graph_arrays(b)
                assert x.keys() == y.keys()
                for k in x:
                    np.testing.assert_array_equal(x[k], y[k], err_msg=f"{k} n={n} variant={variant} pre={pre}")


def test_device_graph_build_rejects_bad_ids_and_fits_alike(oracle_port):
    with pytest.raises(ValueError):
        db.Graph(5, [0, 7], [1, 2], device_build=True)
    n, U, V = graphs.chung_lu(2000, 12000, 2.3, 300, seed=8)
    with db.Graph(n, U, V, device_build=True) as g:
        it, dl = db.fit_graph(g, 100, 1e-6)
        ed = g.edge_dress
    ref = oracle_port.fit(n, U, V)
    assert it == ref["iterations"]
    np.testing.assert_array_equal(bits(ed), bits(ref["edge_dress"]))


def test_large_fit_digests():
    """The single-fit workload at full size -- Chung-Lu, 4M vertices, 28M
    edges, weighted U[0.5, 2] and unweighted -- against the reference's own
    dress_fit_omp on the same graph: identical iteration count, final delta
    and SHA-256 digests of every edge and vertex value
    (tests/golden/large_fit.json, made by tests/golden/make_large_golden.py)."""
    import hashlib
    with open(os.path.join(ROOT, "tests", "golden", "large_fit.json")) as f:
        gold = json.load(f)
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
    n, U, V = graphs.chung_lu(4_000_000, 28_000_000, 2.3, 20000, seed=42)
    W = graphs.uniform_weights(len(U), seed=7)
    assert (n, len(U)) == (gold["graph"]["N"], gold["graph"]["E"])
    assert sha(U) == gold["graph"]["sha_U"] and sha(V) == gold["graph"]["sha_V"] and sha(W) == gold["graph"]["sha_W"]
    for label, w in (("weighted", W), ("unweighted", None)):
        ref = gold[label]["full"]
        with db.Graph(n, U, V, w, device_build=True) as g:
            it, dl = db.fit_graph(g, 100, 1e-6)
            assert it == ref["iterations"], label
            assert int(np.float64(dl).view(np.int64)) == ref["delta_bits"], label
            assert sha(g.edge_dress) == ref["sha_edge_dress"], label
            assert sha(g.vertex_dress) == ref["sha_vertex_dress"], label


def test_large_graph_layout(oracle_port):
    """A power-law graph above the size where the fit renumbers edges for
    gather locality (2^20 edges): owner order, per-class edge lists and the
    product copy that the vertex phase writes for the pair gathers --
    weighted with vertex weights, and unweighted -- against the oracle."""
    n, U, V = graphs.chung_lu(200_000, 1_200_000, 2.3, 3000, seed=5)
    W = graphs.uniform_weights(len(U), seed=6)
    NW = np.random.default_rng(3).uniform(0.5, 2.0, n)
    assert_same(gpu_fit(n, U, V, W, NW, max_iterations=30), oracle_port.fit(n, U, V, W, NW, precompute=1, max_iterations=30))
    assert_same(gpu_fit(n, U, V, max_iterations=30), oracle_port.fit(n, U, V, precompute=1, max_iterations=30))
