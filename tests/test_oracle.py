"""The oracle (CPU restatement) is pinned to the reference.

* against the golden fixtures produced by the reference library
  (tests/golden/make_golden.py);
* against the reference's own known-answer checks (tests/c/test_dress.c,
  tests/c/test_delta_dress.c), restated;
* against the reference library itself on seeded random graphs, where it was
  built (oracle/_ref).
"""
import gzip
import json
import os

import numpy as np
import pytest

from dress_b200 import graphs

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    with gzip.open(os.path.join(GOLDEN, name), "rt") as f:
        return json.load(f)


def bits(a):
    return np.asarray(a, dtype=np.float64).view(np.int64)


def test_oracle_golden_fits(oracle_port):
    cases = load("fit_cases.json.gz")
    assert len(cases) > 400
    for c in cases:
        r = oracle_port.fit(c["N"], c["U"], c["V"], c["W"], variant=c["variant"], precompute=c["precompute"],
                            max_iterations=c["max_iterations"], epsilon=c["eps"])
        assert r["iterations"] == c["iterations"], c["name"]
        assert bits([r["delta"]])[0] == c["delta"], c["name"]
        np.testing.assert_array_equal(bits(r["edge_dress"]), c["edge_dress"], err_msg=c["name"])
        np.testing.assert_array_equal(bits(r["vertex_dress"]), c["vertex_dress"], err_msg=c["name"])


def test_oracle_golden_hists(oracle_port):
    cases = load("hist_cases.json.gz")
    assert len(cases) > 400
    for c in cases:
        fn = oracle_port.delta_fit if c["kind"] == "delta" else oracle_port.nabla_fit
        r = fn(c["N"], c["U"], c["V"], c["W"], k=c["k"], n_samples=c["n_samples"], seed=c["seed"],
               offset=c["offset"], stride=c["stride"], keep_multisets=True, variant=c["variant"])
        assert r["num"] == c["num"]
        np.testing.assert_array_equal(r["hist"], np.asarray(c["hist"], dtype=np.int64))
        if c["multisets"] is not None:
            np.testing.assert_array_equal(bits(r["multisets"].ravel()), c["multisets"])


def _hist_pairs(flat):
    f = np.asarray(flat, dtype=np.int64).reshape(-1, 2)
    return f[:, 0].copy().view(np.float64), f[:, 1]


def test_oracle_known_answers(oracle_port):
    """Restated checks of tests/c/test_delta_dress.c:123-341 and
    tests/c/test_dress.c:103-105."""
    K3 = (3, [0, 1, 0], [1, 2, 2])
    K4 = (4, [0, 0, 0, 1, 1, 2], [1, 2, 3, 2, 3, 3])
    P4 = (4, [0, 1, 2], [1, 2, 3])
    for (n, U, V), k, total, single2 in ((K3, 0, 3, True), (K3, 1, 3, False), (K3, 2, 0, False),
                                         (K4, 0, 6, True), (K4, 1, 12, True), (K4, 2, 6, False)):
        r = oracle_port.delta_fit(n, U, V, k=k, epsilon=1e-3)
        v, c = _hist_pairs(r["hist"])
        assert c.sum() == total
        if single2:
            assert len(v) == 1 and abs(v[0] - 2.0) < 1e-9
    r = oracle_port.delta_fit(*K3, k=3)
    assert r["hist"].size == 0
    r = oracle_port.delta_fit(*P4, k=0, epsilon=1e-3)
    assert len(_hist_pairs(r["hist"])[0]) > 1
    # precompute == merge
    a = oracle_port.delta_fit(*K4, k=1, epsilon=1e-3, precompute=0)
    b = oracle_port.delta_fit(*K4, k=1, epsilon=1e-3, precompute=1)
    np.testing.assert_array_equal(a["hist"], b["hist"])
    # undirected weights double
    g = oracle_port.build(3, [0, 1, 0], [1, 2, 2], [1.0, 2.0, 3.0])
    np.testing.assert_array_equal(oracle_port.csr(g)["edge_weight"], [2.0, 4.0, 6.0])
    oracle_port.free_graph(g)


def test_oracle_relabel_invariance(oracle_port):
    """Sorted fingerprints are bitwise equal under relabelling and edge
    reordering (tests/c/test_dress.c:500-636)."""
    rng = np.random.default_rng(4)
    n, U, V = graphs.erdos_renyi(40, 120, seed=2)
    W = graphs.uniform_weights(120, seed=5)
    base = np.sort(oracle_port.fit(n, U, V, W)["edge_dress"])
    perm = rng.permutation(n)
    order = rng.permutation(120)
    r = oracle_port.fit(n, perm[U][order], perm[V][order], W[order])
    np.testing.assert_array_equal(bits(np.sort(r["edge_dress"])), bits(base))


def _random_case(rng, kind):
    if kind == "er":
        return graphs.erdos_renyi(50, 150, seed=int(rng.integers(1 << 30)))
    if kind == "multi":
        n = 12
        U = rng.integers(0, n, 40).astype(np.int32)
        V = rng.integers(0, n, 40).astype(np.int32)
        return n, U, V
    n, U, V = graphs.chung_lu(200, 700, 2.3, 40, seed=int(rng.integers(1 << 30)))
    return n, U, V


def test_oracle_vs_reference_random(oracle_port, oracle_ref):
    rng = np.random.default_rng(123)
    for trial in range(12):
        kind = ("er", "multi", "cl")[trial % 3]
        n, U, V = _random_case(rng, kind)
        W = rng.uniform(0.5, 2.0, len(U)) if trial % 2 else None
        NW = rng.uniform(0.5, 3.0, n) if trial % 4 == 1 else None
        for variant in range(4):
            for pre in (0, 1):
                a = oracle_port.fit(n, U, V, W, NW, variant=variant, precompute=pre)
                b = oracle_ref.fit(n, U, V, W, NW, variant=variant, precompute=pre)
                assert a["iterations"] == b["iterations"]
                np.testing.assert_array_equal(bits(a["edge_dress"]), bits(b["edge_dress"]))
                np.testing.assert_array_equal(bits(a["vertex_dress"]), bits(b["vertex_dress"]))
                ga = oracle_port.build(n, U, V, W, NW, variant, pre)
                gb = oracle_ref.build(n, U, V, W, NW, variant, pre)
                ca, cb = oracle_port.csr(ga), oracle_ref.csr(gb)
                for key in ca:
                    np.testing.assert_array_equal(ca[key], cb[key], err_msg=key)
                oracle_port.free_graph(ga)
                oracle_ref.free_graph(gb)


def test_oracle_vs_reference_hist_random(oracle_port, oracle_ref):
    rng = np.random.default_rng(7)
    for trial in range(6):
        n, U, V = graphs.random_regular(int(rng.choice([10, 12, 14])), 3, seed=trial)
        W = rng.uniform(0.5, 2.0, len(U)) if trial % 2 else None
        for fn in ("delta_fit", "nabla_fit"):
            for k, ns, off, st in ((1, 0, 0, 1), (2, 0, 1, 3), (2, 9, 0, 1), (2, 5, 2, 3)):
                a = getattr(oracle_port, fn)(n, U, V, W, k=k, n_samples=ns, seed=trial, offset=off, stride=st,
                                             keep_multisets=True, variant=trial % 2)
                b = getattr(oracle_ref, fn)(n, U, V, W, k=k, n_samples=ns, seed=trial, offset=off, stride=st,
                                            keep_multisets=True, variant=trial % 2)
                np.testing.assert_array_equal(a["hist"], b["hist"])
                assert a["num"] == b["num"]
                np.testing.assert_array_equal(bits(a["multisets"]), bits(b["multisets"]))


def test_virtual_edge_query_matches_reference(oracle_port, oracle_ref):
    """dress_get (libdress/src/dress.c:651-739): existing edges, virtual
    edges with and without common neighbours, every variant, weights."""
    from dress_b200 import graphs
    rng = np.random.default_rng(4)
    n, U, V = graphs.chung_lu(300, 1500, 2.3, 60, seed=9)
    W = graphs.uniform_weights(len(U), seed=3)
    NW = rng.uniform(0.5, 2.0, n)
    q = [(int(a), int(b)) for a, b in rng.integers(0, n, (400, 2)) if a != b]
    q += [(int(U[i]), int(V[i])) for i in range(0, len(U), 50)]
    for variant in range(4):
        for w, nw, ew in ((None, None, 1.0), (W, NW, 0.7)):
            a = oracle_port.get_many(n, U, V, w, q, NW=nw, variant=variant, edge_weight=ew)
            b = oracle_ref.get_many(n, U, V, w, q, NW=nw, variant=variant, edge_weight=ew)
            np.testing.assert_array_equal(a.view(np.int64), b.view(np.int64))
