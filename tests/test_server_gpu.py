"""The request server: every result is the same alone and in the mix.

Requests of many sizes (whole-graph fits packed into batch launches, large
fits on lanes, Delta^1 / Nabla^1 histograms on both paths) are submitted from
two threads with staggered arrivals, so later requests are admitted while
earlier ones are on the device.  Each served result must be bit-identical to
the same request run alone through the single-request calls (dressx_fit,
dressx_hist_batch), which the other GPU tests pin to the oracle; a few small
ones are checked against the oracle directly as well.
"""
import threading
import time

import numpy as np
import pytest

import dress_b200 as db
from dress_b200 import graphs

pytestmark = pytest.mark.gpu

EINVAL, EBUDGET, ECANCELLED = 1, 6, 7


def bits(a):
    return np.asarray(a, dtype=np.float64).view(np.int64)


def rr_graph(rng, e_target):
    d = int(rng.integers(3, 13))
    n = max(d + 1, (2 * e_target) // d)
    if (n * d) % 2:
        n += 1
    return graphs.random_regular(n, d, seed=int(rng.integers(1 << 30)))


def make_mix(seed=11):
    """(kind, n, U, V, W) tuples: 36 small fits, 3 large fits, 8 Delta^1,
    2 Nabla^1, 2 hub Delta^1 (batched: rows of any length) and one dense
    Delta^1 whose subgraph state exceeds shared memory (lane path)."""
    rng = np.random.default_rng(seed)
    mix = []
    for _ in range(36):
        n, U, V = rr_graph(rng, int(np.exp(rng.uniform(np.log(10), np.log(5000)))))
        W = graphs.uniform_weights(len(U), seed=int(rng.integers(1 << 30))) if rng.random() < 0.3 else None
        mix.append((db.FIT, n, U, V, W))
    for m in (6000, 20000, 60000):
        n, U, V = graphs.chung_lu(m // 7, m, 2.3, 2000, seed=int(rng.integers(1 << 30)))
        W = graphs.uniform_weights(len(U), seed=3) if m == 20000 else None
        mix.append((db.FIT, n, U, V, W))
    for _ in range(8):
        n, U, V = rr_graph(rng, int(np.exp(rng.uniform(np.log(10), np.log(1500)))))
        mix.append((db.DELTA, n, U, V, None))
    for _ in range(2):
        n, U, V = rr_graph(rng, 200)
        mix.append((db.NABLA, n, U, V, None))
    for m in (300, 500):
        n, U, V = graphs.chung_lu(60, m, 2.3, 50, seed=int(rng.integers(1 << 30)))
        mix.append((db.DELTA, n, U, V, graphs.uniform_weights(len(U), seed=5)))
    n, U, V = graphs.erdos_renyi(200, 15000, seed=int(rng.integers(1 << 30)))
    mix.append((db.DELTA, n, U, V, None))
    order = rng.permutation(len(mix))
    return [mix[i] for i in order]


def alone(kind, n, U, V, W):
    with db.Graph(n, U, V, W) as g:
        if kind == db.FIT:
            it, dl = db.fit_graph(g, 100, 1e-6)
            return dict(iterations=it, delta=dl, edge_dress=g.edge_dress, vertex_dress=g.vertex_dress)
        flat, _, nsub, fits, st = db.hist_requests([g], kind, 1)[0]
        assert st == 0
        return dict(hist_flat=flat, num_subgraphs=nsub, fits=fits)


def assert_same(served, ref, kind, name):
    assert served["status"] == 0, (name, served)
    if kind == db.FIT:
        assert served["iterations"] == ref["iterations"], name
        assert bits([served["delta"]])[0] == bits([ref["delta"]])[0], name
        np.testing.assert_array_equal(bits(served["edge_dress"]), bits(ref["edge_dress"]), err_msg=name)
        np.testing.assert_array_equal(bits(served["vertex_dress"]), bits(ref["vertex_dress"]), err_msg=name)
    else:
        assert served["num_subgraphs"] == ref["num_subgraphs"], name
        assert served["fits"] == ref["fits"], name
        np.testing.assert_array_equal(served["hist_flat"], ref["hist_flat"], err_msg=name)


def serve_mix(server, mix, threads=2, gap_s=0.002):
    """Submit the mix from `threads` threads with staggered arrivals; returns
    the served results in mix order."""
    gs = [db.Graph(n, U, V, W) for (_, n, U, V, W) in mix]
    tickets = [None] * len(mix)

    def worker(t):
        for i in range(t, len(mix), threads):
            tickets[i] = server.submit(gs[i], mix[i][0], 1 if mix[i][0] != db.FIT else 0)
            time.sleep(gap_s)

    ths = [threading.Thread(target=worker, args=(t,)) for t in range(threads)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    out = []
    for i, t in enumerate(tickets):
        r = t.wait(timeout_ms=600_000)
        if mix[i][0] == db.FIT:
            r = dict(r, edge_dress=gs[i].edge_dress, vertex_dress=gs[i].vertex_dress)
        out.append(r)
    for g in gs:
        g.close()
    return out


def test_results_same_alone_and_in_mix():
    mix = make_mix()
    with db.Server(lanes=2) as srv:
        served = serve_mix(srv, mix)
        st = srv.stats()
    paths = {(k, r["path"]) for (k, *_), r in zip(mix, served)}
    # both paths of both kinds were exercised
    assert {(db.FIT, db.PATH_BATCH), (db.FIT, db.PATH_LANE), (db.DELTA, db.PATH_BATCH),
            (db.DELTA, db.PATH_LANE), (db.NABLA, db.PATH_BATCH)} <= paths
    for i, (item, r) in enumerate(zip(mix, served)):
        assert_same(r, alone(*item), item[0], f"request {i} kind {item[0]} n={item[1]} E={len(item[2])}")
    assert st["completed"] == len(mix) and st["failed"] == 0
    assert st["batch_launches"] > 0
    assert st["device_work_ms"] >= st["device_busy_ms"] > 0
    for name in ("fit_batch", "fit_lane", "hist_batch", "hist_lane"):
        c = st[name]
        assert c["completed"] > 0 and 0 < c["p50_ms"] <= c["p99_ms"] <= c["max_ms"]
    assert st["reserved_bytes"] == 0


def test_served_fits_match_oracle(oracle_port):
    rng = np.random.default_rng(3)
    mix = []
    for e in (12, 90, 400, 1500):
        n, U, V = rr_graph(rng, e)
        mix.append((db.FIT, n, U, V, graphs.uniform_weights(len(U), seed=e)))
    n, U, V = graphs.erdos_renyi(2000, 10000, seed=42)
    mix.append((db.FIT, n, U, V, None))          # the plain-fit workload, max degree above 16
    with db.Server() as srv:
        served = serve_mix(srv, mix, threads=1, gap_s=0.0)
    for (k, n, U, V, W), r in zip(mix, served):
        ref = oracle_port.fit(n, U, V, W)
        assert r["iterations"] == ref["iterations"]
        assert bits([r["delta"]])[0] == bits([ref["delta"]])[0]
        np.testing.assert_array_equal(bits(r["edge_dress"]), bits(ref["edge_dress"]))
        np.testing.assert_array_equal(bits(r["vertex_dress"]), bits(ref["vertex_dress"]))


def test_fit_continues_from_current_values_and_zero_iterations():
    n, U, V = graphs.random_regular(60, 4, seed=2)
    with db.Graph(n, U, V) as a, db.Graph(n, U, V) as b, db.Server() as srv:
        db.fit_graph(a, 3, 1e-6)
        ra = db.fit_graph(a, 100, 1e-9)
        t = srv.submit(b, db.FIT, max_iterations=3)
        t.wait()
        t = srv.submit(b, db.FIT, max_iterations=100, epsilon=1e-9)
        r = t.wait()
        assert (r["iterations"], r["delta"]) == ra
        np.testing.assert_array_equal(bits(b.edge_dress), bits(a.edge_dress))
        before = b.edge_dress
        t = srv.submit(b, db.FIT, max_iterations=0)
        r = t.wait()
        assert r["status"] == 0 and r["iterations"] == 0
        np.testing.assert_array_equal(bits(b.edge_dress), bits(before))


def test_admission_budget():
    rng = np.random.default_rng(8)
    gs = [db.Graph(*rr_graph(rng, 800)) for _ in range(24)]
    sizes = [db.estimate(g, db.DELTA, 1)[0] for g in gs]
    budget = 4 * max(sizes)
    big_n, big_U, big_V = graphs.random_regular(1000, 12, seed=1)
    with db.Server(memory_budget_bytes=budget) as srv, db.Graph(big_n, big_U, big_V) as big:
        assert db.estimate(big, db.DELTA, 1)[0] > budget
        t_big = srv.submit(big, db.DELTA, 1)
        assert t_big.done and t_big.code == EBUDGET and t_big.result()["status"] == EBUDGET
        ts = [srv.submit(g, db.DELTA, 1) for g in gs]
        res = [t.wait(timeout_ms=600_000) for t in ts]
        st = srv.stats()
    assert all(r["status"] == 0 for r in res)
    assert st["peak_reserved_bytes"] <= budget
    assert st["max_in_service"] <= budget // min(sizes)
    assert st["max_in_service"] < len(gs)            # some requests had to wait
    assert max(r["queue_ms"] for r in res) > 0
    for g, r in zip(gs, res):
        flat, _, nsub, fits, _ = db.hist_requests([g], db.DELTA, 1)[0]
        np.testing.assert_array_equal(r["hist_flat"], flat)
        g.close()


def test_cancel_and_bad_requests():
    hub_n, hub_U, hub_V = graphs.chung_lu(400, 3000, 2.3, 200, seed=4)
    n, U, V = graphs.random_regular(50, 4, seed=3)
    with db.Graph(hub_n, hub_U, hub_V) as hub, db.Graph(n, U, V) as small:
        need = db.estimate(hub, db.DELTA, 1)[0]
        with db.Server(memory_budget_bytes=need + 1024) as srv:
            t1 = srv.submit(hub, db.DELTA, 1)          # holds the budget until it finishes
            t2 = srv.submit(small, db.DELTA, 1)        # waits for admission
            assert t2.cancel() == 0
            r2 = t2.wait()
            assert r2["status"] == ECANCELLED
            r1 = t1.wait()
            assert r1["status"] == 0
            st = srv.stats()
            assert st["cancelled"] == 1 and st["completed"] == 1
            # a malformed request is refused at submission and marked done
            req = db._abi.ServerRequest()
            req.kind = 9
            req.graph = small.ptr
            code = db.lib().dressx_server_submit(srv.handle, db.ctypes.byref(req))
            assert code == EINVAL and req.done == 1 and req.status == EINVAL


def test_served_large_histogram_equals_direct_call():
    """A served Delta^2 request whose one histogram (about 300 MB) a finisher
    copies out in parts across host threads: the same exact pairs as the
    direct call."""
    n, U, V = graphs.random_regular(200, 10, seed=4)
    with db.Graph(n, U, V) as g:
        direct = db.hist_requests([g], db.DELTA, 2)[0][0]
        with db.Server() as srv:
            r = srv.submit(g, db.DELTA, 2).wait(timeout_ms=600_000)
        assert r["status"] == 0
        np.testing.assert_array_equal(r["hist_flat"], direct)
        assert direct.size * 8 > 64 << 20
