"""Host-side planning of served requests (no GPU): path choice and the
device bytes a request reserves at admission."""
import numpy as np

import dress_b200 as db
from dress_b200 import graphs

EINVAL = 1


def test_small_graphs_take_the_batch_path():
    n, U, V = graphs.random_regular(100, 6, seed=1)
    with db.Graph(n, U, V) as g:
        b_fit, p_fit = db.estimate(g, db.FIT)
        b_delta, p_delta = db.estimate(g, db.DELTA, 1)
        b_nabla, p_nabla = db.estimate(g, db.NABLA, 1)
    assert p_fit == p_delta == p_nabla == db.PATH_BATCH
    # a fit holds its graph and outputs; a Delta^1 request also its 100 x 300
    # subgraph values and their histogram scratch
    assert 0 < b_fit < b_delta
    assert b_delta >= 100 * 300 * 8 * 2
    assert b_nabla == b_delta


def test_hub_rows():
    # hub rows: the whole-graph fit runs on the single-graph engine (a warp or
    # a block per long row); the Delta^1 subgraphs are batched, their rows of
    # any length summed in the batch kernel
    n, U, V = graphs.chung_lu(2000, 6000, 2.3, 500, seed=2)
    with db.Graph(n, U, V) as g:
        assert max(np.diff(g.ptr.contents.adj_offset[: n + 1])) > 256
        assert db.estimate(g, db.FIT)[1] == db.PATH_LANE
        assert db.estimate(g, db.DELTA, 1)[1] == db.PATH_BATCH


def test_trivial_orders_take_a_lane():
    n, U, V = graphs.random_regular(40, 4, seed=3)
    with db.Graph(n, U, V) as g:
        assert db.estimate(g, db.DELTA, 0)[1] == db.PATH_LANE     # k = 0 fits in place
        assert db.estimate(g, db.DELTA, 40)[1] == db.PATH_LANE    # k >= N: empty histogram


def test_state_beyond_shared_memory_takes_a_lane():
    # 4-regular with 20000 edges: rows are short but one subgraph's state
    # (2 x 20000 edge values + norms) exceeds shared memory
    n, U, V = graphs.random_regular(10000, 4, seed=4)
    with db.Graph(n, U, V) as g:
        assert db.estimate(g, db.DELTA, 1)[1] == db.PATH_LANE


def test_larger_whole_graph_fits_take_a_lane():
    # 3000 edges: its Delta^1 subgraphs are batched, the whole-graph fit runs
    # on the single-graph engine, which spreads each sweep over the device
    n, U, V = graphs.random_regular(1000, 6, seed=4)
    with db.Graph(n, U, V) as g:
        assert db.estimate(g, db.FIT)[1] == db.PATH_LANE
        assert db.estimate(g, db.DELTA, 1)[1] == db.PATH_BATCH


def test_estimate_grows_with_the_graph():
    sizes = []
    for n in (50, 200, 800):
        nn, U, V = graphs.random_regular(n, 4, seed=5)
        with db.Graph(nn, U, V) as g:
            sizes.append(db.estimate(g, db.DELTA, 1)[0])
    assert sizes[0] < sizes[1] < sizes[2]


def test_malformed_requests_are_refused():
    n, U, V = graphs.random_regular(20, 4, seed=6)
    with db.Graph(n, U, V) as g:
        for kind, k in ((7, 0), (db.DELTA, -1)):
            try:
                db.estimate(g, kind, k)
            except db.DressError as e:
                assert e.code == EINVAL
            else:
                raise AssertionError("accepted a malformed request")
        g.ptr.contents.U[2] = 99         # endpoint out of range
        try:
            db.estimate(g, db.FIT)
        except db.DressError as e:
            assert e.code == EINVAL
        else:
            raise AssertionError("accepted an out-of-range endpoint")
        g.ptr.contents.U[2] = U[2]
