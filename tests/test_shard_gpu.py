"""Strided shards of one Delta/Nabla request (offset = rank, stride = ranks,
the partition of the reference's MPI layer) merge to the unsharded
histogram, on the GPU engine."""
import numpy as np
import pytest

import dress_b200 as db
from dress_b200 import graphs, shard

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,k,world", [(db.DELTA, 1, 2), (db.DELTA, 2, 4), (db.NABLA, 1, 3), (db.DELTA, 1, 7)])
def test_strided_shards_merge_to_unsharded(kind, k, world):
    n, U, V = graphs.random_regular(40, 6, seed=9)
    W = graphs.uniform_weights(len(U), seed=4)
    with db.Graph(n, U, V, W) as g:
        full, _, nsub, fits, st = db.hist_requests([g], kind, k)[0]
        assert st == 0
        parts = [db.hist_requests([g], kind, k, offset=r, stride=world)[0] for r in range(world)]
    assert sum(p[3] for p in parts) == fits
    assert all(p[2] == nsub for p in parts)
    np.testing.assert_array_equal(shard.merge_hists([p[0] for p in parts]), full)


def test_strided_shards_match_oracle(oracle_port):
    n, U, V = graphs.random_regular(30, 4, seed=2)
    with db.Graph(n, U, V) as g:
        parts = [db.hist_requests([g], db.DELTA, 1, offset=r, stride=3)[0][0] for r in range(3)]
    for r in range(3):
        ref = oracle_port.delta_fit(n, U, V, k=1, offset=r, stride=3)["hist"]
        np.testing.assert_array_equal(parts[r], ref)
    np.testing.assert_array_equal(shard.merge_hists(parts), oracle_port.delta_fit(n, U, V, k=1)["hist"])
