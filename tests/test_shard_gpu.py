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


def _fit_rank(rank, world, port, path, kind, k):
    """One rank of shard.fit_sharded: its stride on cuda:0 through the
    engine, the histograms all-gathered over gloo and merged."""
    import os
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.cuda.set_device(0)
        n, U, V = graphs.random_regular(36, 6, seed=12)
        with db.Graph(n, U, V) as g:
            merged, nsub, fits = shard.fit_sharded(g, kind, k)
        np.save(f"{path}.{rank}.npy", np.concatenate([[nsub, fits], merged]).astype(np.int64))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind,k", [(db.DELTA, 1), (db.NABLA, 1)])
def test_fit_sharded_two_ranks(oracle_port, kind, k):
    """shard.fit_sharded end to end: two processes (gloo ranks) each run
    their stride through the engine on the same GPU (no kernel of one waits
    on the other), all-gather and merge; every rank's merged histogram is
    the oracle's unsharded one."""
    import os
    import socket
    import tempfile
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    world = 2
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "h")
        mp.spawn(_fit_rank, args=(world, port, path, kind, k), nprocs=world, join=True)
        outs = [np.load(f"{path}.{r}.npy") for r in range(world)]
    n, U, V = graphs.random_regular(36, 6, seed=12)
    fn = oracle_port.delta_fit if kind == db.DELTA else oracle_port.nabla_fit
    ref = fn(n, U, V, k=k)
    for o in outs:
        assert o[0] == ref["num"]
        assert o[1] == ref["num"]                  # every subgraph of a regular graph has edges
        np.testing.assert_array_equal(o[2:], ref["hist"])
