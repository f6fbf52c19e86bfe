"""Sharded Delta/Nabla host logic without a GPU: the k-way merge of shard
histograms (dressx_hist_merge) and the all-gather of variable-length
histograms over two gloo ranks."""
import os
import socket
import tempfile

import numpy as np
import pytest

from dress_b200 import shard


def flat_of(values):
    """Exact histogram of doubles as flat [bits, count, ...], ascending."""
    v = np.asarray(values, dtype=np.float64)
    if v.size == 0:
        return np.zeros(0, dtype=np.int64)
    u, c = np.unique(v, return_counts=True)
    out = np.empty(2 * u.size, dtype=np.int64)
    out[0::2] = u.view(np.int64)
    out[1::2] = c
    return out


def shards_of(values, parts, rng):
    cut = np.sort(rng.integers(0, values.size + 1, parts - 1))
    return np.split(values, cut)


def test_merge_equals_histogram_of_the_union():
    rng = np.random.default_rng(1)
    for parts in (1, 2, 3, 7):
        values = rng.integers(0, 500, 20000) / 7.0 + 0.25        # many exact repeats
        values = rng.permutation(values)
        flats = [flat_of(s) for s in shards_of(values, parts, rng)]
        np.testing.assert_array_equal(shard.merge_hists(flats), flat_of(values))


def test_merge_of_empty_and_single_lists():
    assert shard.merge_hists([]).size == 0
    assert shard.merge_hists([np.zeros(0, np.int64)] * 3).size == 0
    f = flat_of([1.5, 1.5, 2.0])
    np.testing.assert_array_equal(shard.merge_hists([f]), f)
    np.testing.assert_array_equal(shard.merge_hists([f, np.zeros(0, np.int64), f]), flat_of([1.5] * 4 + [2.0] * 2))


def test_merge_rejects_malformed_lists():
    with pytest.raises(RuntimeError):
        shard.merge_hists([np.array([1, 2, 3], np.int64)])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, path, seed):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(seed)
        values = rng.integers(0, 300, 5000 * (rank + 1)) / 3.0     # shards of different sizes
        got = shard.gather_hists(flat_of(values))
        merged = shard.merge_hists(got)
        np.save(f"{path}.{rank}.npy", merged)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_and_merge():
    import torch.multiprocessing as mp
    world, seed = 2, 7
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "h")
        mp.spawn(_rank_main, args=(world, _free_port(), path, seed), nprocs=world, join=True)
        outs = [np.load(f"{path}.{r}.npy") for r in range(world)]
    rng_vals = []
    for r in range(world):
        rng = np.random.default_rng(seed)
        rng_vals.append(rng.integers(0, 300, 5000 * (r + 1)) / 3.0)
    expect = flat_of(np.concatenate(rng_vals))
    for o in outs:                       # every rank holds the same merged histogram
        np.testing.assert_array_equal(o, expect)


def test_merge_keys_by_bits():
    """Equal bit patterns merge; +0 and -0 stay two entries (-0 first), and
    every NaN is an entry of its own, as in the reference's map."""
    pz, nz = np.float64(0.0).view(np.int64), np.float64(-0.0).view(np.int64)
    nan = np.float64(np.nan).view(np.int64)
    a = np.array([nz, 2, pz, 3], np.int64)
    b = np.array([nz, 1, pz, 4, nan, 1], np.int64)
    got = shard.merge_hists([a, b])
    np.testing.assert_array_equal(got, np.array([nz, 3, pz, 7, nan, 1], np.int64))
    got = shard.merge_hists([b, b])
    np.testing.assert_array_equal(got, np.array([nz, 2, pz, 8, nan, 1, nan, 1], np.int64))
