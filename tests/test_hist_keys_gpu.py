"""Histogram keys on the GPU: a run is one bit pattern.

The reference's map (libdress/src/dress_histogram.c:10-19, 40-60) hashes the
bit pattern of a value and merges by ==, so equal bit patterns always merge,
+0 and -0 (==-equal, different bits) land in different slots, and a NaN never
equals an entry.  The device histogram keeps +0 and -0 as two entries (-0
first) and every NaN apart; values are ascending, NaNs at the ends by bits.
"""
import ctypes

import numpy as np
import pytest

import dress_b200 as db

pytestmark = pytest.mark.gpu


def expected(values):
    k = values.view(np.uint64)
    order_key = np.where(k >> np.uint64(63) == 1, ~k, k | np.uint64(1 << 63))
    v = values[np.argsort(order_key, kind="stable")]
    out = []
    for x in v:
        b = int(np.float64(x).view(np.int64))
        if out and out[-2] == b and not np.isnan(x):
            out[-1] += 1
        else:
            out += [b, 1]
    return np.array(out, np.int64)


def test_signed_zeros_and_nans():
    import torch
    rng = np.random.default_rng(4)
    base = np.array([0.0, -0.0, 1.5, -2.0, np.inf, -np.inf, np.nan, 0.0, -0.0, 1.5, np.nan], np.float64)
    values = rng.permutation(np.concatenate([base, rng.choice(base[:6], 5000)]))
    dev = torch.device("cuda", 0)
    vals = torch.from_numpy(values).to(dev)
    pairs = torch.full((2 * values.size,), -1, dtype=torch.int64, device=dev)
    runs = torch.full((1,), -1, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev)
    rc = db.lib().dressx_histogram_noalloc(ctypes.c_void_p(vals.data_ptr()), values.size,
                                           ctypes.c_void_p(pairs.data_ptr()), ctypes.c_void_p(runs.data_ptr()),
                                           ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0
    stream.synchronize()
    r = int(runs.item())
    got = pairs[: 2 * r].cpu().numpy()
    np.testing.assert_array_equal(got, expected(values))
    zeros = got.reshape(-1, 2)
    assert np.float64(-0.0).view(np.int64) in zeros[:, 0] and np.float64(0.0).view(np.int64) in zeros[:, 0]
