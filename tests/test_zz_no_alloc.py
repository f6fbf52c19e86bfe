"""dressx_histogram_noalloc: the exact histogram for callers that cannot
allocate device memory.

Some callers cannot call cudaMalloc when they need a histogram -- code that
runs while a CUDA graph is being captured, frameworks whose caching allocator
owns all device memory, loops that must not allocate after start-up.  This
entry point takes values already in device memory and writes the
(value bits, count) pairs into caller-provided device memory, using only a
fixed scratch array compiled into the library.  Here it is called through the
C ABI twice in a row, on the converged values of two different Delta^1 runs,
and each result must equal, bit for bit, the histogram that the existing
entry point (dressx_hist_batch) returns for the same run.  The second call
also shows that nothing of the first call's data leaks into it.

This file is collected last so that a run that stops at the first failure
has already run every other test.
"""
import ctypes

import numpy as np
import pytest

import dress_b200 as db
from dress_b200 import _abi, graphs

pytestmark = pytest.mark.gpu


def _existing_histogram_and_values(n, U, V, W=None):
    """Histogram from dressx_hist_batch, plus the values it was built from
    (the live entries of the multiset rows)."""
    with db.Graph(n, U, V, W) as g:
        flat, ms, num, fits, status = db.hist_requests([g], db.DELTA, 1, keep_multisets=True)[0]
    values = ms[~np.isnan(ms)]
    assert values.size == int(flat.reshape(-1, 2)[:, 1].sum())
    return flat, values


def _noalloc(values):
    import torch
    dev = torch.device("cuda", 0)
    vals = torch.from_numpy(values.astype(np.float64)).to(dev)
    pairs = torch.full((2 * max(1, values.size),), -1, dtype=torch.int64, device=dev)
    runs = torch.full((1,), -1, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev)
    rc = db.lib().dressx_histogram_noalloc(ctypes.c_void_p(vals.data_ptr()), values.size,
                                           ctypes.c_void_p(pairs.data_ptr()), ctypes.c_void_p(runs.data_ptr()),
                                           ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0
    stream.synchronize()
    r = int(runs.item())
    return pairs[: 2 * r].cpu().numpy()


def test_noalloc_histogram_matches_existing_entry_point_twice():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    n1, U1, V1 = graphs.random_regular(60, 6, seed=21)
    W1 = graphs.uniform_weights(len(U1), seed=4)
    n2, U2, V2 = graphs.erdos_renyi(90, 400, seed=5)
    first_ref, first_vals = _existing_histogram_and_values(n1, U1, V1, W1)
    second_ref, second_vals = _existing_histogram_and_values(n2, U2, V2)
    assert first_vals.size > 8192 and second_vals.size > 8192      # several tiles each
    first = _noalloc(first_vals)
    second = _noalloc(second_vals)
    np.testing.assert_array_equal(first, first_ref)
    np.testing.assert_array_equal(second, second_ref)


def test_noalloc_rejects_sizes_beyond_the_maximum():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    dev = torch.device("cuda", 0)
    buf = torch.zeros(4, dtype=torch.float64, device=dev)
    out = torch.zeros(8, dtype=torch.int64, device=dev)
    runs = torch.full((1,), -7, dtype=torch.int64, device=dev)
    rc = db.lib().dressx_histogram_noalloc(ctypes.c_void_p(buf.data_ptr()), _abi.NOALLOC_MAX_VALUES + 1,
                                           ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(runs.data_ptr()),
                                           None)
    assert rc == 5                              # DRESSX_EUNSUPPORTED, nothing enqueued
    torch.cuda.synchronize()
    assert int(runs.item()) == -7
