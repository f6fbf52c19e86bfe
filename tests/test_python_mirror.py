"""Host-side pieces of the Python mirror, without a GPU: the packed view
over an array of request structs, and the zero-copy handover of malloc'd
histogram arrays (the library's own dressx_free releases them)."""
import ctypes

import numpy as np

import dress_b200 as db
from dress_b200 import _abi


def test_request_view_maps_every_field():
    reqs = (_abi.HistRequest * 3)()
    v = db._request_view(reqs)
    assert v.shape == (3,)
    v["graph"] = [0x1000, 0x2000, 0x3000]
    v["kind"] = db.NABLA
    v["k"] = 2
    v["max_iterations"] = 77
    v["epsilon"] = 1e-9
    v["seed"] = 0xFFFFFFFF
    v["offset"] = 5
    v["stride"] = 3
    v["want_histogram"] = 1
    v["hist_len"] = [4, 6, 8]
    for i, r in enumerate(reqs):
        assert ctypes.cast(r.graph, ctypes.c_void_p).value == 0x1000 * (i + 1)
        assert (r.kind, r.k, r.max_iterations, r.offset, r.stride) == (db.NABLA, 2, 77, 5, 3)
        assert r.epsilon == 1e-9 and r.seed == 0xFFFFFFFF and r.want_histogram == 1
        assert r.hist_len == 4 + 2 * i
    # and back: fields the library writes are read through the view
    reqs[1].fits = 12345
    reqs[2].status = 7
    assert v["fits"][1] == 12345 and v["status"][2] == 7


def _malloc_i64(values):
    a = np.asarray(values, dtype=np.int64)
    p = db._libc.malloc(a.nbytes)
    ctypes.memmove(p, a.ctypes.data, a.nbytes)
    return p


def test_take_i64_is_zero_copy_and_outlives_views():
    p = _malloc_i64(np.arange(10) * 3)
    arr = db._take_i64(p, 10)
    assert arr.dtype == np.int64 and arr.shape == (10,)
    assert arr.__array_interface__["data"][0] == p          # no copy
    np.testing.assert_array_equal(arr, np.arange(10) * 3)
    view = arr[3:6]
    del arr                                                 # the slice keeps the block alive
    np.testing.assert_array_equal(view, [9, 12, 15])
    del view


def test_take_i64_empty_and_null():
    assert db._take_i64(None, 5).size == 0
    p = _malloc_i64([1, 2])
    assert db._take_i64(p, 0).size == 0                     # freed at once
