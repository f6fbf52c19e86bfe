"""The reference's own callers of the CUDA entry points, unmodified, against
this library:

* tests/c/cuda/test_dress_cuda.c -- the reference's CPU-vs-GPU fit test
  (15 cases, tolerance 1e-12), compiled from the reference sources by
  oracle/Makefile (target ref-tests) and linked against libdress_cuda.so
  (its CPU side against the reference library);
* python/src/dress/cuda -- the reference's Python binding.  It loads
  ``libdress_cuda.so`` through ctypes (its fallback to the loader path,
  python/src/dress/cuda/__init__.py:118-130), so it runs here with this
  library's directory on LD_LIBRARY_PATH.  The package is the reference's
  own install (pip --target baseline/_ref); the test skips where it is
  absent.  Its fit, delta_fit and nabla_fit must give the oracle's bits.
"""
import json
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from dress_b200 import graphs

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "dress-graph_b200", "lib")
REF_PY = os.path.join(ROOT, "baseline", "_ref")


def test_reference_cuda_test_binary():
    exe = os.path.join(ROOT, "oracle", "_ref", "test_dress_cuda")
    if not os.path.exists(exe):
        pytest.skip("reference CUDA test not built")
    # The test's graph copies leave NW and max_degree uninitialised
    # (tests/c/cuda/test_dress_cuda.c:25-86) and the reference's
    # dress_free_graph frees NW (libdress/src/dress.c:630): with stale heap
    # contents the binary aborts in malloc even when dress_fit_cuda does
    # nothing.  MALLOC_PERTURB_=255 makes glibc fill new allocations with
    # zeros, and the tcache (whose fast path skips that fill) is turned off,
    # so NW reads as NULL -- the unit vertex weights the test means.
    env = dict(os.environ, MALLOC_PERTURB_="255", GLIBC_TUNABLES="glibc.malloc.tcache_count=0")
    out = subprocess.run([exe], capture_output=True, text=True, timeout=600, env=env)
    text = out.stdout + out.stderr
    assert out.returncode == 0, text[-4000:]
    assert "ALL TESTS PASSED" in text, text[-4000:]
    # beyond its 1e-12 bar: identical iteration counts and zero differences
    rows = re.findall(r"iters=(\d+)/(\d+)\s+edge_diff=(\S+)\s+node_diff=(\S+)", text)
    assert len(rows) >= 15, text[-4000:]
    for it_cpu, it_gpu, de, dn in rows:
        assert it_cpu == it_gpu and float(de) == 0.0 and float(dn) == 0.0, text[-4000:]


CALLER = r"""
import json, sys
import numpy as np
from dress import cuda
spec = json.loads(sys.stdin.read())
out = {}
n, U, V, W = spec["n"], spec["U"], spec["V"], spec["W"]
r = cuda.fit(n, U, V, weights=W, epsilon=1e-6)
out["fit"] = dict(edge=np.asarray(r.edge_dress, np.float64).view(np.int64).tolist(),
                  vertex=np.asarray(r.vertex_dress, np.float64).view(np.int64).tolist(),
                  iterations=int(r.iterations))
for name, fn in (("delta", cuda.delta_fit), ("nabla", cuda.nabla_fit)):
    h = fn(n, U, V, weights=W, k=1, epsilon=1e-6).histogram
    vals = np.asarray([v for v, c in h], np.float64).view(np.int64).tolist()
    out[name] = dict(values=vals, counts=[int(c) for v, c in h])
print(json.dumps(out))
"""


def test_reference_python_binding(oracle_port):
    if not os.path.isdir(os.path.join(REF_PY, "dress", "cuda")):
        pytest.skip("the reference's Python package is not installed in baseline/_ref")
    n, U, V = graphs.erdos_renyi(40, 120, seed=5)
    W = graphs.uniform_weights(len(U), seed=6)
    env = dict(os.environ)
    env["PYTHONPATH"] = REF_PY
    env["LD_LIBRARY_PATH"] = LIBDIR + (":" + env["LD_LIBRARY_PATH"] if env.get("LD_LIBRARY_PATH") else "")
    spec = json.dumps(dict(n=n, U=U.tolist(), V=V.tolist(), W=W.tolist()))
    out = subprocess.run([sys.executable, "-c", CALLER], input=spec, capture_output=True, text=True,
                         env=env, cwd=ROOT, timeout=600)
    assert out.returncode == 0, out.stderr[-4000:]
    got = json.loads(out.stdout.strip().splitlines()[-1])
    ref = oracle_port.fit(n, U, V, W)
    assert got["fit"]["iterations"] == ref["iterations"]
    np.testing.assert_array_equal(np.asarray(got["fit"]["edge"], np.int64), ref["edge_dress"].view(np.int64))
    np.testing.assert_array_equal(np.asarray(got["fit"]["vertex"], np.int64), ref["vertex_dress"].view(np.int64))
    for name, fn in (("delta", oracle_port.delta_fit), ("nabla", oracle_port.nabla_fit)):
        flat = fn(n, U, V, W, k=1)["hist"].reshape(-1, 2)
        np.testing.assert_array_equal(np.asarray(got[name]["values"], np.int64), flat[:, 0])
        np.testing.assert_array_equal(np.asarray(got[name]["counts"], np.int64), flat[:, 1])
