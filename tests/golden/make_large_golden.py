"""Golden digests of the single large fit, made by the reference library.

Graph: the Chung-Lu power-law graph of the single-fit workload -- 4,000,000
vertices, 28,000,000 undirected edges, degree exponent 2.3, degree cap 20,000,
dress_b200.graphs.chung_lu(..., seed=42) -- weighted with
dress_b200.graphs.uniform_weights(E, seed=7) (U[0.5, 2.0]) and unweighted.

For each variant this runs the reference's own dress_fit_omp (libdress
compiled unchanged into oracle/_ref/libdress_ref.so) twice:
  * the full fit (max 100 sweeps, epsilon 1e-6): iteration count, final
    delta bits and SHA-256 digests of the edge_dress and vertex_dress bytes;
  * three sweeps with epsilon 0: the same digests, a cheaper check.
The digests of the generated U, V, W arrays are stored too, so a check on
another machine knows it regenerated the same graph.  Output:
tests/golden/large_fit.json.  Runs for about 25 minutes on 8 cores.

    python tests/golden/make_large_golden.py
"""
import ctypes
import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
for p in (ROOT, os.path.join(ROOT, "dress-graph_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

from dress_b200 import graphs  # noqa: E402
import oracle  # noqa: E402


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def workload(edges=28_000_000):
    n = 4_000_000 * edges // 28_000_000
    n, U, V = graphs.chung_lu(n, edges, 2.3, 20000, seed=42)
    return n, U, V, graphs.uniform_weights(len(U), seed=7)


def main():
    ref = oracle.reference()
    if ref is None:
        raise SystemExit("oracle/_ref/libdress_ref.so is not built (make -C oracle ref)")
    t0 = time.time()
    n, U, V, W = workload()
    out = {"graph": {"N": int(n), "E": int(len(U)), "sha_U": sha(U), "sha_V": sha(V), "sha_W": sha(W)},
           "generator": "dress_b200.graphs.chung_lu(4000000, 28000000, 2.3, 20000, seed=42); "
                        "uniform_weights(E, seed=7)",
           "made_by": "the reference's dress_fit_omp, libdress compiled unchanged (oracle/_ref)"}
    print(f"graph generated in {time.time() - t0:.0f} s", flush=True)
    for label, w in (("weighted", W), ("unweighted", None)):
        res = {}
        for run, (max_it, eps) in (("three_sweeps", (3, 0.0)), ("full", (100, 1e-6))):
            t1 = time.time()
            r = ref.fit(n, U, V, w, max_iterations=max_it, epsilon=eps, omp=True)
            res[run] = {"max_iterations": max_it, "epsilon": eps, "iterations": int(r["iterations"]),
                        "delta_bits": int(np.float64(r["delta"]).view(np.int64)),
                        "sha_edge_dress": sha(r["edge_dress"]), "sha_vertex_dress": sha(r["vertex_dress"]),
                        "seconds": round(time.time() - t1, 1)}
            print(label, run, res[run], flush=True)
        out[label] = res
    with open(os.path.join(ROOT, "tests", "golden", "large_fit.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
