"""Generates tests/golden/*.json.gz from the reference library itself.

Run where the reference sources are available (they are compiled unchanged
into oracle/_ref/libdress_ref.so by ``make -C oracle ref``):

    python tests/golden/make_golden.py

Cases: the topologies of the reference's own tests
(tests/c/cuda/test_dress_cuda.c:88-133, tests/python/test_dress_ab.py:78-176,
tests/c/test_delta_dress.c), every variant with and without intercepts, and
a few seeded random graphs.  Values are stored as int64 bit patterns so the
comparison is exact.
"""
import gzip
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "dress-graph_b200"))

import oracle  # noqa: E402
from dress_b200 import graphs  # noqa: E402

TOPOLOGIES = {
    "single_edge": (2, [0], [1], None),
    "triangle": (3, [0, 1, 0], [1, 2, 2], None),
    "triangle_w": (3, [0, 1, 0], [1, 2, 2], [1.0, 2.0, 3.0]),
    "path4": (4, [0, 1, 2], [1, 2, 3], None),
    "path4_w": (4, [0, 1, 2], [1, 2, 3], [0.5, 1.5, 2.5]),
    "k4": (4, [0, 0, 0, 1, 1, 2], [1, 2, 3, 2, 3, 3], None),
    "k4_w": (4, [0, 0, 0, 1, 1, 2], [1, 2, 3, 2, 3, 3], [1.0, 2.0, 3.0, 4.0, 5.0, 6.0]),
    "star5": (5, [0, 0, 0, 0], [1, 2, 3, 4], None),
    "cycle5": (5, [0, 1, 2, 3, 4], [1, 2, 3, 4, 0], None),
    "k5_minus_edge": (5, [0, 0, 0, 1, 1, 1, 2, 2, 3], [1, 2, 3, 2, 3, 4, 3, 4, 4], None),
    "house": (5, [0, 0, 1, 1, 2, 3], [1, 3, 2, 4, 3, 4], None),
    "weighted_star": (4, [0, 0, 0], [1, 2, 3], [1.0, 2.0, 3.0]),
    "two_triangles": (4, [0, 0, 1, 1, 2], [1, 2, 2, 3, 3], None),
    "disconnected": (4, [0, 2], [1, 3], None),
    "directed_reciprocal": (3, [0, 1, 1, 2], [1, 0, 2, 1], [3.0, 5.0, 1.0, 2.0]),
    "directed_cycle": (4, [0, 1, 2, 3], [1, 2, 3, 0], None),
    "petersen": (10, [0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9],
                 [1, 2, 3, 4, 0, 5, 6, 7, 8, 9, 7, 8, 9, 5, 6], None),
}


def long_parallel_runs():
    """Multigraphs whose rows hold long runs of parallel edges to one
    neighbour.  The reference sorts each row by neighbour id only
    (libdress/src/dress.c:25-30, 283-293) with the C library's qsort, so the
    order inside such a run -- which decides how the merge walk pairs
    parallel edges -- is the qsort's; these cases pin it (the C library the
    fixtures were made with is recorded in golden_meta.json)."""
    rng = np.random.default_rng(31)
    U = [0] * 40 + [1] * 25 + [0, 0, 1, 2, 3, 4] + [2] * 12
    V = [1] * 40 + [2] * 25 + [2, 3, 3, 3, 4, 0] + [4] * 12
    order = rng.permutation(len(U))                 # parallel edges listed out of order
    U = [U[i] for i in order]
    V = [V[i] for i in order]
    W = rng.uniform(0.5, 2.0, len(U)).round(6).tolist()
    return {"multi_long_runs": (5, U, V, None), "multi_long_runs_w": (5, U, V, W)}


def bits(a):
    return np.asarray(a, dtype=np.float64).view(np.int64).tolist()


def random_cases():
    out = {}
    n, U, V = graphs.erdos_renyi(60, 240, seed=11)
    out["er60"] = (n, U.tolist(), V.tolist(), None)
    out["er60_w"] = (n, U.tolist(), V.tolist(), graphs.uniform_weights(240, seed=3).tolist())
    n, U, V = graphs.random_regular(20, 4, seed=5)
    out["rr20_4"] = (n, U.tolist(), V.tolist(), None)
    n, U, V = graphs.chung_lu(300, 1200, 2.3, 60, seed=9)
    out["cl300"] = (n, U.tolist(), V.tolist(), None)
    return out


def main():
    ref = oracle.reference()
    if ref is None:
        raise SystemExit("build the reference first: make -C oracle ref")
    cases = dict(TOPOLOGIES)
    cases.update(random_cases())
    cases.update(long_parallel_runs())
    fits, hists = [], []
    for name, (n, U, V, W) in cases.items():
        for variant in range(4):
            for pre in (0, 1):
                for eps, it in ((1e-6, 100), (1e-15, 100), (1e-3, 5)):
                    r = ref.fit(n, U, V, W, variant=variant, precompute=pre, max_iterations=it, epsilon=eps)
                    fits.append(dict(name=name, N=n, U=list(map(int, U)), V=list(map(int, V)), W=W,
                                     variant=variant, precompute=pre, eps=eps, max_iterations=it,
                                     edge_dress=bits(r["edge_dress"]), vertex_dress=bits(r["vertex_dress"]),
                                     iterations=r["iterations"], delta=bits([r["delta"]])[0]))
        if n > 20 and name != "rr20_4":
            continue
        for kind in ("delta", "nabla"):
            for k in (0, 1, 2):
                for variant in (0, 1):
                    for (ns, seed, off, st) in ((0, 0, 0, 1), (0, 0, 1, 2), (3, 7, 0, 1)):
                        fn = ref.delta_fit if kind == "delta" else ref.nabla_fit
                        r = fn(n, U, V, W, k=k, n_samples=ns, seed=seed, offset=off, stride=st,
                               keep_multisets=True, variant=variant, max_iterations=100, epsilon=1e-6)
                        hists.append(dict(name=name, N=n, U=list(map(int, U)), V=list(map(int, V)), W=W,
                                          kind=kind, k=k, variant=variant, n_samples=ns, seed=seed,
                                          offset=off, stride=st, hist=r["hist"].tolist(), num=int(r["num"]),
                                          multisets=(bits(r["multisets"].ravel())
                                                     if r["multisets"] is not None and r["multisets"].size <= 4096
                                                     else None)))
    with gzip.open(os.path.join(HERE, "fit_cases.json.gz"), "wt") as f:
        json.dump(fits, f)
    with gzip.open(os.path.join(HERE, "hist_cases.json.gz"), "wt") as f:
        json.dump(hists, f)
    import platform
    with open(os.path.join(HERE, "golden_meta.json"), "w") as f:
        json.dump({"made_by": "the reference library compiled unchanged (oracle/_ref/libdress_ref.so)",
                   "libc": " ".join(platform.libc_ver()), "fit_cases": len(fits), "hist_cases": len(hists)},
                  f, indent=1)
    print(len(fits), "fit cases,", len(hists), "histogram cases")


if __name__ == "__main__":
    main()
