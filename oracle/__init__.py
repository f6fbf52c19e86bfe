"""CPU oracle of the B200 DRESS engine's parity tests (test infrastructure only).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package.  It wraps two CPU implementations behind
one interface:

* ``kind="port"``       -- ``liboracle.so``, the plain-C restatement in
  ``dress_oracle.c`` (always built);
* ``kind="reference"``  -- ``_ref/libdress_ref.so``, libdress's own C sources
  (``libdress/src/dress.c`` etc.) compiled unchanged; present only where the
  reference sources were available at build time.

Both operate on the reference's ``dress_graph_t`` layout
(``libdress/include/dress/dress.h:43-75``).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libdress_ref.so")

UNDIRECTED, DIRECTED, FORWARD, BACKWARD = 0, 1, 2, 3

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_dbl_p = ctypes.POINTER(ctypes.c_double)


class Graph(ctypes.Structure):
    _fields_ = [
        ("variant", ctypes.c_int), ("N", ctypes.c_int), ("E", ctypes.c_int),
        ("U", _c_int_p), ("V", _c_int_p),
        ("adj_offset", _c_int_p), ("adj_target", _c_int_p), ("adj_edge_idx", _c_int_p),
        ("max_degree", ctypes.c_int),
        ("W", _c_dbl_p), ("edge_weight", _c_dbl_p), ("edge_dress", _c_dbl_p),
        ("edge_dress_next", _c_dbl_p), ("NW", _c_dbl_p), ("vertex_dress", _c_dbl_p),
        ("precompute_intercepts", ctypes.c_int),
        ("intercept_offset", _c_int_p), ("intercept_edge_ux", _c_int_p),
        ("intercept_edge_vx", _c_int_p),
    ]


PGraph = ctypes.POINTER(Graph)
_libc = ctypes.CDLL(None)
_libc.malloc.restype = ctypes.c_void_p
_libc.malloc.argtypes = [ctypes.c_size_t]
_libc.free.argtypes = [ctypes.c_void_p]


def _malloc_copy(arr, ctype):
    arr = np.ascontiguousarray(arr)
    n = max(1, arr.size)
    raw = _libc.malloc(n * ctypes.sizeof(ctype))
    if not raw:
        raise MemoryError("malloc failed")
    ctypes.memmove(raw, arr.ctypes.data, arr.nbytes)
    return ctypes.cast(raw, ctypes.POINTER(ctype))


def _arr(ptr, n, dtype):
    if n <= 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


def flat_to_pairs(flat):
    """[bits, count, ...] int64 -> (values float64, counts int64)."""
    flat = np.asarray(flat, dtype=np.int64).reshape(-1, 2)
    return flat[:, 0].copy().view(np.float64), flat[:, 1].copy()


class CpuDress:
    """One CPU implementation (``port`` or ``reference``)."""

    def __init__(self, kind="port"):
        self.kind = kind
        path = PORT_SO if kind == "port" else REF_SO
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        lib = ctypes.CDLL(path)
        p = "oracle_" if kind == "port" else "dress_"
        self.init_graph = getattr(lib, p + "init_graph")
        self.free_graph = getattr(lib, p + "free_graph")
        self.fit_fn = getattr(lib, p + "fit")
        self.delta_fn = getattr(lib, "oracle_delta_fit_flat" if kind == "port"
                                else "dress_delta_fit_strided_flat")
        self.nabla_fn = getattr(lib, "oracle_nabla_fit_flat" if kind == "port"
                                else "dress_nabla_fit_strided_flat")
        self.init_graph.restype = PGraph
        self.init_graph.argtypes = [ctypes.c_int, ctypes.c_int, _c_int_p, _c_int_p,
                                    _c_dbl_p, _c_dbl_p, ctypes.c_int, ctypes.c_int]
        self.free_graph.argtypes = [PGraph]
        self.fit_fn.argtypes = [PGraph, ctypes.c_int, ctypes.c_double,
                                _c_int_p, _c_dbl_p]
        hist_args = [PGraph, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                     ctypes.c_int, ctypes.c_uint, _c_int_p, ctypes.c_int,
                     ctypes.POINTER(_c_dbl_p), ctypes.POINTER(ctypes.c_int64),
                     ctypes.c_int, ctypes.c_int]
        for f in (self.delta_fn, self.nabla_fn):
            f.restype = ctypes.POINTER(ctypes.c_int64)
            f.argtypes = hist_args
        self.get_fn = getattr(lib, p + "get")
        self.get_fn.restype = ctypes.c_double
        self.get_fn.argtypes = [PGraph, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        self.lib = lib
        if kind == "reference":
            self.fit_omp = lib.dress_fit_omp
            self.fit_omp.argtypes = self.fit_fn.argtypes
            self.delta_omp = lib.dress_delta_fit_omp_strided_flat
            self.delta_omp.restype = ctypes.POINTER(ctypes.c_int64)
            self.delta_omp.argtypes = hist_args
            self.nabla_omp = lib.dress_nabla_fit_omp_strided_flat
            self.nabla_omp.restype = ctypes.POINTER(ctypes.c_int64)
            self.nabla_omp.argtypes = hist_args

    # -- graph life cycle -------------------------------------------------
    def build(self, N, U, V, W=None, NW=None, variant=UNDIRECTED, precompute=0):
        U = np.asarray(U, dtype=np.int32)
        V = np.asarray(V, dtype=np.int32)
        pW = _malloc_copy(np.asarray(W, dtype=np.float64), ctypes.c_double) if W is not None else None
        pNW = _malloc_copy(np.asarray(NW, dtype=np.float64), ctypes.c_double) if NW is not None else None
        return self.init_graph(int(N), int(U.size), _malloc_copy(U, ctypes.c_int),
                               _malloc_copy(V, ctypes.c_int), pW, pNW,
                               int(variant), int(precompute))

    @staticmethod
    def csr(g):
        c = g.contents
        S = c.adj_offset[c.N]
        out = dict(adj_offset=_arr(c.adj_offset, c.N + 1, np.int32),
                   adj_target=_arr(c.adj_target, S, np.int32),
                   adj_edge_idx=_arr(c.adj_edge_idx, S, np.int32),
                   edge_weight=_arr(c.edge_weight, c.E, np.float64),
                   max_degree=c.max_degree)
        if c.precompute_intercepts:
            T = c.intercept_offset[c.E]
            out.update(intercept_offset=_arr(c.intercept_offset, c.E + 1, np.int32),
                       intercept_edge_ux=_arr(c.intercept_edge_ux, T, np.int32),
                       intercept_edge_vx=_arr(c.intercept_edge_vx, T, np.int32))
        return out

    # -- fit ----------------------------------------------------------------
    def fit(self, N, U, V, W=None, NW=None, variant=UNDIRECTED, precompute=0,
            max_iterations=100, epsilon=1e-6, omp=False):
        g = self.build(N, U, V, W, NW, variant, precompute)
        it, dl = ctypes.c_int(-1), ctypes.c_double(-1.0)
        (self.fit_omp if omp else self.fit_fn)(g, int(max_iterations), float(epsilon),
                                               ctypes.byref(it), ctypes.byref(dl))
        c = g.contents
        res = dict(edge_dress=_arr(c.edge_dress, c.E, np.float64),
                   vertex_dress=_arr(c.vertex_dress, c.N, np.float64),
                   iterations=it.value, delta=dl.value)
        self.free_graph(g)
        return res

    # -- virtual-edge queries -------------------------------------------------
    def get_many(self, N, U, V, W, queries, max_iterations=100, epsilon=1e-6, edge_weight=1.0,
                 NW=None, variant=UNDIRECTED, fit_iterations=100, fit_epsilon=1e-6):
        """Fit the graph, then dress_get for every (u, v) in queries."""
        g = self.build(N, U, V, W, NW, variant, 0)
        it, dl = ctypes.c_int(-1), ctypes.c_double(-1.0)
        self.fit_fn(g, int(fit_iterations), float(fit_epsilon), ctypes.byref(it), ctypes.byref(dl))
        out = np.array([self.get_fn(g, int(u), int(v), int(max_iterations), float(epsilon), float(edge_weight))
                        for u, v in queries], dtype=np.float64)
        self.free_graph(g)
        return out

    # -- Delta / Nabla --------------------------------------------------------
    def _hist(self, fn, N, U, V, W, NW, variant, k, max_iterations, epsilon,
              n_samples, seed, keep_multisets, offset, stride, precompute):
        g = self.build(N, U, V, W, NW, variant, precompute)
        hs = ctypes.c_int(0)
        ns = ctypes.c_int64(0)
        ms = _c_dbl_p()
        flat = fn(g, int(k), int(max_iterations), float(epsilon), int(n_samples),
                  ctypes.c_uint(seed), ctypes.byref(hs), 1 if keep_multisets else 0,
                  ctypes.byref(ms), ctypes.byref(ns), int(offset), int(stride))
        E = g.contents.E
        hist = _arr(flat, hs.value, np.int64)
        if flat:
            _libc.free(ctypes.cast(flat, ctypes.c_void_p))
        multisets = None
        if keep_multisets and ms:
            multisets = _arr(ms, ns.value * E, np.float64).reshape(ns.value, E)
            _libc.free(ctypes.cast(ms, ctypes.c_void_p))
        self.free_graph(g)
        return dict(hist=hist, num=ns.value, multisets=multisets)

    def delta_fit(self, N, U, V, W=None, k=1, max_iterations=100, epsilon=1e-6,
                  n_samples=0, seed=0, keep_multisets=False, offset=0, stride=1,
                  variant=UNDIRECTED, NW=None, precompute=0, omp=False):
        fn = self.delta_omp if omp else self.delta_fn
        return self._hist(fn, N, U, V, W, NW, variant, k, max_iterations, epsilon,
                          n_samples, seed, keep_multisets, offset, stride, precompute)

    def nabla_fit(self, N, U, V, W=None, k=1, max_iterations=100, epsilon=1e-6,
                  n_samples=0, seed=0, keep_multisets=False, offset=0, stride=1,
                  variant=UNDIRECTED, NW=None, precompute=0, omp=False):
        fn = self.nabla_omp if omp else self.nabla_fn
        return self._hist(fn, N, U, V, W, NW, variant, k, max_iterations, epsilon,
                          n_samples, seed, keep_multisets, offset, stride, precompute)


def port():
    return CpuDress("port")


def reference():
    """The reference library, or None where it was not built."""
    return CpuDress("reference") if os.path.exists(REF_SO) else None
