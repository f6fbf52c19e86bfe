"""B200 DRESS engine -- Python mirror of the reference's ``dress.cuda`` API.

Same entry points, argument names, defaults and result fields as
``python/src/dress/cuda/__init__.py`` of the reference (``fit`` :451,
``delta_fit`` :497, ``nabla_fit`` :370, ``dress_cuda`` :239,
``dress_fit_cuda`` :306), all running through ``libdress_cuda.so``'s C ABI.
``delta_fit_many`` / ``nabla_fit_many`` add what the reference cannot do:
many graphs' histograms in one persistent launch.
"""
import ctypes
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

from . import _abi

UNDIRECTED, DIRECTED, FORWARD, BACKWARD = 0, 1, 2, 3
DELTA, NABLA = 0, 1

_libc = ctypes.CDLL(None)
_libc.malloc.restype = ctypes.c_void_p
_libc.malloc.argtypes = [ctypes.c_size_t]
_libc.free.argtypes = [ctypes.c_void_p]


class DressError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"dress_b200 error {code}: {msg}")
        self.code = code


def lib():
    return _abi.load()


def is_available():
    """True when the engine library loads and a CUDA device is visible."""
    try:
        lib()
    except (RuntimeError, OSError):
        return False
    try:
        import torch
        return torch.cuda.is_available()
    except ImportError:
        return True


def _malloc_copy(arr, ctype):
    arr = np.ascontiguousarray(arr)
    raw = _libc.malloc(max(1, arr.nbytes))
    if not raw:
        raise MemoryError("malloc failed")
    if arr.nbytes:
        ctypes.memmove(raw, arr.ctypes.data, arr.nbytes)
    return ctypes.cast(raw, ctypes.POINTER(ctype))


class _Block:
    """A malloc'd int64 array handed over by the library: numpy reads it in
    place through the array interface, and the block is released with
    dressx_free when the last array over it goes away."""

    __slots__ = ("addr", "n", "free")

    def __init__(self, addr, n, free):
        self.addr, self.n, self.free = addr, n, free

    @property
    def __array_interface__(self):
        return {"shape": (self.n,), "typestr": "<i8", "data": (self.addr, False), "version": 3}

    def __del__(self):
        self.free(self.addr)


def _take_i64(ptr, n):
    """A malloc'd int64 array from the library as numpy, without a copy; the
    memory is released with dressx_free once no array refers to it."""
    if not ptr:
        return np.zeros(0, dtype=np.int64)
    addr = ptr if isinstance(ptr, int) else ctypes.cast(ptr, ctypes.c_void_p).value
    if n <= 0:
        lib().dressx_free(addr)
        return np.zeros(0, dtype=np.int64)
    return np.asarray(_Block(addr, int(n), lib().dressx_free))


def _request_view(reqs):
    """The request array as a numpy record array over the same memory, for
    filling and reading many requests at once."""
    T = _abi.HistRequest
    ptr_fields = {"graph", "hist_flat", "multisets"}
    names, formats, offsets = [], [], []
    for name, ctype in T._fields_:
        names.append(name)
        formats.append(np.uintp if name in ptr_fields else np.dtype(ctype))
        offsets.append(getattr(T, name).offset)
    dt = np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": ctypes.sizeof(T)})
    raw = (ctypes.c_char * ctypes.sizeof(reqs)).from_buffer(reqs)
    return np.frombuffer(raw, dtype=dt)


def _arr(ptr, n, dtype):
    if n <= 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


class Graph:
    """Owns one ``dress_graph_t`` built by the library's ``dress_init_graph``."""

    def __init__(self, n_vertices, sources, targets, weights=None, vertex_weights=None,
                 variant=UNDIRECTED, precompute_intercepts=False, device_build=False):
        U = np.asarray(sources, dtype=np.int32)
        V = np.asarray(targets, dtype=np.int32)
        if U.shape != V.shape:
            raise ValueError("sources and targets differ in length")
        pW = _malloc_copy(np.asarray(weights, dtype=np.float64), ctypes.c_double) if weights is not None else None
        pNW = (_malloc_copy(np.asarray(vertex_weights, dtype=np.float64), ctypes.c_double)
               if vertex_weights is not None else None)
        init = lib().dressx_init_graph if device_build else lib().dress_init_graph
        pU, pV = _malloc_copy(U, ctypes.c_int), _malloc_copy(V, ctypes.c_int)
        self.ptr = init(int(n_vertices), int(U.size), pU, pV, pW, pNW, int(variant), int(bool(precompute_intercepts)))
        if not self.ptr:                      # the arrays stay ours on failure
            for p in (pU, pV, pW, pNW):
                if p:
                    _libc.free(ctypes.cast(p, ctypes.c_void_p))
        if not self.ptr:
            raise ValueError("dress_init_graph rejected the graph (vertex id out of range?)")
        self.addr = ctypes.cast(self.ptr, ctypes.c_void_p).value     # for packed request arrays
        self.N = int(n_vertices)
        self.E = int(U.size)

    @property
    def edge_dress(self):
        return _arr(self.ptr.contents.edge_dress, self.E, np.float64)

    @property
    def vertex_dress(self):
        return _arr(self.ptr.contents.vertex_dress, self.N, np.float64)

    @property
    def edge_weight(self):
        return _arr(self.ptr.contents.edge_weight, self.E, np.float64)

    def close(self):
        if self.ptr:
            lib().dress_free_graph(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


@dataclass
class DRESSResult:
    sources: list
    targets: list
    edge_dress: list
    edge_weight: list
    vertex_dress: list
    iterations: int
    delta: float


@dataclass
class DeltaDRESSResult:
    histogram: List[Tuple[float, int]]
    multisets: Optional[np.ndarray] = None
    num_subgraphs: int = 0
    flat: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=np.int64))


@dataclass
class NablaDRESSResult:
    histogram: List[Tuple[float, int]]
    multisets: Optional[np.ndarray] = None
    num_tuples: int = 0
    flat: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=np.int64))


def _check(code):
    if code != 0:
        c, msg = _abi.last_error()
        raise DressError(code, msg)


def fit_graph(g: Graph, max_iterations=100, epsilon=1e-6):
    """GPU fit of an existing graph in place; returns (iterations, delta)."""
    it, dl = ctypes.c_int(0), ctypes.c_double(0.0)
    _check(lib().dressx_fit(g.ptr, int(max_iterations), float(epsilon), ctypes.byref(it), ctypes.byref(dl)))
    return it.value, dl.value


def get(g: Graph, u, v, max_iterations=100, epsilon=1e-6, edge_weight=1.0):
    """Virtual-edge values for the vertex pairs (u[i], v[i]) of a fitted graph
    (the reference's dress_get, many pairs in one call).  edge_weight is a
    scalar or one weight per pair."""
    u = np.ascontiguousarray(u, dtype=np.int32)
    v = np.ascontiguousarray(v, dtype=np.int32)
    if u.shape != v.shape:
        raise ValueError("u and v differ in length")
    out = np.empty(u.size, dtype=np.float64)
    ew = None
    ew0 = 1.0
    if np.ndim(edge_weight) == 0:
        ew0 = float(edge_weight)
    else:
        ew = np.ascontiguousarray(edge_weight, dtype=np.float64)
        if ew.shape != u.shape:
            raise ValueError("one edge weight per pair")
    ip = ctypes.POINTER(ctypes.c_int)
    dp = ctypes.POINTER(ctypes.c_double)
    _check(lib().dressx_get_batch(g.ptr, u.ctypes.data_as(ip), v.ctypes.data_as(ip), u.size, int(max_iterations),
                                  float(epsilon), ew.ctypes.data_as(dp) if ew is not None else None, ew0,
                                  out.ctypes.data_as(dp)))
    return out


def last_fit_stats():
    st = _abi.FitStats()
    lib().dressx_last_fit_stats(ctypes.byref(st))
    return dict(common_terms=st.common_terms, sweeps=st.sweeps, setup_ms=st.setup_ms, iterate_ms=st.iterate_ms,
                vertex_bins=list(zip(st.vertex_bin_items, st.vertex_bin_terms)),
                edge_bins=list(zip(st.edge_bin_items, st.edge_bin_terms)),
                phases_ms=dict(zip(("upload", "validate", "pairs_and_bins", "renumber", "download"), st.phase_ms)))


def dress_cuda(N, E, U, V, W=None, NW=None, variant=UNDIRECTED, precompute_intercepts=0,
               max_iterations=100, epsilon=1e-10):
    """(edge_dress, vertex_dress, edge_weight, iterations, delta) -- reference
    ``python/src/dress/cuda/__init__.py:239-303``."""
    with Graph(N, list(U)[:E] if not isinstance(U, np.ndarray) else U[:E],
               list(V)[:E] if not isinstance(V, np.ndarray) else V[:E], W, NW, variant,
               precompute_intercepts) as g:
        it, dl = fit_graph(g, max_iterations, epsilon)
        return g.edge_dress, g.vertex_dress, g.edge_weight, it, dl


def dress_fit_cuda(g_ptr, max_iterations=100, epsilon=1e-10):
    """Fit a raw ``dress_graph_t`` pointer (reference :306-326)."""
    it, dl = ctypes.c_int(0), ctypes.c_double(0.0)
    lib().dress_fit_cuda(g_ptr, int(max_iterations), float(epsilon), ctypes.byref(it), ctypes.byref(dl))
    return it.value, dl.value


def fit(n_vertices, sources, targets, weights=None, vertex_weights=None, variant=UNDIRECTED,
        max_iterations=100, epsilon=1e-6, precompute_intercepts=False):
    """GPU DRESS fit -- reference ``dress.cuda.fit`` (:451-494)."""
    src, tgt = list(sources), list(targets)
    with Graph(n_vertices, src, tgt, weights, vertex_weights, variant, precompute_intercepts) as g:
        it, dl = fit_graph(g, max_iterations, epsilon)
        return DRESSResult(sources=src, targets=tgt, edge_dress=g.edge_dress.tolist(),
                           edge_weight=g.edge_weight.tolist(), vertex_dress=g.vertex_dress.tolist(),
                           iterations=it, delta=dl)


def _flat_to_list(flat):
    if flat.size == 0:
        return []
    f = flat.reshape(-1, 2)
    vals = f[:, 0].copy().view(np.float64)
    return [(float(v), int(c)) for v, c in zip(vals, f[:, 1])]


def hist_requests(graphs, kind, k, max_iterations=100, epsilon=1e-6, n_samples=0, seed=0,
                  keep_multisets=False, offset=0, stride=1, compute_histogram=True, per_fit=False):
    """Run one Delta/Nabla request per graph in a single engine call.

    Returns a list of (flat int64 [bits, count, ...], multisets or None,
    num_subgraphs, fits)."""
    n = len(graphs)
    reqs = (_abi.HistRequest * n)()
    v = _request_view(reqs)
    v["graph"] = [g.addr for g in graphs]
    v["kind"] = int(kind)
    v["k"] = int(k)
    v["max_iterations"] = int(max_iterations)
    v["epsilon"] = float(epsilon)
    v["n_samples"] = int(n_samples)
    v["seed"] = int(seed) & 0xFFFFFFFF
    v["offset"] = int(offset)
    v["stride"] = int(stride)
    v["want_histogram"] = 1 if compute_histogram else 0
    v["keep_multisets"] = 1 if keep_multisets else 0
    fn = lib().dressx_hist_batch_per_fit if per_fit else lib().dressx_hist_batch
    code = fn(reqs, n)
    flats, lens = v["hist_flat"].tolist(), v["hist_len"].tolist()
    mss, nsub = v["multisets"].tolist(), v["num_subgraphs"].tolist()
    fits, status = v["fits"].tolist(), v["status"].tolist()
    v["hist_flat"] = 0
    out = []
    for i, g in enumerate(graphs):
        ms = None
        if mss[i]:
            ms = _arr(ctypes.cast(mss[i], ctypes.POINTER(ctypes.c_double)), nsub[i] * g.E,
                      np.float64).reshape(nsub[i], g.E)
            lib().dressx_free(mss[i])
        out.append((_take_i64(flats[i], lens[i]), ms, nsub[i], fits[i], status[i]))
    _check(code)
    return out


def _graph_args(n_vertices, sources, targets, weights, vertex_weights, variant, precompute):
    return Graph(n_vertices, sources, targets, weights, vertex_weights, variant, precompute)


def delta_fit(n_vertices, sources, targets, weights=None, vertex_weights=None, k=0, variant=UNDIRECTED,
              max_iterations=100, epsilon=1e-6, precompute=False, keep_multisets=False, offset=0, stride=1,
              n_samples=0, seed=0, compute_histogram=True):
    """GPU Delta^k-DRESS -- reference ``dress.cuda.delta_fit`` (:497-575)."""
    with _graph_args(n_vertices, sources, targets, weights, vertex_weights, variant, precompute) as g:
        flat, ms, ns, _, _ = hist_requests([g], DELTA, k, max_iterations, epsilon, n_samples, seed,
                                           keep_multisets, offset, stride, compute_histogram)[0]
        return DeltaDRESSResult(histogram=_flat_to_list(flat), multisets=ms, num_subgraphs=ns, flat=flat)


def nabla_fit(n_vertices, sources, targets, weights=None, vertex_weights=None, k=0, variant=UNDIRECTED,
              max_iterations=100, epsilon=1e-6, precompute=False, keep_multisets=False, n_samples=0, seed=0,
              compute_histogram=True, offset=0, stride=1):
    """GPU Nabla^k-DRESS -- reference ``dress.cuda.nabla_fit`` (:370-445)."""
    with _graph_args(n_vertices, sources, targets, weights, vertex_weights, variant, precompute) as g:
        flat, ms, ns, _, _ = hist_requests([g], NABLA, k, max_iterations, epsilon, n_samples, seed,
                                           keep_multisets, offset, stride, compute_histogram)[0]
        return NablaDRESSResult(histogram=_flat_to_list(flat), multisets=ms, num_tuples=ns, flat=flat)


def delta_fit_many(graphs, k=1, **kw):
    """Delta^k histograms of many ``Graph`` objects in one persistent launch;
    returns a list of flat int64 [bits, count, ...] arrays."""
    return [r[0] for r in hist_requests(graphs, DELTA, k, **kw)]


def nabla_fit_many(graphs, k=1, **kw):
    return [r[0] for r in hist_requests(graphs, NABLA, k, **kw)]


def configure(device=-1, memory_budget_bytes=0, fit_chunk=0, group_threads=0, exact_sums=0,
              one_launch_max_edges=0):
    """Replace the engine configuration (``dressx_configure``).  exact_sums=1
    sends every sum through the sorted path that backs the certified sums
    (same bits, slower); tests use it to exercise that path.
    one_launch_max_edges: graphs up to this many edges are fitted in one
    launch (0 = the built-in limit, -1 = never)."""
    cfg = _abi.Config()
    cfg.device = int(device)
    cfg.memory_budget_bytes = int(memory_budget_bytes)
    cfg.fit_chunk = int(fit_chunk)
    cfg.group_threads = int(group_threads)
    cfg.exact_sums = int(exact_sums)
    cfg.one_launch_max_edges = int(one_launch_max_edges)
    _check(lib().dressx_configure(ctypes.byref(cfg)))


class Batch:
    """A prepared batch of Delta/Nabla requests resident in device memory
    (``dressx_batch_*``): ``run()`` re-runs every fit and histogram on the
    device, ``fetch()`` copies the histograms back."""

    def __init__(self, graphs, kind=DELTA, k=1, max_iterations=100, epsilon=1e-6, n_samples=0, seed=0,
                 keep_multisets=False, offset=0, stride=1, compute_histogram=True):
        self.graphs = list(graphs)
        n = len(self.graphs)
        self.reqs = (_abi.HistRequest * n)()
        for i, g in enumerate(self.graphs):
            r = self.reqs[i]
            r.graph = g.ptr
            r.kind, r.k = int(kind), int(k)
            r.max_iterations, r.epsilon = int(max_iterations), float(epsilon)
            r.n_samples, r.seed = int(n_samples), int(seed) & 0xFFFFFFFF
            r.offset, r.stride = int(offset), int(stride)
            r.want_histogram = 1 if compute_histogram else 0
            r.keep_multisets = 1 if keep_multisets else 0
        h = ctypes.c_void_p()
        _check(lib().dressx_batch_create(self.reqs, n, ctypes.byref(h)))
        self.handle = h

    def run(self):
        _check(lib().dressx_batch_run(self.handle))

    def autotune(self):
        """Measure the batch kernel's schedules on the batch and keep the first,
        in the order of the returned dict, within 3 % of the fastest (median of
        three timed runs each).  Returns (threads per subgraph, CTAs per SM,
        {(threads, CTAs per SM): fits per ms})."""
        gt, cps = ctypes.c_int(), ctypes.c_int()
        rates = (ctypes.c_float * 8)()
        _check(lib().dressx_batch_autotune(self.handle, ctypes.byref(gt), ctypes.byref(cps), rates))
        keys = [(32, 1), (64, 1), (128, 1), (256, 1), (32, 2), (64, 2), (128, 2)]
        return gt.value, cps.value, {k: float(r) for k, r in zip(keys, rates)}

    def capture(self):
        """Capture the fit stage into a CUDA graph replayed by ``run()``."""
        _check(lib().dressx_batch_capture(self.handle))

    def fetch(self):
        _check(lib().dressx_batch_fetch(self.handle))
        out = []
        for i in range(len(self.graphs)):
            r = self.reqs[i]
            out.append(_take_i64(r.hist_flat, r.hist_len))
            r.hist_flat = None                       # the array owns it now
        return out

    def stats(self):
        f, s, e = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _check(lib().dressx_batch_stats(self.handle, ctypes.byref(f), ctypes.byref(s), ctypes.byref(e)))
        return dict(fits=f.value, sweeps=s.value, edge_updates=e.value)

    def timing(self):
        """(fit_ms, hist_ms) of the last run, CUDA events on the engine stream."""
        a, b = ctypes.c_double(), ctypes.c_double()
        _check(lib().dressx_batch_timing(self.handle, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def close(self):
        if self.handle:
            for i in range(len(self.graphs)):
                r = self.reqs[i]
                if r.hist_flat:
                    lib().dressx_free(ctypes.cast(r.hist_flat, ctypes.c_void_p))
                    r.hist_flat = None
                if r.multisets:
                    lib().dressx_free(ctypes.cast(r.multisets, ctypes.c_void_p))
                    r.multisets = None
            lib().dressx_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def stream_handle():
    """The engine's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
    p = ctypes.c_void_p()
    _check(lib().dressx_stream(ctypes.byref(p)))
    return p.value or 0


def counters(reset=False):
    h, d, l = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    lib().dressx_counters(ctypes.byref(h), ctypes.byref(d), ctypes.byref(l), 1 if reset else 0)
    return dict(h2d_bytes=h.value, d2h_bytes=d.value, launches=l.value)


FIT = 2                                   # DRESSX_FIT (DELTA = 0, NABLA = 1)
PATH_NONE, PATH_BATCH, PATH_LANE = 0, 1, 2


def estimate(g: Graph, kind=FIT, k=0):
    """Host-only plan of a served request: (device bytes reserved, path)."""
    b, p = ctypes.c_int64(), ctypes.c_int()
    _check(lib().dressx_server_estimate(g.ptr, int(kind), int(k), ctypes.byref(b), ctypes.byref(p)))
    return b.value, p.value


class Ticket:
    """One request in a Server; ``wait()`` returns its result dict."""

    def __init__(self, server, graph, kind, k, max_iterations, epsilon):
        self.server = server
        self.graph = graph                     # kept alive until done
        self.req = _abi.ServerRequest()
        r = self.req
        r.graph = graph.ptr
        r.kind, r.k = int(kind), int(k)
        r.max_iterations, r.epsilon = int(max_iterations), float(epsilon)
        self.code = lib().dressx_server_submit(server.handle, ctypes.byref(r))
        self._result = None

    @property
    def done(self):
        return bool(self.req.done)

    def wait(self, timeout_ms=-1):
        code = lib().dressx_server_wait(self.server.handle, ctypes.byref(self.req), int(timeout_ms))
        if code == 4 and not self.req.done:            # DRESSX_ETIMEOUT
            raise TimeoutError("request still in service")
        return self.result()

    def cancel(self):
        return lib().dressx_server_cancel(self.server.handle, ctypes.byref(self.req))

    def result(self):
        if self._result is not None:
            return self._result
        r = self.req
        if not r.done:
            return None
        out = dict(status=r.status, path=r.path, queue_ms=r.queue_ms, latency_ms=r.latency_ms,
                   reserved_bytes=r.reserved_bytes, fits=r.fits, edge_sweeps=r.edge_sweeps)
        if r.kind == FIT:
            out.update(iterations=r.iterations, delta=r.delta)
        else:
            flat = _take_i64(r.hist_flat, r.hist_len)
            r.hist_flat = None
            out.update(hist_flat=flat, num_subgraphs=r.num_subgraphs)
        self._result = out
        return out


class Server:
    """A continuous-batching request server (``dressx_server_*``): submit
    fits and Delta/Nabla requests from any thread; small ones share short
    persistent batch launches, large ones run on lanes beside them, all
    admitted against a device-memory budget."""

    def __init__(self, memory_budget_bytes=0, lanes=0, launch_slots=0, launch_work=0, finishers=0,
                 max_queued=0, device=-1):
        cfg = _abi.ServerConfig()
        cfg.device = int(device)
        cfg.memory_budget_bytes = int(memory_budget_bytes)
        cfg.lanes, cfg.launch_slots = int(lanes), int(launch_slots)
        cfg.launch_work, cfg.finishers = int(launch_work), int(finishers)
        cfg.max_queued = int(max_queued)
        h = ctypes.c_void_p()
        _check(lib().dressx_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self.handle = h

    def submit(self, graph: Graph, kind=FIT, k=0, max_iterations=100, epsilon=1e-6) -> Ticket:
        return Ticket(self, graph, kind, k, max_iterations, epsilon)

    def drain(self, timeout_ms=-1):
        _check(lib().dressx_server_drain(self.handle, int(timeout_ms)))

    def stats(self, reset=False):
        st = _abi.ServerStats()
        _check(lib().dressx_server_stats(self.handle, ctypes.byref(st), 1 if reset else 0))
        out = {name: getattr(st, name) for name, _ in _abi.ServerStats._fields_ if name != "cls"}
        for i, name in enumerate(_abi.SERVER_CLASSES):
            c = st.cls[i]
            out[name] = {f: getattr(c, f) for f, _ in _abi.ServerClassStats._fields_}
        return out

    def close(self):
        if self.handle:
            lib().dressx_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
