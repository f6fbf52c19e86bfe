"""Benchmark of the B200 DRESS engine (one JSON line on rank 0).

Headline workload (batched Delta^1): 2,000 random
d-regular graphs (configuration model with switching repair), n ~ U[16,100],
d ~ U{3..12}, unweighted, k = 1, epsilon 1e-6, max 100 sweeps, exact
(value, count) histogram per graph.  One step = all ~115K vertex-deleted
subgraph fits plus the 2,000 histograms.  Metric: subgraph-fits/s.

* ``value``: the prepared batch (graphs resident in HBM), device time of
  the fits + histograms from CUDA events on the engine stream, L2 flushed
  (256 MiB write) between timed steps, outside the timed regions.
* ``e2e``: the public C-ABI call ``dressx_hist_batch`` with host graphs,
  wall clock per step: host packing, H2D, fits, histograms, D2H, results
  in malloc'd host arrays.  The caller frees the previous step's arrays
  before the step's timer starts.
* ``per_fit_gpu``: the reference's driver structure with this engine's GPU
  fit (``dressx_hist_batch_per_fit``: host subgraph build + one fit launch
  sequence per subgraph) on a bounded sample -- the batched/per-fit ratio.
* ``cpu_baseline``: the reference's single-thread C ``dress_delta_fit``
  (compiled from its sources into oracle/_ref) on a bounded sample.
* ``single_fit``: the 28M-edge Chung-Lu fit (the single large fit),
  edge-iters/s and the HBM roofline of its sweeps.
* ``delta2_nabla1``: Delta^2 and Nabla^1 of 64 random 10-regular graphs of
  200 vertices, autotuned and replayed from a CUDA graph.
* ``plain_fit``: one G(2000, 10000) fit (the plain fit) through
  dress_fit_cuda and through the server's batch path.
* ``serving``: a stream of fit and Delta^1 requests (the serving stream)
  submitted to the request server at Poisson arrival rates
  swept over ``--serve-rates``: graphs/s, subgraph-fits/s, p50/p99 latency
  per request kind and per path, device overlap, admission statistics, a
  spot check that served results equal the same requests run alone, and the
  reference's sequential single-thread calls on the same stream as the CPU
  baseline.

``--impl reference`` times the reference's own CPU implementation
(``dress_delta_fit_omp``, all host threads) on a bounded sample of the same
workload.  With ``--gpus N`` (torchrun), the 2,000 graphs are sharded over
ranks (no collective on the data path); value = all ranks' fits / max time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "dress-graph_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

HBM_FALLBACK_GBS = 6650.0

# k_batch on the 2,000-graph headline batch (64 threads per subgraph, two CTAs
# per SM), one launch under `ncu --set full` (profiles/k_batch_delta1_2000graphs.md):
# dram__bytes_read.sum + dram__bytes_write.sum, and the issue-bound figures
KBATCH_HEADLINE_NCU = {"dram_bytes": 19.33e6 + 190.33e6,
                       "issue": {"issue_active_frac": 0.724, "lanes_per_inst": 19.5, "fp64_pipe_frac": 0.227}}

# The 28M-edge single fit: dram__bytes_read.sum + dram__bytes_write.sum of the
# twelve sweep kernels of one sweep (sweep 10), one capture per variant
# (profiles/single_fit_chunglu28m_sweep_dram.md)
SINGLE_FIT_NCU = {"edges": 28_000_000, "weighted": 4.218e9 + 0.512e9, "unweighted": 3.858e9 + 0.283e9}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--graphs", type=int, default=2000)
    ap.add_argument("--no-single-fit", action="store_true", help="skip the 28M-edge single fit")
    ap.add_argument("--single-fit-edges", type=int, default=28_000_000)
    ap.add_argument("--single-fit-only", action="store_true",
                    help="run only the single large fit and print its JSON object (profiling runs)")
    ap.add_argument("--single-fit-variants", default="weighted,unweighted")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="budget of the CPU baseline sample")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving stream")
    ap.add_argument("--no-k2", action="store_true", help="skip the Delta^2 / Nabla^1 workload")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-fit workload")
    ap.add_argument("--serve-requests", type=int, default=200)
    ap.add_argument("--serve-rates", default="20,80,320", help="Poisson arrival rates (requests/s) to sweep")
    ap.add_argument("--detail", default="", help="also write every measured figure to this JSON file")
    ap.add_argument("--no-parity", action="store_true", help="skip the comparisons with the reference")
    ap.add_argument("--profile-plain", action="store_true",
                    help="fit the plain-fit graph (Erdos-Renyi G(2000, 10000)) once, then once more between "
                         "cudaProfilerStart/Stop, and exit")
    ap.add_argument("--profile-headline", action="store_true",
                    help="set up the headline batch (autotuned), run it once, then run it once more between "
                         "cudaProfilerStart/Stop (for ncu --profile-from-start off), and exit")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return HBM_FALLBACK_GBS, "fallback"


class Clocks:
    """Samples nvidia-smi clocks/throttle reasons during a timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_init(n_gpus):
    """Rank/world from torchrun's environment (gloo-free: N=1 needs nothing)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
        pg = dist
    return rank, world, local, pg


def allmax(pg, x):
    if pg is None:
        return x
    import torch
    t = torch.tensor([float(x)], device="cuda")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def allsum(pg, x):
    if pg is None:
        return x
    import torch
    t = torch.tensor([float(x)], device="cuda")
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


# ---------------------------------------------------------------------------
# headline: batched Delta^1 over 2,000 random regular graphs
# ---------------------------------------------------------------------------

def regular_workload(count):
    from dress_b200 import graphs
    return graphs.regular_batch(count, (16, 100), (3, 12), seed=42)


def cpu_delta1_sample(gs, budget_s, kind):
    """Reference single-thread Delta^1 on graphs taken in order until the
    time budget is spent; returns (fits/s, graphs, fits, seconds)."""
    import oracle
    cpu = oracle.reference() if kind == "reference" else oracle.port()
    fits, t0, used = 0, time.perf_counter(), 0
    for n, U, V in gs:
        cpu.delta_fit(n, U, V, k=1, max_iterations=100, epsilon=1e-6)
        fits += n
        used += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return fits / dt, used, fits, dt


def bench_delta1(args, rank, world, pg, torch, clocks):
    import dress_b200 as db
    gs_all = regular_workload(args.graphs)
    mine = gs_all[rank::world]
    objs = [db.Graph(n, U, V) for n, U, V in mine]
    stream = torch.cuda.ExternalStream(db.stream_handle())
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MiB > L2

    # ---- device throughput, inputs resident --------------------------------
    db.counters(reset=True)
    batch = db.Batch(objs, db.DELTA, 1, max_iterations=100, epsilon=1e-6)
    create = db.counters(reset=True)
    tune = batch.autotune()              # schedule for this size class (later batches reuse it)
    batch.capture()                      # fit stage replayed from a CUDA graph
    for _ in range(args.warmup):
        batch.run()
    ref_hist = batch.fetch()
    barrier(pg)
    torch.cuda.synchronize()
    clocks.start()
    dev_ms = fit_ms = hist_ms = 0.0
    db.counters(reset=True)
    wall0 = time.perf_counter()
    for step in range(args.steps):
        flush.fill_(float(step))
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        batch.run()
        ev1.record(stream)
        ev1.synchronize()
        dev_ms += ev0.elapsed_time(ev1)
        f, h = batch.timing()
        fit_ms += f
        hist_ms += h
    wall = time.perf_counter() - wall0
    launches = db.counters()["launches"]
    torch.cuda.synchronize()
    barrier(pg)
    st = batch.stats()
    fits_step = st["fits"]
    max_dev_ms = allmax(pg, dev_ms)
    total_fits = allsum(pg, fits_step * args.steps)
    value = total_fits / (max_dev_ms / 1e3)

    # ---- end to end through the C ABI, host graphs ---------------------------
    db.counters(reset=True)
    e2e_s = 0.0
    out = None
    for step in range(args.steps + 1):
        out = None                 # the caller releases the previous step's histograms before the timer starts
        t0 = time.perf_counter()
        out = db.hist_requests(objs, db.DELTA, 1, max_iterations=100, epsilon=1e-6)
        dt = time.perf_counter() - t0
        if step == 0:                                    # untimed warm-up call
            db.counters(reset=True)
            continue
        e2e_s += dt
    cnt = db.counters()
    clk = clocks.stop()            # samples cover the device-timed steps and the e2e calls
    same = all(np.array_equal(a[0], b) for a, b in zip(out, ref_hist))
    e2e_s = allmax(pg, e2e_s)
    e2e_value = total_fits / e2e_s
    h2d_step = cnt["h2d_bytes"] / args.steps
    d2h_step = cnt["d2h_bytes"] / args.steps

    # ---- the reference's per-fit structure with this engine's GPU fit ------------
    per_fit = None
    if rank == 0:
        fits, t0, used = 0, time.perf_counter(), 0
        for g in objs:
            db.hist_requests([g], db.DELTA, 1, per_fit=True)
            fits += g.N
            used += 1
            if time.perf_counter() - t0 > 8.0:
                break
        dt = time.perf_counter() - t0
        per_fit = {"value": fits / dt, "unit": "subgraph-fits/s", "sample": f"first {used} graphs, {fits} fits",
                   "batched_over_per_fit": value / (fits / dt)}

    # ---- roofline of the dominant kernel (the batched fit) -----------------------
    peak, peak_kind = peaks()
    live_values = sum(n * (len(U) - (2 * len(U)) // n) for n, U, V in mine)   # E - d per subgraph
    alg_bytes = create["h2d_bytes"] + 8 * live_values                           # parents read + values written
    achieved = alg_bytes / (fit_ms / args.steps / 1e3) / 1e9
    # DRAM bytes and issue figures of one launch on this workload and schedule,
    # from the committed ncu capture (profiles/k_batch_delta1_2000graphs.md)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": KBATCH_HEADLINE_NCU["dram_bytes"] if args.graphs == 2000 else None,
                "peak_source": peak_kind, "kernel": "k_batch",
                "issue": dict(KBATCH_HEADLINE_NCU["issue"], source="profiles/k_batch_delta1_2000graphs.md")}

    for g in objs:
        g.close()
    batch.close()
    return dict(value=value, ms_per_step=max_dev_ms / args.steps, fits_per_step=allsum(pg, fits_step),
                edge_updates_per_step=allsum(pg, st["edge_updates"]), fit_ms=fit_ms / args.steps,
                hist_ms=hist_ms / args.steps, wall_ms=wall * 1e3 / args.steps, launches=launches,
                e2e={"value": e2e_value, "unit": "subgraph-fits/s", "h2d_bytes_per_step": int(h2d_step),
                     "d2h_bytes_per_step": int(d2h_step), "matches_device_run": bool(same)},
                per_fit=per_fit, roofline=roofline, clocks=clk, gs=gs_all, hists=ref_hist, mine=mine,
                tune={"threads_per_subgraph": tune[0], "ctas_per_sm": tune[1]})


# ---------------------------------------------------------------------------
# parity with the reference, outside every timed region
# ---------------------------------------------------------------------------

def ref_cpu():
    """The reference library compiled from its sources (oracle/_ref), else the
    oracle's C restatement; the second value names which."""
    import oracle
    cpu = oracle.reference()
    return (cpu, "reference") if cpu is not None else (oracle.port(), "port")


def parity_hists(pairs, kind, k):
    """Histograms of this engine against the reference's call on the same
    graph: pairs is [((n, U, V), flat [bits, count] array)]."""
    cpu, which = ref_cpu()
    omp = which == "reference"
    fn = cpu.delta_fit if kind == "delta" else cpu.nabla_fit
    t0 = time.perf_counter()
    bad = 0
    for (n, U, V), flat in pairs:
        ref = fn(n, U, V, k=k, max_iterations=100, epsilon=1e-6, omp=omp)
        bad += not np.array_equal(flat, ref["hist"])
    name = f"dress_{kind}_fit" + ("_omp" if omp else " (oracle port)")
    return {"graphs": len(pairs), "identical": bad == 0, "mismatched": bad, "against": name,
            "seconds": round(time.perf_counter() - t0, 1)}


def sha256(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def golden_large(n, U, V, W):
    """The reference's digests of the single-fit workload
    (tests/golden/large_fit.json, made by tests/golden/make_large_golden.py),
    when this run generated the same graph; else None."""
    path = os.path.join(ROOT, "tests", "golden", "large_fit.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        gold = json.load(f)
    gg = gold["graph"]
    if (gg["N"], gg["E"]) != (n, len(U)) or gg["sha_U"] != sha256(U) or gg["sha_V"] != sha256(V) \
            or gg["sha_W"] != sha256(W):
        return None
    return gold


# ---------------------------------------------------------------------------
# single large fit: Chung-Lu 4M vertices / 28M edges
# ---------------------------------------------------------------------------

def bench_single_fit(args, torch):
    import dress_b200 as db
    from dress_b200 import graphs
    n = 4_000_000 * args.single_fit_edges // 28_000_000
    n, U, V = graphs.chung_lu(n, args.single_fit_edges, 2.3, 20000, seed=42)
    E = len(U)
    out = {"workload": f"Chung-Lu power law, N={n}, E={E}, gamma 2.3, max degree 20000, epsilon 1e-6"}
    peak, peak_kind = peaks()
    variants = [v for v in args.single_fit_variants.split(",") if v]
    if not args.single_fit_only:
        # graph construction: the host build and the device build of the same graph
        Wb = graphs.uniform_weights(E, seed=7)
        t0 = time.perf_counter()
        gh = db.Graph(n, U, V, Wb)
        host_ms = (time.perf_counter() - t0) * 1e3
        db.Graph(n, U[:1000], V[:1000], device_build=True).close()        # warm-up
        t0 = time.perf_counter()
        gd = db.Graph(n, U, V, Wb, device_build=True)
        dev_ms = (time.perf_counter() - t0) * 1e3
        ch, cd = gh.ptr.contents, gd.ptr.contents
        S = ch.adj_offset[n]
        same = (ch.adj_offset[n] == cd.adj_offset[n] and
                np.array_equal(np.ctypeslib.as_array(ch.adj_target, (S,)), np.ctypeslib.as_array(cd.adj_target, (S,))) and
                np.array_equal(np.ctypeslib.as_array(ch.adj_edge_idx, (S,)), np.ctypeslib.as_array(cd.adj_edge_idx, (S,))) and
                np.array_equal(np.ctypeslib.as_array(ch.edge_weight, (E,)).view(np.int64),
                               np.ctypeslib.as_array(cd.edge_weight, (E,)).view(np.int64)))
        gh.close()
        gd.close()
        out["graph_build"] = {"host_ms": host_ms, "device_ms": dev_ms, "identical": bool(same),
                              "note": "dress_init_graph (host, stable counting sorts) vs dressx_init_graph (GPU radix "
                                      "sort), both including the copies of the caller's arrays in and the CSR out"}
    gold = None if args.no_parity else golden_large(n, U, V, graphs.uniform_weights(E, seed=7))
    for label, W in (("weighted", graphs.uniform_weights(E, seed=7)), ("unweighted", None)):
        if label not in variants:
            continue
        g = db.Graph(n, U, V, W)
        S = int(g.ptr.contents.adj_offset[n])
        # an untimed one-sweep fit of the same graph first: it grows the device
        # memory pool to this variant's buffer sizes and pins the stages, as a
        # serving process has done before its requests
        db.fit_graph(g, 1, 1e-6)
        # three timed fits (one for profiling runs), each from the initial
        # values; the figures are the fit of median end-to-end time
        runs = []
        for _ in range(1 if args.single_fit_only else 3):
            _reset_edges(g)
            db.counters(reset=True)
            t0 = time.perf_counter()
            it, dl = db.fit_graph(g, 100, 1e-6)
            runs.append((time.perf_counter() - t0, db.counters(), db.last_fit_stats(), it, dl))
        setups = [r[2]["setup_ms"] for r in runs]
        wall, cnt, st, it, dl = sorted(runs, key=lambda r: r[0])[len(runs) // 2]
        sweeps = st["sweeps"]
        sweep_ms = st["iterate_ms"] / max(1, sweeps)
        # algorithmic bytes per sweep: 24N + 12S + 48E weighted, 24N + 12S + 32E unweighted
        b_iter = 24 * n + 12 * S + (48 if W is not None else 32) * E
        achieved = b_iter / (sweep_ms / 1e3) / 1e9
        traffic = SINGLE_FIT_NCU[label] if E == SINGLE_FIT_NCU["edges"] else None
        out[label] = {
            "iterations": it, "sweeps": sweeps, "delta": dl, "common_terms": st["common_terms"],
            "edge_iters_per_s": E * sweeps / (st["iterate_ms"] / 1e3),
            "edge_iters_per_s_e2e": E * sweeps / wall,
            "sweep_ms": sweep_ms, "setup_ms": st["setup_ms"], "e2e_ms": wall * 1e3, "phases_ms": st["phases_ms"],
            "timed_fits": len(runs), "setup_ms_range": [min(setups), max(setups)],
            "h2d_bytes": cnt["h2d_bytes"], "d2h_bytes": cnt["d2h_bytes"], "launches": cnt["launches"],
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                         "algorithmic_bytes_per_sweep": b_iter,
                         # measured DRAM bytes per sweep over the sweep time: how busy HBM is
                         "dram_frac": (traffic / (sweep_ms / 1e3) / 1e9 / peak) if traffic else None},
        }
        if gold is not None and label in gold:
            f = gold[label]["full"]
            out[label]["parity"] = {
                "ref_iterations": f["iterations"],
                "identical": bool(it == f["iterations"] and int(np.float64(dl).view(np.int64)) == f["delta_bits"]
                                  and sha256(g.edge_dress) == f["sha_edge_dress"]
                                  and sha256(g.vertex_dress) == f["sha_vertex_dress"]),
                "against": "SHA-256 of the reference's dress_fit_omp edge and vertex values "
                           "(tests/golden/large_fit.json)"}
        g.close()
    if not args.single_fit_only:
        # the reference's CPU fits on the same weighted graph, a bounded number
        # of sweeps (epsilon 0 runs exactly that many)
        import ctypes
        import oracle
        cpu = oracle.reference()
        kind = "reference" if cpu is not None else "port"
        cpu = cpu or oracle.port()
        t0 = time.perf_counter()
        gr = cpu.build(n, U, V, graphs.uniform_weights(E, seed=7))
        build_s = time.perf_counter() - t0
        it_, dl_ = ctypes.c_int(), ctypes.c_double()
        res = {}
        # one OpenMP sweep (a single-thread sweep merge-walks the hub rows for
        # minutes: sum of deg^2 is ~4e10 steps on this graph)
        for label, fn, sweeps in (("omp", getattr(cpu, "fit_omp", None), 1),):
            if fn is None:
                continue
            t0 = time.perf_counter()
            fn(gr, sweeps, 0.0, ctypes.byref(it_), ctypes.byref(dl_))
            dt = time.perf_counter() - t0
            res[label] = {"value": E * sweeps / dt, "unit": "edge-iters/s", "ms_per_sweep": dt * 1e3 / sweeps,
                          "cores": len(os.sched_getaffinity(0)) if label == "omp" else 1, "kind": kind,
                          "sample": f"{sweeps} sweep(s) of the weighted fit (epsilon 0)"}
        cpu.free_graph(gr)
        res["graph_build_s"] = build_s
        out["cpu_baseline"] = res
    return out


# ---------------------------------------------------------------------------
# Delta^2 and Nabla^1 on 64 random 10-regular graphs of 200 vertices
# ---------------------------------------------------------------------------

def bench_k2(args, clocks):
    import dress_b200 as db
    from dress_b200 import graphs
    gs = [graphs.random_regular(200, 10, seed=1000 + i) for i in range(64)]
    objs = [db.Graph(n, U, V) for n, U, V in gs]
    out = {"workload": "64 random 10-regular graphs, n=200 (1,000 edges each), epsilon 1e-6; Delta^2 "
                       "(C(200,2)=19,900 subgraphs per graph) and Nabla^1 (200 marked fits per graph); "
                       "autotuned threads per subgraph, fit stage replayed from a CUDA graph",
           "l2": "values of a step (10 GB for Delta^2) exceed L2; parents are staged in shared memory"}
    clocks.start()
    nabla_hists = None
    for label, kind, k in (("delta2", db.DELTA, 2), ("nabla1", db.NABLA, 1)):
        b = db.Batch(objs, kind, k)
        t0 = time.perf_counter()
        best, per_sm, rates = b.autotune()
        tune_s = time.perf_counter() - t0
        b.capture()
        b.run()                                  # warm-up
        steps = min(args.steps, 3) if label == "delta2" else args.steps
        fit_ms = hist_ms = 0.0
        db.counters(reset=True)
        for _ in range(steps):
            b.run()
            f, h = b.timing()
            fit_ms += f
            hist_ms += h
        launches = db.counters()["launches"]
        st = b.stats()
        step_ms = (fit_ms + hist_ms) / steps
        out[label] = {
            "value": st["fits"] / (step_ms / 1e3), "unit": "subgraph-fits/s", "steps": steps,
            "fits_per_step": st["fits"], "edge_updates_per_step": st["edge_updates"],
            "edge_sweeps_per_s": st["edge_updates"] / (fit_ms / steps / 1e3),
            "fit_ms": fit_ms / steps, "hist_ms": hist_ms / steps, "ms_per_step": step_ms,
            "gpu_launches_per_step": launches / steps,
            "autotune": {"threads_per_subgraph": best, "ctas_per_sm": per_sm,
                         "sampled_fits_per_ms": {f"{t}x{c}": v for (t, c), v in rates.items()}, "seconds": tune_s},
            "cuda_graph": True,
        }
        if label == "nabla1" and not args.no_parity:
            nabla_hists = b.fetch()
        b.close()
    out["clocks"] = clocks.stop()
    # end to end through the C ABI on a sample of 4 graphs (a full step's
    # histograms are ~20 GB of host memory); the first call, untimed, pins
    # the 1.25 GB staging buffer and grows the device pool, as the headline's
    # untimed first end-to-end call does
    res = db.hist_requests(objs[:4], db.DELTA, 2)
    del res
    t0 = time.perf_counter()
    res = db.hist_requests(objs[:4], db.DELTA, 2)
    dt = time.perf_counter() - t0
    out["delta2"]["e2e_sample"] = {"value": sum(r[3] for r in res) / dt, "unit": "subgraph-fits/s",
                                   "sample": "first 4 of the 64 graphs, one dressx_hist_batch call after an untimed one",
                                   "seconds": dt, "distinct_values": int(sum(r[0].size // 2 for r in res))}
    if not args.no_parity:
        out["parity"] = {"delta2": parity_hists(list(zip(gs[:4], [r[0] for r in res])), "delta", 2),
                         "nabla1": parity_hists(list(zip(gs, nabla_hists)), "nabla", 1)}
    del res
    # CPU: the reference's single-thread strided call on graph 0, extrapolated
    import oracle
    cpu = oracle.reference()
    kind = "reference" if cpu is not None else "port"
    cpu = cpu or oracle.port()
    n, U, V = gs[0]
    for label, fn, k, stride, per_graph in (("delta2", cpu.delta_fit, 2, 199, 19900),
                                            ("nabla1", cpu.nabla_fit, 1, 10, 200)):
        t0 = time.perf_counter()
        fn(n, U, V, k=k, offset=0, stride=stride)
        dt = time.perf_counter() - t0
        fits = -(-per_graph // stride)
        out[label]["cpu_baseline"] = {
            "value": fits / dt, "unit": "subgraph-fits/s", "cores": 1, "kind": kind,
            "sample": f"graph 0, strided slice offset 0 stride {stride} ({fits} fits, {dt:.2f} s); "
                      f"extrapolated step time {64 * per_graph / (fits / dt):.0f} s"}
    for g in objs:
        g.close()
    return out


# ---------------------------------------------------------------------------
# plain fit: one Erdos-Renyi graph, n=2000, m=10000
# ---------------------------------------------------------------------------

def bench_plain(args):
    import dress_b200 as db
    from dress_b200 import graphs
    n, U, V = graphs.erdos_renyi(2000, 10000, seed=42)
    E = len(U)
    out = {"workload": "Erdos-Renyi G(2000, 10000), seed 42, unweighted, undirected, epsilon 1e-6, max 100"}
    g = db.Graph(n, U, V)
    for _ in range(3):
        _reset_edges(g)
        db.fit_graph(g, 100, 1e-6)
    reps = 20
    t0 = time.perf_counter()
    dev = 0.0
    for _ in range(reps):
        _reset_edges(g)
        it, dl = db.fit_graph(g, 100, 1e-6)
        st = db.last_fit_stats()
        dev += st["iterate_ms"] + st["setup_ms"]
    wall = time.perf_counter() - t0
    sweeps = st["sweeps"]
    out["dress_fit_cuda"] = {"fits_per_s": reps / wall, "ms_per_fit": wall * 1e3 / reps,
                             "device_ms_per_fit": dev / reps, "iterations": it, "sweeps": sweeps,
                             "edge_iters_per_s": E * sweeps * reps / wall}
    # the same fit through the server's batch path (one request at a time, and 64 in flight)
    with db.Server() as srv:
        for _ in range(3):
            _reset_edges(g)
            srv.submit(g, db.FIT).wait()
        t0 = time.perf_counter()
        for _ in range(reps):
            _reset_edges(g)
            r = srv.submit(g, db.FIT).wait()
        wall1 = time.perf_counter() - t0
        many = [db.Graph(n, U, V) for _ in range(64)]
        t0 = time.perf_counter()
        ts = [srv.submit(x, db.FIT) for x in many]
        for t in ts:
            t.wait()
        wall64 = time.perf_counter() - t0
        same = all(np.array_equal(x.edge_dress.view(np.int64), g.edge_dress.view(np.int64)) for x in many)
        for x in many:
            x.close()
    out["served"] = {"path": r["path"], "ms_per_fit_alone": wall1 * 1e3 / reps,
                     "fits_per_s_64_in_flight": 64 / wall64, "identical_to_dress_fit_cuda": bool(same)}
    g.close()
    import oracle
    cpu = oracle.reference()
    kind = "reference" if cpu is not None else "port"
    cpu = cpu or oracle.port()
    t0 = time.perf_counter()
    for _ in range(3):
        cpu.fit(n, U, V)
    dt1 = (time.perf_counter() - t0) / 3
    res = {"single_thread": {"value": 1.0 / dt1, "unit": "fits/s", "cores": 1, "kind": kind,
                             "sample": "3 fits, dress_fit"}}
    if kind == "reference":
        t0 = time.perf_counter()
        for _ in range(3):
            cpu.fit(n, U, V, omp=True)
        dto = (time.perf_counter() - t0) / 3
        res["omp"] = {"value": 1.0 / dto, "unit": "fits/s", "cores": len(os.sched_getaffinity(0)),
                      "kind": kind, "sample": "3 fits, dress_fit_omp"}
    out["cpu_baseline"] = res
    return out


# ---------------------------------------------------------------------------
# serving: Poisson arrivals of fit and Delta^1 requests through the server
# ---------------------------------------------------------------------------

def _reset_edges(g):
    """Edge values back to the initial 1.0 (a fit continues from them)."""
    if g.E:
        np.ctypeslib.as_array(g.ptr.contents.edge_dress, shape=(g.E,))[:] = 1.0


def _pct(v, q):
    if not v:
        return None
    v = sorted(v)
    return v[max(0, int(np.ceil(q * len(v))) - 1)]


def bench_serving(args, clocks):
    import dress_b200 as db
    from dress_b200 import graphs
    reqs = graphs.serving_stream(args.serve_requests, seed=5)
    objs = [db.Graph(n, U, V, W) for (_, n, U, V, W) in reqs]
    kinds = [k for k, *_ in reqs]
    names = {0: "delta1", 2: "fit"}
    out = {"workload": f"{len(reqs)} requests: {sum(k == 0 for k in kinds)} Delta^1 (edges log-uniform 10..5K) and "
                       f"{sum(k == 2 for k in kinds)} fits (edges log-uniform 10..1M); random d-regular below 5K "
                       "edges, Chung-Lu (gamma 2.3, mean degree 14) above; 30% weighted U[0.5,2]; epsilon 1e-6",
           "total_edges": int(sum(g.E for g in objs)), "rates": []}
    clocks.start()
    with db.Server() as srv:
        # untimed warm-up pass over the whole stream, submitted at once: kernel
        # attributes, and the arena grown to the stream's peak before any rate
        for g in objs:
            _reset_edges(g)
        ws = [srv.submit(g, k, 1 if k == 0 else 0) for g, k in zip(objs, kinds)]
        srv.drain()
        assert all(t.result()["status"] == 0 for t in ws)
        for rate in [float(x) for x in args.serve_rates.split(",") if x]:
            for g in objs:
                _reset_edges(g)
            gaps = np.random.default_rng(17).exponential(1.0 / rate, len(objs))
            srv.stats(reset=True)
            db.counters(reset=True)
            tickets = []
            t0 = time.perf_counter()
            due = t0
            for g, k, gap in zip(objs, kinds, gaps):
                due += gap
                wait = due - time.perf_counter()
                if wait > 0:
                    time.sleep(wait)
                tickets.append(srv.submit(g, k, 1 if k == 0 else 0))
            srv.drain()
            wall = time.perf_counter() - t0
            st = srv.stats()
            cnt = db.counters()
            res = [t.result() for t in tickets]
            lat = {name: [r["latency_ms"] for r, k in zip(res, kinds) if k == kk] for kk, name in names.items()}
            allv = [r["latency_ms"] for r in res]
            row = {
                "offered_rate": rate, "wall_s": wall, "completed": st["completed"], "failed": st["failed"],
                "graphs_per_s": st["completed"] / wall, "subgraph_fits_per_s": st["fits"] / wall,
                "edge_sweeps_per_s": st["edge_sweeps"] / wall,
                "p50_ms": _pct(allv, 0.5), "p99_ms": _pct(allv, 0.99),
                "by_kind": {name: {"n": len(v), "p50_ms": _pct(v, 0.5), "p99_ms": _pct(v, 0.99)}
                            for name, v in lat.items()},
                "by_path": {name: {"n": st[name]["completed"], "p50_ms": st[name]["p50_ms"],
                                   "p99_ms": st[name]["p99_ms"], "queue_p99_ms": st[name]["queue_p99_ms"]}
                            for name in ("fit_batch", "fit_lane", "hist_batch", "hist_lane")},
                "batch_launches": st["batch_launches"], "gpu_launches": cnt["launches"],
                "device_busy_ms": st["device_busy_ms"], "device_work_ms": st["device_work_ms"],
                "overlap": st["device_work_ms"] / st["device_busy_ms"] if st["device_busy_ms"] else None,
                "max_in_service": st["max_in_service"], "peak_reserved_bytes": st["peak_reserved_bytes"],
                "pool_bytes": st["pool_bytes"], "budget_bytes": st["budget_bytes"],
                "h2d_bytes": cnt["h2d_bytes"], "d2h_bytes": cnt["d2h_bytes"],
            }
            out["rates"].append(row)
        # spot check: served results equal the same requests run alone
        rng = np.random.default_rng(3)
        idx = rng.choice(len(objs), size=min(12, len(objs)), replace=False)
        served_fit = {int(i): objs[int(i)].edge_dress for i in idx if kinds[int(i)] == 2}
        same = True
        for i in idx:
            i = int(i)
            if kinds[i] == 0:
                flat = db.hist_requests([objs[i]], db.DELTA, 1)[0][0]
                same &= bool(np.array_equal(flat, tickets[i].result()["hist_flat"]))
            else:
                _reset_edges(objs[i])
                db.fit_graph(objs[i], 100, 1e-6)
                same &= bool(np.array_equal(objs[i].edge_dress.view(np.int64), served_fit[i].view(np.int64)))
        out["same_alone_and_in_mix"] = {"checked": len(idx), "identical": same}
    out["clocks"] = clocks.stop()

    # CPU: the reference's sequential single-thread calls, requests in arrival order
    import oracle
    cpu = oracle.reference()
    kind = "reference" if cpu is not None else "port"
    cpu = cpu or oracle.port()
    t0 = time.perf_counter()
    done, per = 0, {"fit": [], "delta1": []}
    for (k, n, U, V, W) in reqs:
        t1 = time.perf_counter()
        if k == 0:
            cpu.delta_fit(n, U, V, W, k=1)
        else:
            cpu.fit(n, U, V, W)
        per[names[k]].append((time.perf_counter() - t1) * 1e3)
        done += 1
        if time.perf_counter() - t0 > args.cpu_seconds:
            break
    dt = time.perf_counter() - t0
    out["cpu_baseline"] = {"value": done / dt, "unit": "requests/s", "cores": 1, "kind": kind,
                           "sample": f"first {done} requests of the stream in arrival order, one at a time "
                                     f"({dt:.1f} s)",
                           "mean_ms": {kk: (sum(v) / len(v) if v else None) for kk, v in per.items()}}
    for g in objs:
        g.close()
    return out


# ---------------------------------------------------------------------------
# the reference arm: the reference's own CPU implementation
# ---------------------------------------------------------------------------

def reference_arm(args, rank):
    if rank != 0:
        return
    import oracle
    cpu = oracle.reference()
    kind = "reference"
    if cpu is None:
        cpu, kind = oracle.port(), "port"
    cores = len(os.sched_getaffinity(0))
    gs = regular_workload(args.graphs)
    # a bounded sample per step: consecutive graphs of the workload
    per_step = max(1, int(os.environ.get("DRESS_REF_GRAPHS", "150")))
    omp = kind == "reference"

    def step(i):
        fits = 0
        base = (i * per_step) % len(gs)
        for j in range(per_step):
            n, U, V = gs[(base + j) % len(gs)]
            cpu.delta_fit(n, U, V, k=1, max_iterations=100, epsilon=1e-6, omp=omp)
            fits += n
        return fits

    for i in range(args.warmup):
        step(i)
    t0 = time.perf_counter()
    fits = sum(step(args.warmup + i) for i in range(args.steps))
    dt = time.perf_counter() - t0
    v = fits / dt
    line = {"metric": "Delta^1 subgraph-fits/s", "value": v, "unit": "subgraph-fits/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": f"batched Delta^1, {per_step} of the {len(gs)} random regular graphs per step "
                                   "(n~U[16,100], d~U{3..12}), epsilon 1e-6"},
            "cpu_baseline": {"value": v, "unit": "subgraph-fits/s", "cores": cores if omp else 1, "kind": kind,
                             "sample": f"{per_step} graphs per step ({'dress_delta_fit_omp' if omp else 'oracle port'})"},
            "e2e": {"value": v, "unit": "subgraph-fits/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# the figures of the other workloads that go on the one JSON line (all of
# them go to --detail)
# ---------------------------------------------------------------------------

def _r(x, nd=3):
    return None if x is None else float(f"{x:.{nd}g}")


def compact_sections(single, serving, k2, plain):
    out = {}
    if single:
        sf = {}
        for label in ("weighted", "unweighted"):
            v = single.get(label)
            if v:
                sf[label] = {"sweep_ms": _r(v["sweep_ms"]), "hbm_frac": _r(v["roofline"]["frac"]),
                             "edge_iters_per_s": _r(v["edge_iters_per_s"]), "iterations": v["iterations"],
                             "setup_ms": _r(v["setup_ms"]), "e2e_ms": _r(v["e2e_ms"])}
                if v["roofline"].get("traffic"):
                    sf[label]["traffic_gb"] = _r(v["roofline"]["traffic"] / 1e9)
                    sf[label]["dram_frac"] = _r(v["roofline"]["dram_frac"])
        cb = single.get("cpu_baseline", {}).get("omp")
        if cb:
            sf["cpu_omp_ms_per_sweep"] = _r(cb["ms_per_sweep"])
        out["single_fit"] = sf
    if k2:
        out["delta2_nabla1"] = {lab: {"value": _r(k2[lab]["value"]),
                                      "schedule": f"{k2[lab]['autotune']['threads_per_subgraph']}x"
                                                  f"{k2[lab]['autotune']['ctas_per_sm']}",
                                      "cpu_1t": _r(k2[lab]["cpu_baseline"]["value"])}
                                for lab in ("delta2", "nabla1")}
    if plain:
        cb = plain.get("cpu_baseline", {})
        out["plain_fit"] = {"ms_per_fit": _r(plain["dress_fit_cuda"]["ms_per_fit"]),
                            "cpu_1t_ms": _r(1e3 / cb["single_thread"]["value"]) if "single_thread" in cb else None,
                            "cpu_omp_ms": _r(1e3 / cb["omp"]["value"]) if "omp" in cb else None}
    if serving:
        out["serving"] = [{"rate": r["offered_rate"], "graphs_per_s": _r(r["graphs_per_s"]),
                           "p50_ms": _r(r["p50_ms"]), "p99_ms": _r(r["p99_ms"]), "failed": r["failed"]}
                          for r in serving["rates"]]
    return out


# ---------------------------------------------------------------------------

def main():
    args = parse()
    rank, world, local, pg = dist_init(args.gpus)
    if args.impl == "reference":
        reference_arm(args, rank)
        if pg is not None:
            pg.destroy_process_group()
        return
    import torch
    torch.cuda.set_device(local)
    import dress_b200 as db
    db.configure(device=local)
    if args.single_fit_only:
        print(json.dumps({"single_fit": bench_single_fit(args, torch)}), flush=True)
        return
    if args.profile_plain:
        from dress_b200 import graphs
        n, U, V = graphs.erdos_renyi(2000, 10000, seed=42)
        with db.Graph(n, U, V) as g:
            db.fit_graph(g, 100, 1e-6)
            _reset_edges(g)
            torch.cuda.synchronize()
            torch.cuda.cudart().cudaProfilerStart()
            it, _ = db.fit_graph(g, 100, 1e-6)
            torch.cuda.synchronize()
            torch.cuda.cudart().cudaProfilerStop()
        print(json.dumps({"profiled": "plain fit, one call", "iterations": it}), flush=True)
        return
    if args.profile_headline:
        gs = regular_workload(args.graphs)
        objs = [db.Graph(n, U, V) for n, U, V in gs]
        b = db.Batch(objs, db.DELTA, 1, max_iterations=100, epsilon=1e-6)
        tune = b.autotune()
        b.run()
        torch.cuda.synchronize()
        torch.cuda.cudart().cudaProfilerStart()
        b.run()
        torch.cuda.synchronize()
        torch.cuda.cudart().cudaProfilerStop()
        print(json.dumps({"profiled": "headline batch, one run", "schedule": list(tune[:2]),
                          "fit_ms": b.timing()[0]}), flush=True)
        b.close()
        return
    clocks = Clocks(local)
    head = bench_delta1(args, rank, world, pg, torch, clocks)
    single = None
    serving = k2 = plain = None
    cpu = None
    if rank == 0 and world == 1:
        v, used, fits, dt = cpu_delta1_sample(head["gs"], args.cpu_seconds,
                                              "reference" if __import__("oracle").reference() else "port")
        kind = "reference" if __import__("oracle").reference() else "port"
        cpu = {"value": v, "unit": "subgraph-fits/s", "cores": 1, "kind": kind,
               "sample": f"single-thread dress_delta_fit on the first {used} graphs ({fits} fits, {dt:.1f} s)"}
        if not args.no_single_fit:
            single = bench_single_fit(args, torch)
        if not args.no_serving:
            serving = bench_serving(args, Clocks(local))
        if not args.no_k2:
            k2 = bench_k2(args, Clocks(local))
        if not args.no_plain:
            plain = bench_plain(args)
    parity = {}
    if rank == 0 and not args.no_parity:
        # every graph this rank fitted, against the reference's OpenMP Delta^1
        parity["delta1"] = parity_hists(list(zip(head["mine"], head["hists"])), "delta", 1)
        if k2 and "parity" in k2:
            parity.update(k2["parity"])
        if single:
            for label in ("weighted", "unweighted"):
                pr = (single.get(label) or {}).get("parity")
                if pr:
                    parity[f"single_fit_{label}"] = {"identical": pr["identical"],
                                                     "ref_iterations": pr["ref_iterations"]}
    if rank == 0:
        clk = head["clocks"]
        detail = {"headline": {k: v for k, v in head.items() if k not in ("gs", "hists", "mine")},
                  "cpu_baseline": cpu, "single_fit": single, "serving": serving, "delta2_nabla1": k2,
                  "plain_fit": plain, "parity": parity}
        if args.detail:
            with open(args.detail, "w") as f:
                json.dump(detail, f, indent=1, default=float)
        line = {
            "metric": "Delta^1 subgraph-fits/s", "value": head["value"], "unit": "subgraph-fits/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"batched Delta^1 of {args.graphs} random d-regular graphs (n~U[16,100], "
                                   "d~U{3..12}, seed 42), k=1, epsilon 1e-6, exact histogram per graph",
                       "fits_per_step": head["fits_per_step"],
                       "l2": "256 MiB flush between timed steps",
                       "parallelism": f"graphs sharded over {world} GPU(s)",
                       "schedule": f"{head['tune']['threads_per_subgraph']} threads/subgraph, "
                                   f"{head['tune']['ctas_per_sm']} CTA/SM"},
            "e2e": head["e2e"], "gpu_launches": head["launches"], "roofline": head["roofline"],
            "cpu_baseline": cpu, "clocks": clk,
            "breakdown_ms": {"fits": head["fit_ms"], "histograms": head["hist_ms"]},
        }
        if head["per_fit"]:
            line["per_fit_gpu"] = {"value": head["per_fit"]["value"],
                                   "batched_over_per_fit": head["per_fit"]["batched_over_per_fit"]}
        line.update(compact_sections(single, serving, k2, plain))
        if parity:
            line["parity"] = {k: {"graphs": v["graphs"], "identical": v["identical"]} if "graphs" in v else v
                              for k, v in parity.items()}
        print(json.dumps(line, default=float), flush=True)
    if pg is not None:
        barrier(pg)
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
