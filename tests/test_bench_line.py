"""The compact sections of the bench line (bench.compact_sections), on
synthetic measurements: the single-fit HBM fractions with the measured DRAM
traffic, the serving percentiles and the other workloads' summaries stay on
the one JSON line; full figures go to --detail.  CPU only."""
import json

import bench


def _fit(sweep_ms, frac, traffic=None, dram_frac=None):
    return {"sweep_ms": sweep_ms, "edge_iters_per_s": 1.8e10, "iterations": 27, "setup_ms": 48.6,
            "e2e_ms": 100.0, "phases_ms": {"upload": 19.0},
            "roofline": {"frac": frac, "traffic": traffic, "dram_frac": dram_frac}}


def test_single_fit_fractions_and_traffic():
    single = {"weighted": _fit(1.53, 0.2116, 4.730e9, 0.481),
              "unweighted": _fit(1.44, 0.1768),
              "cpu_baseline": {"omp": {"ms_per_sweep": 11412.0}}}
    out = bench.compact_sections(single, None, None, None)
    sf = out["single_fit"]
    assert sf["weighted"]["hbm_frac"] == 0.212 and sf["weighted"]["sweep_ms"] == 1.53
    assert sf["weighted"]["traffic_gb"] == 4.73 and sf["weighted"]["dram_frac"] == 0.481
    # no capture for this size: no traffic keys rather than a made-up figure
    assert "traffic_gb" not in sf["unweighted"] and "dram_frac" not in sf["unweighted"]
    assert sf["cpu_omp_ms_per_sweep"] == 11400.0
    assert set(out) == {"single_fit"}


def test_serving_and_other_sections_are_compact():
    serving = {"rates": [{"offered_rate": r, "graphs_per_s": r * 1.05, "p50_ms": 2.0, "p99_ms": 33.3,
                          "failed": 0, "by_path": {"fit_lane": {"n": 3}}} for r in (20.0, 80.0, 320.0)]}
    k2 = {lab: {"value": 2.01e6, "autotune": {"threads_per_subgraph": 128, "ctas_per_sm": 2},
                "cpu_baseline": {"value": 497.0}} for lab in ("delta2", "nabla1")}
    plain = {"dress_fit_cuda": {"ms_per_fit": 0.587},
             "cpu_baseline": {"single_thread": {"value": 34.4}, "omp": {"value": 487.8}}}
    out = bench.compact_sections(None, serving, k2, plain)
    assert [r["rate"] for r in out["serving"]] == [20.0, 80.0, 320.0]
    assert all(set(r) == {"rate", "graphs_per_s", "p50_ms", "p99_ms", "failed"} for r in out["serving"])
    assert out["delta2_nabla1"]["delta2"] == {"value": 2010000.0, "schedule": "128x2", "cpu_1t": 497.0}
    assert out["plain_fit"]["ms_per_fit"] == 0.587
    assert out["plain_fit"]["cpu_1t_ms"] == 29.1 and out["plain_fit"]["cpu_omp_ms"] == 2.05
    # the summaries stay small: the whole line is read from the tail of the log
    assert len(json.dumps(out)) < 1200


def test_single_fit_traffic_constants_cover_both_variants():
    c = bench.SINGLE_FIT_NCU
    assert c["edges"] == 28_000_000
    assert 4e9 < c["unweighted"] < c["weighted"] < 6e9
