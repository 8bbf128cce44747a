"""The committed default bench line (profiles/bench_batched_default.json.txt,
written by `python bench.py` on a B200) keeps the output contract: every key
the JSON line must carry, and numbers that agree with one another and with
the workload they describe."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LINE = os.path.join(ROOT, "profiles", "bench_batched_default.json.txt")


@pytest.fixture(scope="module")
def line():
    with open(LINE) as f:
        return json.loads(f.read())


def test_top_level_keys(line):
    for k, t in [("metric", str), ("value", float), ("unit", str), ("n_gpus", int), ("steps", int),
                 ("warmup", int), ("ms_per_step", float), ("higher_is_better", bool), ("scaling", str),
                 ("dtype", str), ("data", str), ("config", dict), ("roofline", dict), ("cpu_baseline", dict),
                 ("e2e", dict), ("gpu_launches", int), ("clocks", dict)]:
        assert isinstance(line[k], t), k
    assert "vs_baseline" in line
    assert line["higher_is_better"] is True and line["scaling"] == "weak"
    assert line["n_gpus"] >= 1 and line["steps"] >= 1 and line["warmup"] >= 3
    assert "workload" in line["config"]


def test_value_is_the_workload_bytes_over_the_step(line):
    cfg = line["config"]
    n, ncols, nq = cfg["nrows_per_gpu"], cfg["ncols"], cfg["queries_per_step"]
    step_bytes = 4 * n * ncols + nq * n / 8  # columns once per batch, one bitmap per query
    gbs = step_bytes * line["n_gpus"] / (line["ms_per_step"] * 1e-3) / 1e9
    assert abs(gbs - line["value"]) / line["value"] < 0.01
    assert abs(line["queries_per_s"] - nq * line["n_gpus"] / (line["ms_per_step"] * 1e-3)) / line["queries_per_s"] < 0.01


def test_roofline(line):
    r = line["roofline"]
    assert r["bound"] in ("hbm", "tensor")
    assert r["unit"] == ("GB/s" if r["bound"] == "hbm" else "TFLOP/s")
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 0.002
    peaks = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks):
        with open(peaks) as f:
            hbm = json.load(f).get("hbm_gbs")
        if hbm:
            assert abs(r["peak"] - hbm) < 1.0
    assert r["traffic"] is None or r["traffic"] > 0
    assert line["gpu_launches"] == line["steps"] * r["kernel_launches_per_step"]


def test_cpu_baseline_and_e2e(line):
    c = line["cpu_baseline"]
    assert c["kind"] in ("reference", "port") and c["cores"] >= 1 and c["value"] > 0 and c["sample"]
    e = line["e2e"]
    cfg = line["config"]
    n, ncols, nq = cfg["nrows_per_gpu"], cfg["ncols"], cfg["queries_per_step"]
    words = (n + 31) // 32
    assert e["unit"] == line["unit"]
    # what the call moved: every column up (plus the plan), the bitmaps down,
    # sparse row chunks as nonzero-word masks and values, so at most the whole bitmaps
    # and counts plus the per-chunk nonzero-word counts
    assert 4 * n * ncols <= e["h2d_bytes_per_step"] < 4 * n * ncols * 1.01
    assert e["dense_d2h_bytes_per_step"] == nq * (words * 4 + 8)
    assert 0 < e["d2h_bytes_per_step"] <= e["dense_d2h_bytes_per_step"] * 1.01
    assert 0 < e["value"] < line["value"]


def test_clocks(line):
    k = line["clocks"]
    assert k["sm_mhz"] > 0 and k["sm_max_mhz"] > 0 and isinstance(k["reasons"], list)
    bad = {"hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"}
    assert not bad & set(k["reasons"])


def test_bench_help_runs_without_a_gpu():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--help"], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0 and "--impl" in r.stdout


def test_every_scan_configuration_is_in_the_line(line):
    """The plain single-column 1e8-row scan (>= 70 % of the HBM peak), the
    2-4 column conjunctions fused and separate, the selectivity sweep on
    uniform, 256- and 64-value columns through the fused scan and the BinDex,
    and the served rates 1k-50k q/s with the highest rate kept up with."""
    s = line["single_1e8"]
    assert s["frac"] >= 0.70 and abs(s["frac"] - s["GB_s"] / s["peak"]) < 0.002
    m = line["multi_1e8"]["queries"]
    assert [q["columns"] for q in m] == [2, 3, 4] and all(q["equal"] for q in m)
    sw = line["sweep_1e8"]["queries"]
    assert {q["column"] for q in sw} == {"uniform", "range:0:256", "range:0:64"}
    assert {q["target"] for q in sw if q["column"] == "uniform"} == {0.001, 0.01, 0.1, 0.5, 0.9}
    assert all(q["equal"] for q in sw)
    rates = [r["offered_qps"] for r in line["served"]["rates"]]
    assert min(rates) <= 1000 and max(rates) >= 50000
    top = line["served"]["max_sustained"]
    assert top["offered_qps"] in rates and top["achieved_qps"] >= 0.98 * top["offered_qps"]


def test_autotune_report_in_the_line(line):
    a = line["batch_config"]["autotune"]
    assert a["sample_rows"] == line["config"]["nrows_per_gpu"] and len(a["candidates"]) >= 18
    assert {c["warps_per_cta"] for c in a["candidates"]} == {8, 16}
    assert a["best_ms"] == min(c["ms"] for c in a["candidates"])
