"""bench.py's roofline arithmetic and peak selection, on the CPU."""
import json
import os
import sys
import types

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_measured_peaks_reads_the_pool_file(tmp_path):
    p = tmp_path / "peaks.json"
    p.write_text(json.dumps({"hbm_gbs": 6500.0, "bf16_tflops": 1700.0}))
    assert bench.measured_peaks(str(p))["hbm_gbs"] == 6500.0
    assert bench.measured_peaks(str(tmp_path / "absent.json")) is None
    (tmp_path / "bad.json").write_text("not json")
    assert bench.measured_peaks(str(tmp_path / "bad.json")) is None


def test_tridiag_roofline_uses_the_pool_peak_and_reports_the_in_run_one():
    args = types.SimpleNamespace(precision="fp64-gram")
    kernel = {"ms": 2.0, "bytes": 4.0e9, "flops": 1.0e9, "phases": 8}
    r = bench.roofline(args, {}, kernel, None, 5000.0, {"hbm_gbs": 6400.0})
    assert r["achieved"] == pytest.approx(2000.0)          # 4 GB / 2 ms
    assert r["peak"] == 6400.0 and r["frac"] == pytest.approx(2000.0 / 6400.0)
    assert r["peak_in_run"] == 5000.0 and r["frac_of_in_run"] == pytest.approx(0.4)
    assert "MEASURED_PEAKS" in r["peak_source"] and r["frac_of"] == "measured"
    r = bench.roofline(args, {}, kernel, None, 5000.0, None)   # no pool file: the in-run copy
    assert r["peak"] == 5000.0 and r["frac"] == pytest.approx(0.4)
    assert "this run" in r["peak_source"]


def test_plain_roofline_counts_flops_over_the_timed_region():
    args = types.SimpleNamespace(precision="fp64")
    r = bench.roofline(args, {"svd_flops": 3.0e13, "seconds": 2.0}, None, 30.0, 5000.0, {"hbm_gbs": 6400.0})
    assert r["bound"] == "tensor" and r["achieved"] == pytest.approx(15.0)
    assert r["frac"] == pytest.approx(0.5)
