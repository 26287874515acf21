"""bench.py's JSON line on the host: the keys the benchmark contract asks for,
assembled from one run's figures (the GPU measurements replaced by fixed
numbers), so that an edit to the line's assembly cannot break the round's
benchmark unnoticed.  The measurements themselves run on a B200."""
import argparse
import json

import pytest


@pytest.fixture
def bench_line(monkeypatch):
    import bench
    import nbb

    stages = {"reset": 0.04, "bbox": 0.02, "morton_sort_groups": 0.14, "tree": 0.25, "traversal": 2.9}

    def fake_run(args, rank, world, local):
        res = {}
        for name, ms in (("mixed", 3.4), ("fp64", 16.4)):
            res[name] = {"ms_per_step": ms, "step_ms": [ms] * args.steps, "launches": 17 * args.steps,
                         "stages_ms": dict(stages), "interactions": 4.2e9, "mac_tests": 7.0e7,
                         "stack_overflow": 0, "n_groups": 872909, "n_octree_nodes": 1208671,
                         "group_size": 128, "cache_depth": 2}
        clocks = {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 80}
        return None, res, 4.8, clocks

    monkeypatch.setattr(bench, "run_nbb", fake_run)
    monkeypatch.setattr(nbb, "measure_fma_tflops",
                        lambda precision: 33.8 if precision == nbb.PRECISION_FP64 else 74.0)
    args = argparse.Namespace(steps=10, warmup=3, n=1 << 20, no_error=True, no_cpu_baseline=True, gpus=1,
                              impl="nbb")
    return bench.bench_nbb(args, 0, 1, 0)


def test_bench_line_has_the_contract_keys(bench_line):
    line = json.loads(json.dumps(bench_line))
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "e2e", "gpu_launches", "clocks",
                "roofline"):
        assert key in line, key
    assert line["value"] == pytest.approx(1000.0 / 3.4)
    assert line["ms_per_step_median"] == pytest.approx(3.4)
    assert line["higher_is_better"] is True and line["n_gpus"] == 1 and line["steps"] == 10
    assert line["config"]["workload"].startswith("plummer N=2^20")
    assert line["e2e"]["value"] == pytest.approx(1000.0 / 4.8)
    assert line["e2e"]["h2d_bytes_per_step"] == 7 * 8 * (1 << 20)
    assert line["e2e"]["d2h_bytes_per_step"] == 6 * 8 * (1 << 20)
    assert line["gpu_launches"] == 170


def test_bench_line_rooflines(bench_line):
    r = bench_line["roofline"]
    assert r["bound"] == "fp32" and r["unit"] == "TFLOP/s" and r["peak"] == 74.0
    assert r["achieved"] == pytest.approx(20.0 * 4.2e9 / 2.9e-3 / 1e12)
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])
    b = bench_line["build_roofline"]
    assert b["bound"] == "hbm" and b["unit"] == "GB/s"
    assert b["ms"] == pytest.approx(0.02 + 0.14 + 0.25)
    assert b["achieved"] == pytest.approx(b["algorithmic_bytes"] / (b["ms"] * 1e-3) / 1e9)
    assert bench_line["plain_fp64"]["roofline"]["peak"] == 33.8
    assert bench_line["speedup_mixed_vs_fp64"] == pytest.approx(16.4 / 3.4)
