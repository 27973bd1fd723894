"""The synthetic workloads bench.py measures: shapes, ranges and seeds as the configurations
name them, and the same jobs on every call."""
import math
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_scale_is_the_256_cubed_lattice():
    (j,) = bench.workload_jobs("scale")
    assert j["box"] == (256, 256, 256) and j["blocks"] == (16, 16, 16)
    assert j["n_vacancies"] == round(2e-5 * 2 * 256 ** 3) == 671
    assert j["temperature"] == 563.0 and j["precision"] == 0
    assert dict(j["alloy"]) == {1: 9766, 2: 134, 4: 70, 8: 30}  # Fe-1.34Cu-0.7Ni-0.3Mn at.%
    assert bench.workload_jobs("scale32")[0]["precision"] == 1


def test_batched_boxes_follow_their_ranges():
    jobs = bench.workload_jobs("batched")
    assert len(jobs) == 512 and jobs == bench.workload_jobs("batched")
    edges = np.array([j["box"][0] for j in jobs])
    assert edges.min() >= 16 and edges.max() <= 48
    assert abs(np.mean(np.log(edges)) - (math.log(16) + math.log(48)) / 2) < 0.05  # log-uniform
    for j in jobs:
        a = dict(j["alloy"])
        assert 50 <= a[2] <= 150 and 0 <= a[4] <= 100 and 0 <= a[8] <= 50 and sum(a.values()) == 10000
        assert 473.0 <= j["temperature"] <= 673.0 and j["precision"] == 1
        assert j["n_vacancies"] == max(1, round(1e-4 * 2 * j["box"][0] ** 3))
    assert len({j["seed"] for j in jobs}) == 512


def test_serving_stream_is_poisson_with_the_named_ranges():
    jobs = bench.serve_jobs(200.0, 60.0)
    assert jobs == bench.serve_jobs(200.0, 60.0)
    t = np.array([j["t"] for j in jobs])
    assert np.all(np.diff(t) > 0) and t[-1] < 60.0
    assert abs(len(jobs) - 12000) < 4 * math.sqrt(12000)  # 200/s for 60 s
    gaps = np.diff(t)
    assert abs(gaps.mean() - 1 / 200) < 0.1 / 200 and abs(gaps.std() / gaps.mean() - 1) < 0.05  # exponential
    edges = np.array([j["box"][0] for j in jobs])
    budgets = np.array([j["hop_budget"] for j in jobs])
    assert edges.min() >= 16 and edges.max() <= 96 and budgets.min() >= 1e4 and budgets.max() <= 1e6
    assert abs(np.mean(np.log(budgets)) - (math.log(1e4) + math.log(1e6)) / 2) < 0.05
    for j in jobs[:200]:
        assert all(b >= 1 and e // b >= 8 for e, b in zip(j["box"], j["blocks"]))  # blocks of >= 8 cells
        assert all(-(-e // b) <= 24 for e, b in zip(j["box"], j["blocks"]))  # staged regions fit


def test_reference_arm_prints_the_contract_line():
    # one process, no GPU: the reference arm times the oracle on the host cores and prints one
    # JSON line with the benchmark's keys, an end-to-end figure without transfers and its own
    # CPU baseline record
    import json
    import subprocess

    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--workload", "serial",
                        "--steps", "3", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.strip().splitlines()
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "hops/s" and d["higher_is_better"] is True
    assert d["n_gpus"] == 1 and d["steps"] == 3 and d["warmup"] == 3 and d["dtype"] == "f64"
    assert d["value"] > 0 and d["ms_per_step"] > 0 and d["vs_baseline"] is None
    assert d["e2e"] == {"value": d["value"], "unit": "hops/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    c = d["cpu_baseline"]
    assert c["value"] == d["value"] and c["kind"] == "port" and c["cores"] >= 1 and c["sample"]
    assert "20^3" in d["config"]["workload"]
