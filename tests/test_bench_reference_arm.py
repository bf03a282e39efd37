"""The benchmark's reference arm runs the reference's CPU path on every host
core it can use, as concurrent single-rank replicas (spawned processes timed
together behind a barrier).  Checked on the CPU with two replicas of a small
grid: both report, the throughput is all points over the slowest replica's
time, and a single replica reports the same kind of sample."""
import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def _single_sample():
    import bench

    return bench.cpu_reference_sample(1, 0, n=32)


@pytest.mark.timeout(300)
def test_reference_arm_replicas_on_two_cores():
    import multiprocessing as mp

    import bench

    v, kind, cores, sample = bench.cpu_reference_parallel(1, 0, n=32, workers=2)
    assert cores == 2 and v > 0
    assert kind in ("reference", "port")
    assert sample.startswith("2 concurrent single-rank replicas")
    # in a child process: the sample selects the reference shim's fast FFT,
    # a choice the loaded library keeps for the rest of its process
    with mp.get_context("spawn").Pool(1) as pool:
        v1, kind1, cores1, _ = pool.apply(_single_sample)
    assert cores1 == 1 and v1 > 0 and kind1 == kind


def test_reference_arm_prints_only_on_rank_zero(monkeypatch, capsys):
    """Under torchrun every rank starts the reference arm; the ranks other
    than 0 exit 0 at once, without work or output."""
    import argparse

    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("LOCAL_RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    called = []
    monkeypatch.setattr(bench, "cpu_reference_parallel", lambda *a, **k: called.append(a))
    assert bench.run_reference(argparse.Namespace(steps=1, warmup=1, gpus=2)) == 0
    assert called == [] and capsys.readouterr().out == ""


def test_reference_arm_line_carries_the_contract_keys(monkeypatch, capsys):
    import argparse
    import json

    import bench

    monkeypatch.setenv("RANK", "0")
    monkeypatch.setenv("WORLD_SIZE", "1")
    monkeypatch.setattr(bench, "cpu_reference_parallel",
                        lambda *a, **k: (12.5, "reference", 4, "4 concurrent single-rank replicas (test)"))
    assert bench.run_reference(argparse.Namespace(steps=2, warmup=1, gpus=1)) == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] == 12.5
    for key in ("metric", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["cpu_baseline"]["cores"] == 4 and line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"] == {"value": 12.5, "unit": line["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert line["metric"] == bench.METRIC
