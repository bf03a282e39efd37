"""The benchmark's reference arm runs the reference's CPU path on every host
core it can use, as concurrent single-rank replicas (spawned processes timed
together behind a barrier).  Checked on the CPU with two replicas of a small
grid: both report, and the throughput is all points over the slowest
replica's time.  The bench's CPU-leg worker solves and saves a grid in a
child process, and its chunked error check agrees with numpy."""
import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


REF_LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "libppref.so")


@pytest.mark.timeout(300)
@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference build absent (make -C oracle PITTPACK_SRC=...)")
def test_reference_arm_replicas_on_two_cores():
    import bench

    v, cores, sample = bench.cpu_reference_parallel(n=32, workers=2)
    assert cores == 2 and v > 0
    assert sample.startswith("2 concurrent single-rank replicas")


@pytest.mark.timeout(300)
@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference build absent (make -C oracle PITTPACK_SRC=...)")
def test_cpu_leg_worker_and_chunked_error(tmp_path):
    import multiprocessing as mp

    import numpy as np

    import bench
    from oracle import oracle as O

    n = 24
    f = np.random.default_rng(2).uniform(-1, 1, (n, n, n))
    np.save(tmp_path / "f.npy", f)
    with mp.get_context("spawn").Pool(2) as pool:
        jobs = [pool.apply_async(bench._cpu_job, (k, n, "NNNNDD", str(tmp_path / "f.npy"), str(tmp_path / f"{k}.npy")))
                for k in ("reference", "oracle")]
        res = [j.get(timeout=240) for j in jobs]
    assert [r[2] for r in res] == ["ok", "ok"]
    P_ref = np.load(tmp_path / "reference.npy")
    P_orc = np.load(tmp_path / "oracle.npy")
    # the reference's solve equals the oracle's compat-mode solve; the exact-mode
    # one differs in the kx = ky = 0 column only
    assert O.rel_l2(O.solve(O.problem(n, n, n, "NNNNDD"), f), P_ref) <= 1e-13
    assert O.rel_l2(O.solve(O.problem(n, n, n, "NNNNDD", compat_zero_mode=0), f), P_orc) == 0.0
    pert = P_ref + 1e-9 * np.random.default_rng(0).standard_normal(P_ref.shape)
    assert abs(bench.rel_l2_files(pert, str(tmp_path / "reference.npy"), chunk=1000) - O.rel_l2(pert, P_ref)) < 1e-15


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
    assert bench.run_reference(argparse.Namespace(steps=1, warmup=1, gpus=2, n=512)) == 0
    assert called == [] and capsys.readouterr().out == ""


def test_reference_arm_line_carries_the_contract_keys(monkeypatch, capsys):
    import argparse
    import json

    import bench

    monkeypatch.setenv("RANK", "0")
    monkeypatch.setenv("WORLD_SIZE", "1")
    monkeypatch.setattr(bench, "cpu_reference_parallel",
                        lambda *a, **k: (12.5, 4, "4 concurrent single-rank replicas (test)"))
    monkeypatch.setattr(bench, "REF_LIB", bench.__file__)
    assert bench.run_reference(argparse.Namespace(steps=2, warmup=1, gpus=1, n=512)) == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] == 12.5
    for key in ("metric", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["cpu_baseline"]["cores"] == 4 and line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"] == {"value": 12.5, "unit": line["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert line["metric"] == bench.METRIC
