"""The benchmark's reference arm runs the reference's CPU path on every host
core it can use, as concurrent single-rank replicas (spawned processes timed
together behind a barrier).  Checked on the CPU with two replicas of a small
grid: both report, the throughput is all points over the slowest replica's
time, and a single replica reports the same kind of sample."""
import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


@pytest.mark.timeout(300)
def test_reference_arm_replicas_on_two_cores():
    import bench

    v, kind, cores, sample = bench.cpu_reference_parallel(1, 0, n=32, workers=2)
    assert cores == 2 and v > 0
    assert kind in ("reference", "port")
    assert sample.startswith("2 concurrent single-rank replicas")
    v1, kind1, cores1, _ = bench.cpu_reference_sample(1, 0, n=32)
    assert cores1 == 1 and v1 > 0 and kind1 == kind
