"""Host logic of bench.py's convergence leg (CPU): the crossing of relMSE 1e-3
read off a progressive trace, log-log interpolated between checkpoints."""
import math

import pytest


def test_crossing_time_interpolates_a_power_law_exactly():
    import bench
    # relMSE = c / spp and time proportional to spp: the log-log interpolation
    # between the checkpoints around the target is exact
    c, ms_per_spp = 0.7, 9.5
    trace = [(spp, spp * ms_per_spp, c / spp) for spp in (64, 128, 256, 512, 1024)]
    chk, t = bench.crossing_time(trace, 1e-3)
    assert chk == pytest.approx(1024 * ms_per_spp)
    assert t == pytest.approx(700 * ms_per_spp, rel=1e-9)


def test_crossing_time_edge_cases():
    import bench
    # never reaches the target
    assert bench.crossing_time([(64, 10.0, 0.5), (128, 20.0, 0.2)], 1e-3) == (None, None)
    # the first checkpoint is already below it: its own time
    assert bench.crossing_time([(64, 10.0, 5e-4), (128, 20.0, 2e-4)], 1e-3) == (10.0, 10.0)
    # a noisy trace that rises before it falls below: the checkpoint's time
    chk, t = bench.crossing_time([(64, 10.0, 2e-3), (128, 20.0, 3e-3), (192, 30.0, 9e-4)], 1e-3)
    assert chk == 30.0
    f = math.log(3e-3 / 1e-3) / math.log(3e-3 / 9e-4)
    assert t == pytest.approx(20.0 * (30.0 / 20.0) ** f)
    # a trace that does not fall between the two checkpoints
    assert bench.crossing_time([(64, 10.0, 8e-4), (128, 20.0, 9e-4)], 1e-3) == (10.0, 10.0)
