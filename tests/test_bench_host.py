"""Host-side pieces of bench.py that need no GPU: the served stream's device-timeline split, the
C3 / c3small shape draws, and the reference arm's step bound.  (The timed legs themselves are GPU
work and are checked by running bench.py on a B200.)"""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)
import bench  # noqa: E402


def test_gpu_timeline_split():
    # (copies issued, copies landed, kernels started, kernels done) per unit, ms
    units = {
        (0.0, 5.0, 5.0, 105.0),      # first unit: waited 5 ms for its own copy
        (50.0, 90.0, 105.0, 205.0),  # issued and landed under the first unit: no gap
        (230.0, 240.0, 240.0, 300.0),  # issued 25 ms after the previous unit ended, copy 10 ms
        (240.0, 320.0, 320.0, 400.0),  # issued in time, copy landed 20 ms after the previous end
    }
    t = bench.gpu_timeline(units)
    assert t["gpu_kernels_ms"] == pytest.approx(100 + 100 + 60 + 80)
    assert t["gpu_idle_before_issue_ms"] == pytest.approx(25.0)
    assert t["gpu_waiting_for_copy_ms"] == pytest.approx(10.0 + 20.0)
    assert t["gpu_span_ms"] == pytest.approx(400.0 - 5.0)
    # kernel time + the gaps tile the span exactly
    assert t["gpu_kernels_ms"] + t["gpu_idle_before_issue_ms"] + t["gpu_waiting_for_copy_ms"] == \
        pytest.approx(t["gpu_span_ms"])


def test_gpu_timeline_ignores_incomplete_units():
    assert bench.gpu_timeline({(-1.0, -1.0, -1.0, -1.0)}) == {}
    t = bench.gpu_timeline({(0.0, 1.0, 1.0, 2.0), (-1.0, -1.0, -1.0, -1.0)})
    assert t["gpu_kernels_ms"] == pytest.approx(1.0)


def test_c3_shape_draws():
    shapes = bench.c3_shapes()
    assert len(shapes) == 64 and shapes == bench.c3_shapes()  # seeded
    assert all(16 <= nb <= 22 and nbe - nb in (1, 2) and 16 <= nc <= 512 for nb, nbe, nc in shapes)
    assert sum(1 for nb, nbe, nc in shapes if nbe - nb == 2) == 16
    small = bench.c3small_shapes()
    assert len(small) == 256 and all(10 <= nb <= 16 and 8 <= nc <= 128 for nb, nbe, nc in small)


def test_reference_arm_step_bound():
    assert bench.REF_MAX_STEPS >= 1
    assert max(1, min(20, bench.REF_MAX_STEPS)) == bench.REF_MAX_STEPS
