"""Interpolation of planned paths and their curve quality on the GPU: the
cells of every interpolated curve equal the host interpolation's
(interpolate_planned_path_p, the reference's interpolation.cpp:36-135
arithmetic) and their headings agree within 1e-5 rad (the device's and the
host library's atan2f / cosf may differ in the last bit); length, jerk and
tangential discontinuity equal the CPU restatement of the reference's
curve_quality.py within 1e-6 relative."""
import math

import numpy as np
import pytest

from fastrrt_b200 import synth
from oracle import curve_quality as Q

pytestmark = pytest.mark.gpu
COSTS = synth.CLASS_COSTS


def test_batch_interpolation_matches_host_and_quality_matches_oracle(gpu):
    n = 24
    args = [synth.c0_request(s) for s in range(n)]
    reqs = [gpu.make_request(c, COSTS, a, b, seed=s, max_iterations=200) for s, (c, a, b) in enumerate(args)]
    B = gpu.BatchPlanner(n, 256, 256)
    valid, _, _, _ = B.plan(reqs, 400, 4)
    assert valid.sum() >= n - 2
    length, jerk, disc = B.interpolate()
    assert len(length) == n
    fr = gpu.SearchFrame(class_ids=args[0][0], class_costs=COSTS)
    host = gpu.FastRRT(search_frame=fr, perception_width_m=34.56, perception_height_m=34.56,
                       max_steering_angle_deg=40, vehicle_length_m=5.4, timeout_ms=-1, min_dist_x=22,
                       min_dist_z=40, path_costs=COSTS, seed=0)
    host.set_plan_data(fr, args[0][1], args[0][2], 2.0)
    checked = 0
    for k in range(n):
        if not valid[k]:
            continue
        path = B.path(k)
        got = B.interpolated_path(k)
        want = np.array([(w.x, w.z, w.heading.rad()) for w in host.interpolate_planned_path_p(path)],
                        np.float32)
        assert got.shape == want.shape, k
        assert np.array_equal(got[:, :2], want[:, :2]), k
        assert np.max(np.abs(got[:, 2] - want[:, 2])) <= 1e-5, k
        L, J, D = Q.assess(got, float(path[0, 2]))
        assert math.isclose(length[k], L, rel_tol=1e-6), k
        assert math.isclose(jerk[k], J, rel_tol=1e-6, abs_tol=1e-9), k
        assert disc[k] == int(D), k
        checked += 1
    assert checked >= n - 2
    # the metrics vary over the paths (not a constant placeholder)
    assert len(set(np.round(jerk[valid > 0], 4))) > 1
