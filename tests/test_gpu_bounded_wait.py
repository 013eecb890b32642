"""The bounded device waits run out without a fault: with the wait limit of
the per-candidate kernels' staged masks set to zero polls, every block gives
up at once, counts a timeout, drains its own bulk copy and reads the global
masks, and the results are bit-identical to a normal run."""
import ctypes as C
import math

import numpy as np
import pytest

from fastrrt_b200 import synth

pytestmark = pytest.mark.gpu
MS = math.radians(40.0)


def timeouts(F):
    c = C.c_uint64(0)
    assert F.lib().fastrrt_debug_stage_timeouts(C.byref(c)) == 0, F._lib.last_error()
    return c.value


def test_stage_wait_runs_out(gpu):
    L = gpu.lib()
    cls = synth.make_frame(31, 256, coverage=0.15)
    heading, sx, sz, steer, seg = synth.candidates(50000, 256, 256, 31)
    fr = gpu.SearchFrame(class_ids=cls, class_costs=synth.CLASS_COSTS)
    ctx = gpu.Candidates(fr, min_dist=(22, 40), max_steering_rad=MS, lr_m=2.7, heading_grid=heading)
    x, z, lh, gx, gz, gh = synth.hermite_pairs(4096, 256, 256, 3, num_points=64)
    timeouts(gpu)
    want_k, want_kp = ctx.kinematic(sx, sz, steer, seg, 2.0)
    want_h, want_hp = ctx.hermite(x, z, lh, gx, gz, gh, 0.8)
    assert timeouts(gpu) == 0
    assert L.fastrrt_debug_set_stage_wait_limit(0) == 0
    try:
        got_k, got_kp = ctx.kinematic(sx, sz, steer, seg, 2.0)
        got_h, got_hp = ctx.hermite(x, z, lh, gx, gz, gh, 0.8)
        n = timeouts(gpu)
    finally:
        assert L.fastrrt_debug_set_stage_wait_limit(1 << 22) == 0
    assert n > 0
    assert np.array_equal(got_k.view(np.uint32), want_k.view(np.uint32)) and got_kp == want_kp
    assert np.array_equal(got_h.view(np.uint32), want_h.view(np.uint32)) and got_hp == want_hp
    # back to normal
    again, _ = ctx.kinematic(sx, sz, steer, seg, 2.0)
    assert np.array_equal(again.view(np.uint32), want_k.view(np.uint32))
    assert timeouts(gpu) == 0
