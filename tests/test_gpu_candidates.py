"""Per-candidate kernels on the GPU through the C ABI: bit-exact against the
reference's own kernels compiled for sm_100a (oracle/_ref, run on the same
GPU), against the golden fixtures, and close to the CPU oracle."""
import ctypes
import math
import os

import numpy as np
import pytest

from fastrrt_b200 import synth

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
W = H = 256
MS = math.radians(40.0)
LR = 5.4 / 2


def ctx_for(F, cls, heading=None, min_dist=(22, 40)):
    fr = F.SearchFrame(class_ids=cls, class_costs=synth.CLASS_COSTS)
    return fr, F.Candidates(fr, min_dist=min_dist, max_steering_rad=MS, lr_m=LR, heading_grid=heading)


@pytest.mark.parametrize("coverage", [0.05, 0.15, 0.30])
def test_kinematic_bit_exact_vs_reference_kernel(gpu, ref, coverage):
    # the per-candidate microbench at full size: 2^20 candidates per density
    cls = synth.make_frame(100 + int(coverage * 100), 256, coverage=coverage)
    heading, sx, sz, steer, seg = synth.candidates(1 << 20, W, H, int(coverage * 1000))
    fr, ctx = ctx_for(gpu, cls, heading)
    out, probes = ctx.kinematic(sx, sz, steer, seg, 2.0)
    rc = ref.RefCase(ref.Frame(cls, synth.CLASS_COSTS), heading=heading, max_steer_rad=MS, lr=LR,
                     mdx=11, mdz=20)
    r = rc.kinematic(sx, sz, steer, seg, 2.0, device=True)
    assert np.array_equal(out.view(np.uint32), r.view(np.uint32))
    assert probes > 0


def test_kinematic_probe_count_equals_reference_algorithm(gpu, orc):
    cls, _, _ = synth.c0_request(3)
    heading, sx, sz, steer, seg = synth.candidates(4000, W, H, 7)
    fr, ctx = ctx_for(gpu, cls, heading)
    out, probes = ctx.kinematic(sx, sz, steer, seg, 2.0)
    orc.set_fp_mode(orc.FP_DEVICE)
    try:
        g = orc.Graph(W, H, 34.56, 34.56, 40.0, 5.4, -1.0, (22, 40))
        g.g.pp.lr, g.g.pp.max_steer_rad = LR, MS
        g.heading[:] = heading
        od, pr, _ = g.kinematic_batch(orc.Frame(cls, synth.CLASS_COSTS), sx, sz, steer, seg, 2.0)
    finally:
        orc.set_fp_mode(orc.FP_HOST)
    same_cells = np.all(od[:, :2] == out[:, :2], axis=1)
    assert same_cells.mean() > 0.999
    if same_cells.all():
        assert probes == int(pr.sum())


def test_kinematic_matches_golden_fixture(gpu):
    d = np.load(os.path.join(GOLD, "kinematic_c0.npz"))
    fr = gpu.SearchFrame(class_ids=d["cls"], class_costs=synth.CLASS_COSTS)
    ctx = gpu.Candidates(fr, min_dist=(22, 40), max_steering_rad=float(d["max_steer"]),
                         lr_m=float(d["lr"]), heading_grid=d["heading"])
    out, _ = ctx.kinematic(d["sx"], d["sz"], d["steer"], d["length"], float(d["velocity"]))
    gold = d["out"]
    # cells and feasibility exact; float fields within the FP32 tolerance
    # (the fixture is the reference's host build, the GPU fuses multiply-adds)
    assert np.array_equal(out[:, :2], gold[:, :2])
    ok = gold[:, 0] >= 0
    assert np.allclose(out[ok, 3], gold[ok, 3], atol=1e-5, rtol=0)
    assert np.allclose(out[ok, 2], gold[ok, 2], atol=1e-4, rtol=1e-5)


def test_pose_error_against_fp64_integrator(gpu, ref, orc):
    """Integrated poses on an open frame (1-cell footprint, paths run to the
    frame edge): bit-exact against the reference's kernel, and the error of
    that FP32 arithmetic against an FP64 integrator of the same bicycle model
    stated and bounded.  FP32 accumulation over up to ~200 steps of a heading
    near pi costs ~2.5e-5 rad in the reference itself, so the FP64 bound on
    heading is 5e-5 rad; positions stay within 1e-4 m."""
    cls = np.zeros((H, W), np.uint8)
    heading, sx, sz, steer, seg = synth.candidates(2000, W, H, 9)
    fr, ctx = ctx_for(gpu, cls, heading, min_dist=(0, 0))
    out, _ = ctx.kinematic(sx, sz, steer, seg, 2.0)
    rc = ref.RefCase(ref.Frame(cls, synth.CLASS_COSTS), heading=heading, max_steer_rad=MS, lr=LR)
    r = rc.kinematic(sx, sz, steer, seg, 2.0, device=True)
    assert np.array_equal(out.view(np.uint32), r.view(np.uint32))
    g = orc.Graph(W, H, 34.56, 34.56, 40.0, 5.4, -1.0, (0, 0))
    g.g.pp.lr, g.g.pp.max_steer_rad = LR, MS
    g.heading[:] = heading
    # the step count of each candidate from the oracle in device arithmetic;
    # candidates whose end cell differs there (a corner touched in one
    # rounding and not the other) are left out of the FP64 comparison
    orc.set_fp_mode(orc.FP_DEVICE)
    try:
        od, _, steps = g.kinematic_batch(orc.Frame(cls, synth.CLASS_COSTS), sx, sz, steer, seg, 2.0)
    finally:
        orc.set_fp_mode(orc.FP_HOST)
    same = np.all(od[:, :2] == out[:, :2], axis=1)
    assert same.mean() > 0.99
    ok = (out[:, 0] >= 0) & same
    p32 = (ctypes.c_double * 3)()
    p64 = (ctypes.c_double * 3)()
    max_m = max_rad = 0.0
    for i in np.nonzero(ok)[0][::3]:
        orc.lib().orc_kinematic_f32_pose(g.p, int(sx[i]), int(sz[i]), float(steer[i]), 2.0,
                                         int(steps[i]), p32)
        orc.lib().orc_kinematic_f64_pose(g.p, int(sx[i]), int(sz[i]), float(steer[i]), 2.0,
                                         int(steps[i]), p64)
        max_rad = max(max_rad, abs(float(out[i, 3]) - p64[2]))
        max_m = max(max_m, math.hypot(p32[0] - p64[0], p32[1] - p64[1]) * synth.M_PER_PX)
    print(f"FP32 kinematic pose vs FP64: max {max_m:.2e} m, {max_rad:.2e} rad")
    assert max_m < 1e-4
    assert max_rad < 5e-5


def test_hermite_bit_exact_vs_reference_kernel(gpu, ref):
    cls, _, _ = synth.c0_request(4)
    fr, ctx = ctx_for(gpu, cls)
    rc = ref.RefCase(ref.Frame(cls, synth.CLASS_COSTS), mdx=11, mdz=20)
    # 65,536 pose pairs at the microbench's 64 samples, and short curves
    for npts, n in ((64, 65536), (2, 8192), (40, 8192)):
        x, z, lh, gx, gz, gh = synth.hermite_pairs(n, W, H, npts, num_points=npts)
        out, _ = ctx.hermite(x, z, lh, gx, gz, gh, 0.8)
        r = rc.direct(0.8, x, z, lh, gx, gz, gh, device=True)
        assert np.array_equal(out.view(np.uint32), r.view(np.uint32)), npts
        out2, _ = ctx.hermite(x, z, lh, gx, gz, gh, 0.285)
        r2 = rc.direct(0.285, x, z, lh, gx, gz, gh, device=True)
        assert np.array_equal(out2.view(np.uint32), r2.view(np.uint32)), npts


def test_hermite_matches_golden_fixture(gpu):
    d = np.load(os.path.join(GOLD, "hermite_c0.npz"))
    fr = gpu.SearchFrame(class_ids=d["cls"], class_costs=synth.CLASS_COSTS)
    ctx = gpu.Candidates(fr, min_dist=(22, 40), max_steering_rad=MS, lr_m=LR)
    out, _ = ctx.hermite(d["x"], d["z"], d["lh"], d["gx"], d["gz"], d["gh"], float(d["max_curvature"]))
    assert np.array_equal(out >= 0, d["out"] >= 0)
    ok = d["out"] >= 0
    assert np.array_equal(out[ok], d["out"][ok])  # costs are integer counts


def test_feasible_bit_exact(gpu, ref):
    d = np.load(os.path.join(GOLD, "feasible_c0.npz"))
    fr = gpu.SearchFrame(class_ids=d["cls"], class_costs=synth.CLASS_COSTS)
    ctx = gpu.Candidates(fr, min_dist=(22, 40), max_steering_rad=MS, lr_m=LR)
    out, _ = ctx.feasible(d["x"], d["z"], d["a"])
    assert np.array_equal(out, d["out"])
    rc = ref.RefCase(ref.Frame(d["cls"], synth.CLASS_COSTS), mdx=11, mdz=20)
    assert np.array_equal(out, rc.feasible(d["x"], d["z"], d["a"], device=True))


def test_edge_cases(gpu):
    # empty input, out-of-frame cells rejected, footprint over the frame edge
    cls = np.zeros((64, 64), np.uint8)
    fr, ctx = ctx_for(gpu, cls, min_dist=(8, 8))
    e = np.zeros(0, np.int32)
    out, pr = ctx.kinematic(e, e, np.zeros(0, np.float32), np.zeros(0, np.float32), 1.0)
    assert out.shape == (0, 4) and pr == 0
    with pytest.raises(gpu.FastRRTError):
        ctx.kinematic(np.array([64], np.int32), np.array([0], np.int32), np.zeros(1, np.float32),
                      np.full(1, 10, np.float32), 1.0)
    out, _ = ctx.feasible(np.array([0, 63], np.int32), np.array([0, 63], np.int32),
                          np.array([0.3, -2.0], np.float32))
    assert out.tolist() == [1, 1]
