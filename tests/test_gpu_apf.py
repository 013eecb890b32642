"""Artificial potential fields (apf.cu:23-154) on the planner's intrinsic
costs: bit-exact against a numpy restatement of the deterministic order the
library uses (obstacle sets first, then each cell's sources in row-major
order, every operation rounded on its own), and against the reference's own
kernels (oracle/_ref on the same GPU, float atomics in an arbitrary order)
within float rounding on free cells, with every obstacle cell at the set value
plus at most its sources' adds."""
import ctypes as C
import math

import numpy as np
import pytest

from fastrrt_b200 import synth

pytestmark = pytest.mark.gpu
COSTS = synth.CLASS_COSTS
W = H = 128


def apf_numpy(cls, kr, radius, ka, goal, lb=(-1, -1), ub=(-1, -1)):
    f32 = np.float32
    obst = COSTS[cls] < 0
    z, x = np.mgrid[0:H, 0:W]
    ego = (x >= lb[0]) & (x <= ub[0]) & (z >= ub[1]) & (z <= lb[1])
    pad = np.pad(obst, 1, constant_values=True)
    interior = pad[1:-1, :-2] & pad[1:-1, 2:] & pad[:-2, 1:-1] & pad[2:, 1:-1]
    src = obst & ~ego & ~interior
    kh = f32(kr * 0.5)
    v = np.where(obst & ~ego, f32(100) * kh, f32(0)).astype(np.float32)
    srcp = np.pad(src, radius, constant_values=False)
    p0 = f32(radius)
    for dz in range(-radius, radius + 1):
        for dx in range(-radius, radius + 1):
            if dx == 0 and dz == 0:
                continue
            p = np.sqrt(f32(dx * dx + dz * dz))
            if p > p0:
                continue
            f = f32(f32(1) / p) - f32(f32(1) / p0)
            c = f32(f32(kh * f) * f)
            s = srcp[radius + dz:radius + dz + H, radius + dx:radius + dx + W] & ~ego
            v = np.where(s, (v + c).astype(np.float32), v)
    rep = v.copy()
    d2 = ((goal[0] - x) ** 2 + (goal[1] - z) ** 2).astype(np.float32)
    kah = f32(ka * 0.5)
    att = np.where(~obst, (v - np.float32(d2 * kah)).astype(np.float32), v)
    return rep, att, obst, ego, src


def planner(F, cls):
    fr = F.SearchFrame(class_ids=cls, class_costs=COSTS)
    p = F.FastRRT(search_frame=fr, perception_width_m=W * 0.135, perception_height_m=H * 0.135,
                  max_steering_angle_deg=40, vehicle_length_m=5.4, timeout_ms=-1, min_dist_x=22,
                  min_dist_z=40, path_costs=COSTS, seed=1)
    p.set_plan_data(fr, (64, 100, 0.0), (64, 0, 0.0), 2.0)
    p.search_init()
    return p, fr


def test_apf_matches_numpy_restatement(gpu):
    cls = synth.make_frame(41, W, coverage=0.2, start=(64, 100), goal=(64, 0))
    p, fr = planner(gpu, cls)
    assert np.all(p.get_intrinsic_costs() == 0)
    p.compute_apf_repulsion(fr, 2.0, 5)
    rep = p.get_intrinsic_costs()
    want_rep, want_att, obst, _, _ = apf_numpy(cls, 2.0, 5, 1e-4, (64, 0))
    assert np.array_equal(rep.view(np.uint32), want_rep.view(np.uint32))
    assert (rep[~obst] > 0).any()
    # attraction is added ... as the attractive kernel of the reference
    p.compute_apf_attraction(fr, 1e-4, 64, 0)
    att = p.get_intrinsic_costs()
    free = ~obst
    assert np.allclose(att[free], want_att[free], rtol=0, atol=1e-5)
    assert np.array_equal(att[obst].view(np.uint32), want_att[obst].view(np.uint32))


def test_apf_against_reference_kernels(gpu, ref):
    cls = synth.make_frame(42, W, coverage=0.2, start=(64, 100), goal=(64, 0))
    p, fr = planner(gpu, cls)
    p.compute_apf_repulsion(fr, 2.0, 5)
    mine = p.get_intrinsic_costs()
    _, _, obst, _, _ = apf_numpy(cls, 2.0, 5, 0.0, (64, 0))
    L = ref.ref_lib()
    L.cudagraph_initialize.restype = C.c_void_p
    L.cudagraph_initialize.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                                       C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                       C.c_float]
    L.compute_apf_repulsion.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_int]
    L.get_intrinsic_costs.restype = C.POINTER(C.c_float)
    L.get_intrinsic_costs.argtypes = [C.c_void_p]
    head = np.ascontiguousarray(np.concatenate(([len(COSTS)], COSTS)), np.float32)
    g = L.cudagraph_initialize(W, H, W * 0.135, H * 0.135, 40.0, 5.4, 22, 40, -1, -1, -1, -1,
                               head.ctypes.data, -1.0)
    xyz = np.zeros((H, W, 3), np.float32)
    xyz[..., 0] = cls
    xyz = np.ascontiguousarray(xyz.reshape(-1))
    frame = L.ref_frame_new(W, H, xyz, np.ascontiguousarray(COSTS), len(COSTS), -1, -1, -1, -1, 11, 20)
    L.compute_apf_repulsion(g, frame, 2.0, 5)
    ptr = L.get_intrinsic_costs(g)
    theirs = np.ctypeslib.as_array(ptr, (H * W,)).reshape(H, W).copy()
    free = ~obst
    assert np.allclose(mine[free], theirs[free], rtol=1e-5, atol=1e-6)
    # an obstacle cell: the set value, plus some or all of its sources' adds
    set_val = np.float32(100) * np.float32(1.0)
    assert np.all(theirs[obst] >= set_val - 1e-4) and np.all(theirs[obst] <= mine[obst] + 1e-3)
    assert np.all(mine[obst] >= set_val)
