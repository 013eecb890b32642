"""The oracle against the reference's own functions compiled for the host
(oracle/_ref), on seeded random inputs: bit-exact in host arithmetic."""
import math

import numpy as np

from fastrrt_b200 import synth


def test_kinematic_matches_reference_host(ref):
    cls, _, _ = synth.c0_request(7)
    fr = ref.Frame(cls, synth.CLASS_COSTS)
    heading, sx, sz, steer, seg = synth.candidates(4000, 256, 256, 21)
    g = ref.Graph(256, 256, 34.56, 34.56, 40.0, 5.4, -1.0, (22, 40))
    g.heading[:] = heading
    out, _, _ = g.kinematic_batch(fr, sx, sz, steer, seg, 2.0)
    rc = ref.RefCase(fr, heading=heading, max_steer_rad=g.g.pp.max_steer_rad, lr=g.g.pp.lr,
                     mdx=11, mdz=20)
    r = rc.kinematic(sx, sz, steer, seg, 2.0)
    assert np.array_equal(out.view(np.uint32), r.view(np.uint32))


def test_kinematic_with_ego_box_and_velocity(ref):
    cls, _, _ = synth.c0_request(8)
    fr = ref.Frame(cls, synth.CLASS_COSTS)
    heading, sx, sz, steer, seg = synth.candidates(2000, 256, 256, 22)
    g = ref.Graph(256, 256, 34.56, 34.56, 30.0, 4.0, -1.0, (10, 18), lb=(119, 148), ub=(137, 108))
    g.heading[:] = heading
    out, _, _ = g.kinematic_batch(fr, sx, sz, steer, seg, 1.0)
    rc = ref.RefCase(fr, heading=heading, max_steer_rad=g.g.pp.max_steer_rad, lr=g.g.pp.lr,
                     mdx=5, mdz=9, lb=(119, 148), ub=(137, 108))
    r = rc.kinematic(sx, sz, steer, seg, 1.0)
    assert np.array_equal(out.view(np.uint32), r.view(np.uint32))


def test_direct_connection_matches_reference_host(ref):
    cls, _, _ = synth.c0_request(9)
    fr = ref.Frame(cls, synth.CLASS_COSTS)
    g = ref.Graph(256, 256, 34.56, 34.56, 40.0, 5.4, -1.0, (22, 40))
    for npts in (2, 20, 64):
        x, z, lh, gx, gz, gh = synth.hermite_pairs(1000, 256, 256, npts, num_points=npts)
        out, _ = g.direct_batch(fr, 0.8, x, z, lh, gx, gz, gh)
        rc = ref.RefCase(fr, mdx=11, mdz=20)
        r = rc.direct(0.8, x, z, lh, gx, gz, gh)
        assert np.array_equal(out.view(np.uint32), r.view(np.uint32)), npts


def test_feasible_and_heading_match_reference_host(ref):
    cls, _, _ = synth.c0_request(10)
    fr = ref.Frame(cls, synth.CLASS_COSTS)
    rng = np.random.default_rng(3)
    x = rng.integers(0, 256, 5000).astype(np.int32)
    z = rng.integers(0, 256, 5000).astype(np.int32)
    a = rng.uniform(-math.pi, math.pi, 5000).astype(np.float32)
    sp = ref.search(256, 256, 22, 40)
    out, _ = ref.feasible_batch(fr, sp, x, z, a)
    assert np.array_equal(out, ref.RefCase(fr, mdx=11, mdz=20).feasible(x, z, a))
    L = ref.ref_lib()
    for i in range(500):
        h = np.float32(ref.lib().orc_compute_heading(int(x[i]), int(z[i]), 128, 0))
        assert h == np.float32(L.ref_h_compute_heading(int(x[i]), int(z[i]), 128, 0))


def test_traversability_bit_quirk(ref):
    # isAllAngleFeasible (path_feasible.cu:13-16) tests bit 0 of frame.z
    cls = np.full((64, 64), 3, np.uint8)
    trav = np.zeros((64, 64), np.int32)
    trav[10, 10] = 1
    trav[20, 20] = 256
    fr = ref.Frame(cls, synth.CLASS_COSTS, trav=trav)
    sp = ref.search(64, 64, 4, 4)
    out, _ = ref.feasible_batch(fr, sp, np.array([10, 20], np.int32), np.array([10, 20], np.int32),
                                np.zeros(2, np.float32))
    assert out.tolist() == [1, 0]
    assert out.tolist() == ref.RefCase(fr, mdx=2, mdz=2).feasible(np.array([10, 20], np.int32),
                                                                   np.array([10, 20], np.int32),
                                                                   np.zeros(2, np.float32)).tolist()
