"""The oracle (host arithmetic) against golden vectors produced by the
reference's own host-compiled functions (tests/golden/make_golden.py) and
its own Python curve-quality code (tests/golden/make_curve_quality.py)."""
import math
import os

import numpy as np
import pytest

from fastrrt_b200 import synth
from oracle import curve_quality as Q

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLD, name))


def test_kinematic_golden(orc):
    d = load("kinematic_c0.npz")
    fr = orc.Frame(d["cls"], synth.CLASS_COSTS)
    g = orc.Graph(256, 256, 34.56, 34.56, 40.0, 5.4, -1.0, (22, 40))
    g.g.pp.lr = float(d["lr"])
    g.g.pp.max_steer_rad = float(d["max_steer"])
    g.heading[:] = d["heading"]
    out, _, _ = g.kinematic_batch(fr, d["sx"], d["sz"], d["steer"], d["length"], float(d["velocity"]))
    assert np.array_equal(out.view(np.uint32), d["out"].view(np.uint32))
    assert 0.2 < (d["out"][:, 0] >= 0).mean() < 0.9


def test_hermite_golden(orc):
    d = load("hermite_c0.npz")
    fr = orc.Frame(d["cls"], synth.CLASS_COSTS)
    g = orc.Graph(256, 256, 34.56, 34.56, 40.0, 5.4, -1.0, (22, 40))
    out, _ = g.direct_batch(fr, float(d["max_curvature"]), d["x"], d["z"], d["lh"], d["gx"], d["gz"],
                            d["gh"])
    assert np.array_equal(out.view(np.uint32), d["out"].view(np.uint32))
    assert (d["out"] >= 0).any() and (d["out"] < 0).any()


def test_feasible_golden(orc):
    d = load("feasible_c0.npz")
    fr = orc.Frame(d["cls"], synth.CLASS_COSTS)
    sp = orc.search(256, 256, 22, 40)
    out, _ = orc.feasible_batch(fr, sp, d["x"], d["z"], d["a"])
    assert np.array_equal(out, d["out"])


def test_graph_dump_fixtures_stay_dag_after_solve(orc):
    # assertGraphRemainsDAGAfterCollision (test_graph_solve_collisions.cpp:144-176)
    # on the reference's recorded graph states (unittests/src/test_data)
    d = load("graph_dumps.npz")
    for name in d.files:
        g = orc.Graph(256, 256, 256.0, 256.0, 40.0, 5.412658773, -1.0, (0, 0))
        for x, z, h, t, px, pz, _, c in d[name]:
            x, z, t, px, pz = int(x), int(z), int(t), int(px), int(pz)
            if t == 1:
                g.add(x, z, h, px, pz, c)
            elif t == 2:
                g.add_temporary(x, z, h, px, pz, c)
            elif t == 4:
                g.add(x, z, h, px, pz, c)
                g.set_collision(x, z, px, pz, h, c)
        g.solve_collisions()
        assert g.consistent(), name


def test_curve_quality_golden():
    """length, jerk and tangential discontinuity of the curve-quality
    restatement against the reference's CurveAssessment on 101 curves,
    including the short ones where its window arithmetic raises"""
    d = load("curve_quality.npz")
    offs = np.concatenate([[0], np.cumsum(d["lengths"])])
    raised = 0
    for k in range(len(d["lengths"])):
        cells = d["cells"][offs[k]:offs[k + 1]]
        curve = [(float(p[0]), float(p[1])) for p in cells]
        assert Q.curve_length(curve) == pytest.approx(d["total_length"][k], rel=1e-12, abs=0)
        if math.isnan(d["jerk"][k]):
            raised += 1
            with pytest.raises(IndexError):
                Q.jerk(curve)
        else:
            # the reference sums |j| one term after another, numpy pairwise
            assert Q.jerk(curve) == pytest.approx(d["jerk"][k], rel=1e-9, abs=1e-12)
        if d["tan"][k] < 0:
            with pytest.raises(IndexError):
                Q.tangential_discontinuity(curve, float(d["start_heading"][k]))
        else:
            assert Q.tangential_discontinuity(curve, float(d["start_heading"][k])) == bool(d["tan"][k])
    # the fixture holds both answers and the raising cases
    assert raised >= 1
    assert 0 < (d["tan"] == 1).sum() < (d["tan"] >= 0).sum()


def test_interpolation_golden(orc):
    """the oracle's Hermite interpolation of planned paths against the
    reference's own interpolate() (src/interpolation.cpp built with g++,
    tests/golden/make_interpolation.py): the same cells and headings on 63
    control-point paths, including sharp turns, paths that leave the frame,
    repeated points and two-point paths"""
    d = load("interpolation.npz")
    W, H = int(d["width"]), int(d["height"])
    pi = np.concatenate([[0], np.cumsum(d["n_in"])])
    po = np.concatenate([[0], np.cumsum(d["n_out"])])
    total = 0
    for k in range(len(d["n_in"])):
        path = d["paths"][pi[k]:pi[k + 1]]
        want = d["out"][po[k]:po[k + 1]]
        got = orc.interpolate(path, W, H)
        assert got.shape == want.shape, k
        assert np.array_equal(got[:, :2], want[:, :2]), k
        assert np.array_equal(got[:, 2].view(np.uint32), want[:, 2].view(np.uint32)), k
        total += len(want)
    assert total > 5000
