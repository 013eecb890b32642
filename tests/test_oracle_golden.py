"""Known answers of the reference's own unit tests (unittests/src/*.cpp),
checked on the CPU oracle."""
import math

import numpy as np
import pytest

PHYS_SIZE = 34.641016151377535
COSTS6 = np.array([0, 1, 2, 3, 4, -1], np.float32)


def empty_frame(orc, W=256, H=256, costs=COSTS6):
    return orc.Frame(np.zeros((H, W), np.uint8), costs)


def test_graph_node_derivation_straight(orc):
    # test_graph_node_derivation.cpp:13-35: (128,128,0 deg), 49 px at 1 m/s ends at (128,78)
    fr = empty_frame(orc)
    g = orc.Graph(256, 256, 256.0, 256.0, 40.0, 5.412658773, -1.0, (0, 0))
    g.add(128, 128, 0.0, -1, -1, 0)
    r = g.derive(fr, 128, 128, 0.0, 49, 1.0)
    assert (r.x, r.y) == (128.0, 78.0)
    assert r.w == 0.0
    assert r.z == 50.0  # one cost unit per new cell: TO_INT(49) + 1 cells


def test_graph_node_derivation_delocated(orc):
    # test_graph_node_derivation.cpp:89-111: (50,200) -> (50,150)
    fr = empty_frame(orc)
    g = orc.Graph(256, 256, 256.0, 256.0, 40.0, 5.412658773, -1.0, (0, 0))
    g.add(50, 200, 0.0, -1, -1, 0)
    r = g.derive(fr, 50, 200, 0.0, 49, 1.0)
    assert (r.x, r.y) == (50.0, 150.0) and r.w == 0.0


def _derive_restated(x0, z0, h0, path_size, steering, v, lr):
    """the test's own restated integrator (test_graph_node_derivation.cpp:113-191)
    in float32 with a (128,128) waypoint origin"""
    f32 = np.float32
    steer = f32(math.tan(f32(steering)))
    dt = f32(0.1)
    ds = f32(f32(v) * dt)
    beta = f32(math.atan(f32(steer / f32(2))))
    hif = f32(float(f32(f32(ds * f32(math.cos(beta))) * steer)) / (2 * lr))
    x = f32(128 - z0)
    y = f32(x0 - 128)
    heading = f32(h0)
    max_size = int(f32(path_size)) + 1
    size = 0
    last = (x0, z0)
    while size < max_size:
        a = f32(heading + beta)
        x = f32(x + f32(ds * f32(math.cos(a))))
        y = f32(y + f32(ds * f32(math.sin(a))))
        heading = f32(heading + hif)
        p = (int(128.0 + float(y)), int(128.0 - float(x)))
        if p == last:
            continue
        if not (0 <= p[0] < 256 and 0 <= p[1] < 256):
            break
        size += 1
        last = p
    return last[0], last[1], float(heading)


def test_graph_node_derivation_curvy_sweep(orc):
    # test_graph_node_derivation.cpp:193-224: heading -180..180 x steering -40..40 step 18
    fr = empty_frame(orc)
    lr = 0.5 * 5.412658773
    mism = 0
    total = 0
    for a in range(-180, 181, 4):
        for i in range(-40, 41, 18):
            g = orc.Graph(256, 256, 256.0, 256.0, 40.0, 5.412658773, -1.0, (0, 0))
            g.add(100, 200, math.radians(a), -1, -1, 0)
            r = g.derive(fr, 100, 200, float(np.float32(math.radians(i))), 15, 1.0)
            ex, ez, eh = _derive_restated(100, 200, float(np.float32(math.radians(a))), 15,
                                          math.radians(i), 1.0, lr)
            total += 1
            if (int(r.x), int(r.y)) != (ex, ez) or abs(r.w - eh) > 1e-5:
                mism += 1
    # libm cosf/sinf and correctly-rounded float32(cos(x)) agree to the last
    # bit almost always; the end cell and heading must match everywhere here
    assert mism == 0, f"{mism}/{total}"


def test_kinematic_connection_after_derivation(orc):
    # test_kinematics.cpp:51-72: derive 20 deg / 50 px / 2 m/s, then checkFeasibleConnection
    fr = empty_frame(orc, costs=np.array([0, 1, 2, 3, 4, 5], np.float32))
    g = orc.Graph(256, 256, PHYS_SIZE, PHYS_SIZE, 40.0, 5.412658773, -1.0, (0, 0))
    g.add(128, 128, 0.0, -1, -1, 0)
    r = g.derive(fr, 128, 128, math.radians(20), 50, 2)
    fh, pc = orc.C.c_double(), orc.C.c_double()
    ok = orc.lib().orc_kinematic_connection(g.p, orc.C.byref(fr.s), 128, 128, int(r.x), int(r.y), 2.0,
                                            orc.C.byref(fh), orc.C.byref(pc))
    assert ok == 1


def test_physical_and_search_params(orc):
    # test_graph.cpp:23-50
    pp = orc.OrcPhysical()
    orc.lib().orc_physical_params(orc.C.byref(pp), 100, 100, 11.1, 11.2, math.radians(21), 11.3, -1.0)
    assert pp.rate_w == pytest.approx(100 / 11.1, rel=1e-6)
    assert pp.inv_rate_w == pytest.approx(11.1 / 100, rel=1e-6)
    assert pp.rate_h == pytest.approx(100 / 11.2, rel=1e-6)
    assert pp.lr == pytest.approx(11.3 / 2, rel=1e-6)
    assert pp.max_steer_deg == pytest.approx(21, rel=1e-6)
    sp = orc.search(100, 100, 4, 6, (4, 5), (6, 7))
    assert (sp.mdx, sp.mdz, sp.lbx, sp.lbz, sp.ubx, sp.ubz) == (2, 3, 4, 5, 6, 7)


def test_basic_graph_features(orc):
    # test_graph.cpp:132-205
    g = orc.Graph(100, 100)
    assert g.count() == 0
    g.add(50, 50, 0.12, -1, -1, 0)
    g.add(50, 45, 0.12, 50, 50, 10)
    g.add(55, 40, 0.12, 50, 45, 10)
    g.add(20, 35, 0.12, 50, 45, 10)
    g.add(20, 15, 0.12, 20, 35, 10)
    g.add(20, 5, 0.12, 20, 15, 10)
    g.add(20, 0, 0.12, 20, 5, 10)
    assert g.count() == 7
    orc.lib().orc_graph_remove(g.p, 20, 0)
    assert g.count() == 6
    orc.lib().orc_graph_remove(g.p, 0, 0)
    orc.lib().orc_graph_remove(g.p, 999, -999)
    assert g.count() == 6
    assert g.parent(20, 0) == (-1, -1)
    assert g.parent(2000, -1000) == (-1, -1)
    assert g.parent(20, 5) == (20, 15)


def test_add_clear(orc):
    # test_graph.cpp:90-110
    g = orc.Graph(100, 100)
    g.add(10, 10, 0.2, -1, -1, 101.2)
    assert g.count_all() == 1 and g.type_at(10, 10) == orc.NODE
    g.clear()
    assert g.count_all() == 0
    g.add_temporary(10, 10, 0.2, -1, -1, 101.2)
    assert g.count_all() == 1 and g.type_at(10, 10) == orc.TEMP


def _tree(orc):
    g = orc.Graph(256, 256, 256.0, 256.0, 40.0, 5.412658773, -1.0, (0, 0))
    return g


def test_single_collision_solve(orc):
    # test_graph_solve_collisions.cpp:14-51
    g = _tree(orc)
    g.add(128, 128, 0, -1, -1, 0)
    g.add(100, 100, 0, 128, 128, 0)
    g.add(135, 100, 0, 128, 128, 0)
    g.add(110, 70, 0, 135, 100, 0)
    g.add(145, 70, 0, 135, 100, 0)
    assert (g.child_at(128, 128), g.child_at(100, 100), g.child_at(135, 100)) == (2, 0, 2)
    g.set_collision(110, 70, 100, 100, 0, 0)
    g.solve_collisions()
    assert (g.child_at(128, 128), g.child_at(100, 100), g.child_at(135, 100)) == (2, 1, 1)
    assert g.consistent()
    assert g.parent(128, 128) == (-1, -1)
    assert g.parent(100, 100) == (128, 128)
    assert g.parent(135, 100) == (128, 128)
    assert g.parent(110, 70) == (100, 100)
    assert g.parent(145, 70) == (135, 100)
    assert g.type_at(110, 70) == orc.NODE


def test_collision_solve_graph_erase(orc):
    # test_graph_solve_collisions.cpp:53-96
    g = _tree(orc)
    g.add(128, 128, 0, -1, -1, 0)
    g.add(100, 100, 0, 128, 128, 0)
    g.add(135, 100, 0, 128, 128, 0)
    g.add(110, 70, 0, 135, 100, 0)
    g.add(90, 50, 0, 110, 70, 0)
    g.add(40, 35, 0, 110, 70, 0)
    g.add(145, 70, 0, 135, 100, 0)
    g.set_collision(110, 70, 100, 100, 0, 0)
    g.solve_collisions()
    assert g.consistent()
    assert g.type_at(90, 50) == orc.NULL and g.type_at(40, 35) == orc.NULL
    assert g.type_at(110, 70) == orc.NODE
    assert [g.child_at(*p) for p in [(128, 128), (100, 100), (135, 100), (110, 70), (145, 70)]] == \
        [2, 1, 1, 0, 0]


def test_dual_collision(orc):
    # test_graph_solve_collisions.cpp:98-142
    g = _tree(orc)
    g.add(128, 128, 0, -1, -1, 0)
    g.add(100, 100, 0, 128, 128, 0)
    g.add(135, 100, 0, 128, 128, 0)
    g.add(110, 70, 0, 135, 100, 0)
    g.add(90, 50, 0, 110, 70, 0)
    g.add(40, 35, 0, 110, 70, 0)
    g.add(145, 70, 0, 135, 100, 0)
    g.add(185, 60, 0, 135, 100, 0)
    g.set_collision(110, 70, 100, 100, 0, 0)
    g.set_collision(90, 50, 185, 60, 0, 0)
    g.solve_collisions()
    assert [g.child_at(*p) for p in [(128, 128), (100, 100), (135, 100), (110, 70), (145, 70),
                                      (90, 50), (185, 60)]] == [2, 1, 2, 0, 0, 0, 1]
    assert g.consistent()
    assert g.type_at(90, 50) == orc.NODE and g.parent(90, 50) == (185, 60)
    assert g.type_at(40, 35) == orc.NULL
    assert g.type_at(110, 70) == orc.NODE and g.parent(110, 70) == (100, 100)


def test_log_collision_replay(orc):
    # test_graph_solve_collisions.cpp:144-191 (inline log of a collision)
    data = [(148, 116, 1.62867, 2, 133, 120, 0, 31), (140, 115, 0.97043, 1, 133, 120, 0, 23),
            (129, 123, 0.14363, 4, 128, 128, 0, 6), (128, 128, 0, 1, -1, -1, 0, 0),
            (130, 117, 0.186008, 2, 129, 123, 0, 12), (133, 120, 0.690726, 1, 128, 128, 0, 12)]
    g = _tree(orc)
    for x, z, h, t, px, pz, _, c in data:
        if t == 1:
            g.add(x, z, h, px, pz, c)
        elif t == 2:
            g.add_temporary(x, z, h, px, pz, c)
        elif t == 4:
            g.add(x, z, h, px, pz, c)
            g.set_collision(x, z, px, pz, h, c)
    assert g.consistent()
    g.solve_collisions()
    assert g.consistent()


@pytest.mark.parametrize("case,expect", [
    ("empty", True), ("one", True), ("two", True), ("circle", False), ("two_circle", False),
    ("self", False), ("branches", True)])
def test_dag_consistency(orc, case, expect):
    # test_graph_dag_consistency.cpp:14-88
    g = _tree(orc)
    if case != "empty":
        g.add(128, 128, 0, -1, -1, 0)
    if case == "two":
        g.add(128, 78, 0, 128, 128, 0)
    elif case == "circle":
        g.add(128, 48, 0, 78, 90, 0)
        g.add(78, 90, 0, 128, 78, 0)
        g.add(128, 78, 0, 128, 48, 0)
    elif case == "two_circle":
        g.add(78, 90, 0, 128, 78, 0)
        g.add(128, 78, 0, 78, 90, 0)
    elif case == "self":
        g.add(78, 90, 0, 78, 90, 0)
    elif case == "branches":
        g.add(100, 100, 0, 128, 128, 0)
        g.add(135, 100, 0, 128, 128, 0)
        g.add(110, 70, 0, 135, 100, 0)
        g.add(145, 70, 0, 135, 100, 0)
    assert g.consistent() == expect


def test_goal_reached_and_best_node(orc):
    # test_graph_best_node.cpp:11-61
    fr = empty_frame(orc, costs=np.array([0, 1, 2, 3, 4, 5], np.float32))
    g = orc.Graph(256, 256, PHYS_SIZE, PHYS_SIZE, 40.0, 5.412658773, -1.0, (0, 0))
    tenth = float(np.float32(math.radians(10)))
    assert not g.goal_reached(fr, 128, 0, tenth, 5.0, 1.0)
    g.add(128, 128, 0, -1, -1, 0)
    g.add(128, 3, tenth, 128, 128, 10)
    assert g.goal_reached(fr, 128, 0, tenth, 5.0, 1.0)
    g2 = orc.Graph(256, 256, PHYS_SIZE, PHYS_SIZE, 40.0, 5.412658773, -1.0, (0, 0))
    g2.add(128, 128, 0, -1, -1, 0)
    g2.add(128, 3, 0, 128, 128, 10)
    g2.add(108, 3, 0, 128, 128, 10)
    g2.add(158, 3, 0, 128, 128, 10)
    assert g2.best_node(fr, 0.0, 50.0, 128, 0, 1.0) == (128, 3)


def _wall_frame(orc):
    cls = np.zeros((256, 256), np.uint8)
    cls[100, :] = 5
    cls[100, 127:130] = 0
    return orc.Frame(cls, COSTS6)


def test_direct_goal_narrow_space(orc):
    # test_graph_direct_goal_connection.cpp:100-193: only x = 128 connects on row 100
    fr = _wall_frame(orc)
    g = orc.Graph(256, 256, 256.0, 256.0, 40.0, 5.412658773, -1.0, (2, 2))
    g.add(128, 128, 0, -1, -1, 0)
    g.process_direct_goal(fr, 128, 0, 0.0)
    row = g.gd_flag.reshape(256, 256)[100]
    assert [i for i in range(256) if row[i] > 0] == [128]


def test_direct_goal_unfeasible_goal(orc):
    # test_graph_direct_goal_connection.cpp:195-208: goal cell is an obstacle
    cls = np.ones((256, 256), np.uint8)
    cls[0, 128] = 0
    fr = orc.Frame(cls, np.array([-1, 1, 2, 3, 4, 5], np.float32))
    g = orc.Graph(256, 256, 256.0, 256.0, 40.0, 5.412658773, -1.0, (2, 2))
    g.add(128, 128, 0, -1, -1, 0)
    g.process_direct_goal(fr, 128, 0, 0.0)
    assert not np.any(g.gd_flag.reshape(256, 256)[100] > 0)


def test_hermite_can_connect(orc):
    # test_graph_can_connect_hermite.cpp:31-109 (canConnectToGoal: obstacle goal -> false;
    # otherwise the Hermite test with the frame's distance channel)
    costs = np.array([0, 1, 2, 3, 4, 5], np.float32)
    fr = empty_frame(orc, costs=costs)
    g = orc.Graph(256, 256, 256.0, 256.0, 40.0, 5.412658773, -1.0, (0, 0))
    g.add(128, 128, 0, -1, -1, 0)
    dist = np.zeros((256, 256), np.float32)
    zz, xx = np.mgrid[0:256, 0:256]
    dist[:] = np.sqrt((xx - 128) ** 2 + (zz - 0) ** 2).astype(np.float32)
    d = dist.reshape(-1)
    r = orc.lib().orc_hermite_test(g.p, orc.C.byref(fr.s), d.ctypes.data_as(orc.C.POINTER(orc.C.c_float)),
                                   128, 128, 128, 0, 0.0, 0, g.g.pp.max_curvature, None)
    assert r >= 0
    blocked = np.zeros((256, 256), np.uint8)
    fr2 = orc.Frame(blocked, np.array([-1, 1, 2, 3, 4, 5], np.float32))
    assert fr2.costs[fr2.cls[0, 128]] < 0  # isObstacle(goal) -> canConnectToGoal is false


def test_philox_known_answer(orc):
    # Random123 known-answer vector for philox4x32-10 (counter 0, key 0)
    out = (orc.C.c_uint32 * 4)()
    orc.lib().orc_philox4x32(0, 0, 0, 0, 0, 0, out)
    assert list(out) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    orc.lib().orc_philox4x32(0xffffffff, 0xffffffff, 0xffffffff, 0xffffffff,
                             0xffffffff, 0xffffffff, out)
    assert list(out) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
