"""The device validator on bad inputs.  The graph check (k_dag) against the
reference's own consistency cases (unittests/src/test_graph_dag_consistency.
cpp:14-88: empty, one and two nodes, a three-node cycle, a two-node cycle, a
node that is its own parent, a branching DAG) and its parent-type rule
(src/graph_check_dag_consistency.cpp:59-66); the path check (k_path_check)
on a planned path and on copies of it broken one way each."""
import os

import numpy as np
import pytest

from fastrrt_b200 import synth

pytestmark = pytest.mark.gpu
COSTS = synth.CLASS_COSTS
W = H = 256
NULL, NODE, TEMP, COLLISION, CONNECT = 0, 1, 2, 4, 5

# (name, [(x, z, parent_x, parent_z, type)], consistent)
DAG_CASES = [
    ("empty", [], True),
    ("one node", [(128, 128, -1, -1, NODE)], True),
    ("two nodes", [(128, 128, -1, -1, NODE), (128, 78, 128, 128, NODE)], True),
    ("three-node cycle", [(128, 128, -1, -1, NODE), (128, 48, 78, 90, NODE), (78, 90, 128, 78, NODE),
                          (128, 78, 128, 48, NODE)], False),
    ("two-node cycle", [(128, 128, -1, -1, NODE), (78, 90, 128, 78, NODE), (128, 78, 78, 90, NODE)],
     False),
    ("self parent", [(128, 128, -1, -1, NODE), (78, 90, 78, 90, NODE)], False),
    ("branching DAG", [(128, 128, -1, -1, NODE), (100, 100, 128, 128, NODE), (135, 100, 128, 128, NODE),
                       (110, 70, 135, 100, NODE), (145, 70, 135, 100, NODE)], True),
    # parents must be NODE, COLLISION or CONNECT_TO_GOAL cells
    ("parent is a TEMP cell", [(128, 128, -1, -1, TEMP), (100, 100, 128, 128, NODE)], False),
    ("parent is a NULL cell", [(100, 100, 128, 128, NODE)], False),
    ("parent is a COLLISION cell", [(128, 128, -1, -1, COLLISION), (100, 100, 128, 128, NODE)], True),
    ("parent is a CONNECT_TO_GOAL cell", [(128, 128, -1, -1, CONNECT), (100, 100, 128, 128, NODE)], True),
]


def planner(F, cls, seed):
    fr = F.SearchFrame(class_ids=cls, class_costs=COSTS)
    p = F.FastRRT(search_frame=fr, perception_width_m=34.56, perception_height_m=34.56,
                  max_steering_angle_deg=40, vehicle_length_m=5.4, timeout_ms=-1,
                  min_dist_x=22, min_dist_z=40, path_costs=COSTS, seed=seed)
    return p, fr


def write_dump(path, nodes):
    """a graph dump (the text format of save_current_graph_state) holding
    only `nodes`"""
    rows = [[-1, -1, NULL, 0] for _ in range(W * H)]
    for x, z, px, pz, t in nodes:
        rows[z * W + x] = [px, pz, t, 0]
    with open(path, "w") as f:
        for px, pz, t, c in rows:
            f.write(f"{px} {pz} {t} {c} 0.000000 0.000000 0.000000 0.000000\n")


@pytest.mark.parametrize("name,nodes,want", DAG_CASES, ids=[c[0] for c in DAG_CASES])
def test_graph_check_reference_cases(gpu, orc, tmp_path, name, nodes, want):
    cls = np.zeros((H, W), np.uint8)
    p, fr = planner(gpu, cls, 1)
    p.set_plan_data(fr, (128, 128, 0.0), (128, 0, 0.0), 2.0)
    p.search_init()
    f = str(tmp_path / "graph.txt")
    write_dump(f, nodes)
    p.load_graph_state(f)
    assert p.check_graph_is_consistent() == want, name
    if all(t == NODE for *_, t in nodes):
        # the oracle's restatement of the same check agrees
        g = orc.Graph(W, H, 34.56, 34.56, 40.0, 5.4, -1.0, (22, 40))
        for x, z, px, pz, _ in nodes:
            g.add(x, z, 0.0, px, pz, 0.0)
        assert g.consistent() == want, name


@pytest.fixture(scope="module")
def planned(gpu):
    """a planned C0 path of at least five waypoints (the first seed from 4
    that gives one) and its planner"""
    for seed in range(4, 64):
        cls, start, goal = synth.c0_request(seed)
        p, fr = planner(gpu, cls, seed)
        p.set_plan_data(fr, start, goal, 2.0)
        p.search_init()
        n = 0
        while not p.goal_reached() and n < 200:
            n += 1
            p.loop(False)
        if p.goal_reached() and len(p.get_planned_path_array()) >= 5:
            return p, cls, start, goal, p.get_planned_path_array()
    pytest.fail("no C0 seed in 4..63 planned a path of five waypoints")


def test_path_check_accepts_the_planned_path(planned):
    p, _, _, _, path = planned
    assert len(path) >= 5
    assert p.check_graph_is_consistent()
    assert p.validate_path(path)


def test_path_check_rejects_broken_paths(planned):
    p, _, _, _, path = planned
    k = len(path) // 2
    broken = {
        "does not start at the start": path[1:],
        "repeats a cell": np.insert(path, k, path[k], axis=0),
        "skips a waypoint (parent link)": np.delete(path, k, axis=0),
        "two waypoints swapped": path[[*range(k - 1), k, k - 1, *range(k + 1, len(path))]],
        "waypoint outside the frame": np.where(np.arange(len(path))[:, None] == k,
                                               [[W + 40, path[k, 1], path[k, 2]]], path),
        "ends off the goal heading": path + np.where(np.arange(len(path))[:, None] == len(path) - 1,
                                                     [[0, 0, 1.0]], 0),
        "one waypoint": path[:1],
        "empty": path[:0],
    }
    for name, bad in broken.items():
        assert not p.validate_path(np.asarray(bad, np.float32)), name


def test_path_check_rejects_a_blocked_footprint(gpu, planned):
    # the same graph and path over a frame with an obstacle on a waypoint
    p, cls, start, goal, path = planned
    k = len(path) // 2
    x, z = int(path[k, 0]), int(path[k, 1])
    blocked = cls.copy()
    blocked[max(0, z - 2):z + 3, max(0, x - 2):x + 3] = 3  # class cost -1: obstacle
    fr = gpu.SearchFrame(class_ids=blocked, class_costs=COSTS)
    p.set_plan_data(fr, start, goal, 2.0)
    try:
        assert not p.validate_path(path)
    finally:
        fr0 = gpu.SearchFrame(class_ids=cls, class_costs=COSTS)
        p.set_plan_data(fr0, start, goal, 2.0)
    assert p.validate_path(path)
