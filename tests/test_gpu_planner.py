"""The whole planner on the GPU against the CPU oracle: the drop-in planner
(FastRRT / loop / path_optimize / get_planned_path) grows the same node grid
and returns the same path as the oracle planner on the same seed, and the
batched planner returns, per request, what the request gives alone."""
import math
import os

import numpy as np
import pytest

from fastrrt_b200 import synth

pytestmark = pytest.mark.gpu
COSTS = synth.CLASS_COSTS
W = H = 256


def gpu_planner(F, cls, seed, **kw):
    fr = F.SearchFrame(class_ids=cls, class_costs=COSTS)
    p = F.FastRRT(search_frame=fr, perception_width_m=34.56, perception_height_m=34.56,
                  max_steering_angle_deg=40, vehicle_length_m=5.4, timeout_ms=-1,
                  min_dist_x=22, min_dist_z=40, path_costs=COSTS, seed=seed, **kw)
    return p, fr


def run_gpu(p, fr, start, goal, max_loops=200, smart=False):
    p.set_plan_data(fr, start, goal, 2.0)
    p.search_init()
    n = 0
    while not p.goal_reached() and n < max_loops:
        n += 1
        if not p.loop(smart):
            break
    return n


def run_oracle(orc, cls, start, goal, seed, loops, smart=False):
    op = orc.Planner(orc.Frame(cls, COSTS), 34.56, 34.56, 40.0, 5.4)
    op.set_plan_data(start, goal, 2.0, (22, 40), seed=seed)
    op.search_init()
    m = 0
    while not op.goal_reached() and m < loops:
        m += 1
        if not op.loop(smart):
            break
    return op, m


def grid_types(nodes):
    g = np.zeros((H, W), np.int32)
    if nodes is not None:
        g[nodes[:, 1], nodes[:, 0]] = nodes[:, 2]
    return g


@pytest.fixture
def dev_orc(orc):
    orc.set_fp_mode(orc.FP_DEVICE)
    yield orc
    orc.set_fp_mode(orc.FP_HOST)


@pytest.mark.parametrize("seed", range(8))
def test_plan_matches_oracle(gpu, dev_orc, seed):
    orc = dev_orc
    cls, start, goal = synth.c0_request(seed)
    p, fr = gpu_planner(gpu, cls, seed)
    n = run_gpu(p, fr, start, goal)
    assert p.goal_reached()
    op, m = run_oracle(orc, cls, start, goal, seed, n)
    assert m == n and op.goal_reached()
    assert p.loop_count() == n
    assert np.array_equal(grid_types(p.export_graph_nodes()), op.type.reshape(H, W))
    path, opath = p.get_planned_path_array(), op.path()
    assert np.array_equal(path[:, :2], opath[:, :2])
    assert np.allclose(path[:, 2], opath[:, 2], atol=1e-5, rtol=0)
    assert op.validate(path)
    assert p.probe_count() > 0
    # path_optimize until it stops changing, on both sides
    k = kk = 0
    while p.path_optimize() and k < 20:
        k += 1
    while op.optimize() and kk < 20:
        kk += 1
    assert k == kk
    po, oo = p.get_planned_path_array(), op.path()
    assert np.array_equal(po[:, :2], oo[:, :2])
    assert op.validate(po)


@pytest.mark.parametrize("seed", [1, 5])
def test_smart_expansion_matches_oracle(gpu, dev_orc, seed):
    cls, start, goal = synth.c0_request(seed)
    p, fr = gpu_planner(gpu, cls, seed)
    n = run_gpu(p, fr, start, goal, smart=True)
    op, m = run_oracle(dev_orc, cls, start, goal, seed, n, smart=True)
    assert m == n and p.goal_reached() == op.goal_reached()
    assert np.array_equal(grid_types(p.export_graph_nodes()), op.type.reshape(H, W))


@pytest.mark.parametrize("seed", [3, 11])
def test_deferred_direct_connections_match_eager_oracle(gpu, dev_orc, seed):
    """Every cell whose goal direct connection the iterations evaluated (on
    demand, with the coarse first pass over every 16th sample before the walk
    in order) has the flag of the oracle's eager pass over the whole frame
    (processDirectGoalConnection at set_plan_data), and a connected cell its
    cost and heading."""
    cls, start, goal = synth.c0_request(seed)
    B = gpu.BatchPlanner(1, W, H)
    B.admit_many([gpu.make_request(cls, COSTS, start, goal, seed=seed, max_iterations=30)])
    B.run(60, 1)
    flag, cost, heading = B.direct_connections(0, W, H)
    op, _ = run_oracle(dev_orc, cls, start, goal, seed, 0)
    done = flag != 255
    assert done.sum() > 1000
    want = np.asarray(op.gd_flag).reshape(-1)[done].astype(np.int32)
    assert np.array_equal(flag[done].astype(np.int32), want)
    ok = done & (flag == 1)
    assert ok.sum() > 0
    assert np.max(np.abs(cost[ok] - np.asarray(op.gd_cost)[ok])) <= 1e-3
    # the cell's heading to the goal comes from atan2f: the device's and the
    # host library's differ in the last bit
    assert np.max(np.abs(heading[ok] - np.asarray(op.gd_heading)[ok])) <= 1e-5


@pytest.mark.parametrize("seed", [3, 5, 7])
def test_probe_counts_by_phase(gpu, dev_orc, seed):
    """Footprint probes of the reference algorithm, per phase, for one request.
    The expansion probes exactly what the oracle does.  The goal direct
    connections are evaluated only for cells that a goal-search window
    reaches, and each node's window is searched once per heading and cost, so
    those phases probe at most what the oracle's eager passes do."""
    cls, start, goal = synth.c0_request(seed)
    B = gpu.BatchPlanner(1, W, H)
    B.admit_many([gpu.make_request(cls, COSTS, start, goal, seed=seed, max_iterations=200)])
    B.run(400, 1)
    done, reached, loops = B.status()
    pr = B.probes()
    op, m = run_oracle(dev_orc, cls, start, goal, seed, int(loops[0]))
    want = op.probes_by_phase
    assert pr["k_expand"] == want["expand"]
    assert 0 < pr["k_gd_eval"] <= want["pre"]
    assert 0 < pr["k_goal"] <= want["goal"]


def test_interpolation_matches_oracle(gpu, orc):
    cls, start, goal = synth.c0_request(5)
    p, fr = gpu_planner(gpu, cls, 5)
    run_gpu(p, fr, start, goal)
    path = p.get_planned_path_array()
    dense = p.get_planned_path_array(interpolate=True)
    ref = orc.interpolate(path, W, H)
    assert dense.shape == ref.shape
    assert np.array_equal(dense[:, :2], ref[:, :2])
    assert np.allclose(dense[:, 2], ref[:, 2], atol=1e-5, rtol=0)
    wp = p.interpolate_planned_path_p(path)
    assert [(w.x, w.z) for w in wp] == [tuple(map(int, r[:2])) for r in ref]


def test_graph_dump_roundtrip(gpu, tmp_path):
    cls, start, goal = synth.c0_request(2)
    p, fr = gpu_planner(gpu, cls, 2)
    run_gpu(p, fr, start, goal)
    f = str(tmp_path / "graph.txt")
    p.save_current_graph_state(f)
    nodes, path = p.export_graph_nodes(), p.get_planned_path_array()
    q, fr2 = gpu_planner(gpu, cls, 99)
    q.set_plan_data(fr2, start, goal, 2.0)
    q.search_init()
    q.load_graph_state(f)
    assert np.array_equal(q.export_graph_nodes(), nodes)
    assert q.goal_reached()
    # the text dump keeps six decimals of each heading (graph.cu:496-520)
    qp = q.get_planned_path_array()
    assert np.array_equal(qp[:, :2], path[:, :2])
    assert np.allclose(qp[:, 2], path[:, 2], atol=1e-6, rtol=0)
    assert os.path.getsize(f) > 0


def test_no_path_and_empty_graph(gpu):
    cls, start, goal = synth.c0_request(0)
    p, fr = gpu_planner(gpu, cls, 0)
    assert p.get_planned_path() is None
    assert p.export_graph_nodes() is None
    p.set_plan_data(fr, start, goal, 2.0)
    p.search_init()
    assert not p.goal_reached()
    assert p.get_planned_path() is None


def oracle_alone(orc, req_args, seed, max_iter):
    cls, start, goal, steer = req_args
    Wq = cls.shape[1]
    op = orc.Planner(orc.Frame(cls, COSTS), Wq * synth.M_PER_PX, cls.shape[0] * synth.M_PER_PX,
                     steer, 5.4)
    op.set_plan_data(start, goal, 2.0, (22, 40), seed=seed)
    op.search_init()
    m = 0
    while not op.goal_reached() and m < max_iter:
        m += 1
        if not op.loop(False):
            break
    return op, m


def test_batch_equals_single_instance(gpu, dev_orc):
    """16 C0 requests in one batch: per request, the loop count and the path
    are the oracle's for the request alone."""
    n = 16
    B = gpu.BatchPlanner(n, W, H)
    args = [synth.c0_request(s) for s in range(n)]
    B.admit_many([gpu.make_request(c, COSTS, a, b, seed=s, max_iterations=200)
                  for s, (c, a, b) in enumerate(args)])
    B.run(400, 4)
    done, goal, loops = B.status()
    assert done.all() and goal.all()
    valid, length, pn = B.collect(np.arange(n))
    assert valid.all()
    for s, (c, a, b) in enumerate(args):
        op, m = oracle_alone(dev_orc, (c, a, b, 40.0), s, 200)
        assert loops[s] == m, s
        path = B.path(s)
        assert np.array_equal(path[:, :2], op.path()[:, :2]), s


def test_batch_mixed_sizes_same_alone_and_in_the_mix(gpu):
    """Uneven frames (128 / 256 / 512, 5-30% obstacles, varied poses and
    steering limits) planned together return what each returns alone."""
    n = 12
    reqs = []
    for s in range(n):
        cls, start, goal, steer, _ = synth.batch_request(1000 + s)
        reqs.append(gpu.make_request(cls, COSTS, start, goal, max_steering_deg=steer, seed=s,
                                     max_iterations=150))
    B = gpu.BatchPlanner(n, 512, 512)
    B.admit_many(reqs)
    B.run(300, 4)
    done, goal, loops = B.status()
    valid, length, pn = B.collect(np.arange(n))
    mixed = [(int(goal[k]), int(loops[k]), int(valid[k]), B.path(k)) for k in range(n)]
    A = gpu.BatchPlanner(1, 512, 512)
    for k in range(n):
        A.admit(0, reqs[k])
        A.run(300, 4)
        d1, g1, l1 = A.status()
        v1, _, _ = A.collect(np.array([0]))
        assert (int(g1[0]), int(l1[0]), int(v1[0])) == mixed[k][:3], k
        assert np.array_equal(A.path(0), mixed[k][3]), k
    assert goal.sum() >= 1
    assert np.all(valid[goal.astype(bool)] == 1)


def test_batch_plan_validates_every_path(gpu, orc):
    n = 32
    args = [synth.c0_request(s) for s in range(n)]
    reqs = [gpu.make_request(c, COSTS, a, b, seed=s, max_iterations=200)
            for s, (c, a, b) in enumerate(args)]
    B = gpu.BatchPlanner(n, W, H)
    valid, length, lat, dev_ms = B.plan(reqs, 400, 4)
    assert valid.sum() == n
    assert np.all(lat > 0) and dev_ms > 0 and np.all(lat <= dev_ms + 1e3)
    # the oracle's validator agrees on every returned path
    for k in range(n):
        cls, start, goal = args[k]
        op = orc.Planner(orc.Frame(cls, COSTS), 34.56, 34.56, 40.0, 5.4)
        op.set_plan_data(start, goal, 2.0, (22, 40), seed=k)
        assert op.validate_waypoints(B.path(k)), k


def test_served_same_alone_and_in_the_mix(gpu):
    """Continuous batching: requests of mixed sizes (60% 256², 30% 128², 10%
    512²) arrive as a Poisson stream, are admitted as slots free up and
    overlap on the device; each result (validity, loops, path length) is the
    one the request gives served alone.  A loop cap instead of a timeout
    keeps the comparison independent of timing."""
    rng = np.random.default_rng(7)
    n = 24
    reqs = []
    for s in range(n):
        size = int(rng.choice([256, 128, 512], p=[0.6, 0.3, 0.1]))
        cls, start, goal, steer, _ = synth.batch_request(2000 + s, sizes=(size,))
        reqs.append(gpu.make_request(cls, COSTS, start, goal, max_steering_deg=steer, seed=s,
                                     max_iterations=60))
    arrival = np.cumsum(rng.exponential(0.5, n))
    B = gpu.BatchPlanner(8, 512, 512)
    mix = B.serve(reqs, arrival_ms=arrival, timeout_ms=0, check_every=2)
    assert mix["wall_ms"] > 0 and mix["device_ms"] > 0
    assert np.all(mix["latency_ms"] >= mix["service_ms"] - 1e-3)
    # the path reaches the host after the device finished it (the device
    # clock's calibration to host time is good to a fraction of a ms)
    assert np.all(mix["result_ms"] >= mix["latency_ms"] - 0.5)
    A = gpu.BatchPlanner(1, 512, 512)
    for k in range(n):
        one = A.serve([reqs[k]], timeout_ms=0, check_every=2)
        got = (int(mix["valid"][k]), int(mix["loops"][k]), float(mix["length"][k]))
        assert got == (int(one["valid"][0]), int(one["loops"][0]), float(one["length"][0])), k
    assert mix["valid"].sum() >= 1


def test_served_timeout(gpu):
    """A request whose planning runs past its timeout finishes unsolved."""
    cls, start, goal = synth.c0_request(3)
    far = gpu.make_request(cls, COSTS, start, goal, seed=3, timeout_ms=1)
    B = gpu.BatchPlanner(2, W, H)
    out = B.serve([far], timeout_ms=1, check_every=1)
    # a 1 ms budget may or may not suffice for one loop; a finished request
    # either validated its path or stopped at the deadline
    assert out["loops"][0] >= 1
    ok = gpu.make_request(cls, COSTS, start, goal, seed=3)
    out = B.serve([ok], timeout_ms=100, check_every=1)
    assert out["valid"][0] == 1


def test_loaded_intrinsic_costs_match_oracle(gpu, dev_orc, tmp_path):
    """A graph dump with intrinsic costs loaded mid-plan (load_graph_state):
    the goal direct connections keep the costs of set_plan_data time, the
    expansion and goal search use the loaded ones, and the plan continues
    exactly like the oracle's from the same state."""
    orc = dev_orc
    seed = 5
    cls, start, goal = synth.c0_request(seed)
    p, fr = gpu_planner(gpu, cls, seed)
    p.set_plan_data(fr, start, goal, 2.0)
    p.search_init()
    for _ in range(3):
        p.loop(False)
    assert not p.goal_reached()
    f = str(tmp_path / "g.txt")
    p.save_current_graph_state(f)
    rows = np.loadtxt(f)
    rng = np.random.default_rng(3)
    band = np.zeros(W * H, bool)
    band[(W * 20):(W * 120)] = True  # rows 20..119
    rows[band, 6] = np.round(rng.uniform(0.0, 3.0, band.sum()), 3)
    f2 = str(tmp_path / "g2.txt")
    np.savetxt(f2, rows, fmt="%d %d %d %d %f %f %f %f")
    q, fr2 = gpu_planner(gpu, cls, seed)
    q.set_plan_data(fr2, start, goal, 2.0)
    q.search_init()
    q.load_graph_state(f2)
    op = orc.Planner(orc.Frame(cls, COSTS), 34.56, 34.56, 40.0, 5.4)
    op.set_plan_data(start, goal, 2.0, (22, 40), seed=seed)
    op.search_init()
    op.px[:] = rows[:, 0]
    op.pz[:] = rows[:, 1]
    op.type[:] = rows[:, 2]
    op.child[:] = rows[:, 3]
    op.heading[:] = rows[:, 4].astype(np.float32)
    op.cost[:] = rows[:, 5].astype(np.float32)
    op.intrinsic[:] = rows[:, 6].astype(np.float32)
    op.p.contents.last_expanded = int((rows[:, 2] == 2).sum())
    n = m = 0
    while not q.goal_reached() and n < 60:
        n += 1
        q.loop(False)
    while not op.goal_reached() and m < 60:
        m += 1
        op.loop(False)
    assert n == m
    assert np.array_equal(grid_types(q.export_graph_nodes()), op.type.reshape(H, W))
    if q.goal_reached():
        assert np.array_equal(q.get_planned_path_array()[:, :2], op.path()[:, :2])
