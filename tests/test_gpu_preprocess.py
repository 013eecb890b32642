"""SearchFrame preprocessing (the driveless SearchFrame's distance-to-goal
and safe-zone channels, whose producers are not in the reference tree: parity
of the producers is unpinned; their consumers are pinned).  The direct goal
connection with isSafeZoneChecked and isDistanceToGoalProcessed set is
bit-exact against the reference's own kernel given the same frame channels
(graph_direct_goal_connection.cu:16-167, 28-36, 124-135); the producers give
the distance the reference computes and safe-zone bits only where every
heading is feasible; planners use the channels as the reference does."""
import math

import numpy as np
import pytest

from fastrrt_b200 import synth

pytestmark = pytest.mark.gpu
COSTS = synth.CLASS_COSTS
W = H = 256
MS = math.radians(40.0)
LR = 5.4 / 2


def test_distance_producer_is_the_reference_distance(gpu):
    cls, _, _ = synth.c0_request(21)
    fr = gpu.SearchFrame(class_ids=cls, class_costs=COSTS)
    assert not fr.is_distance_to_goal_processed()
    fr.process_distance_to_goal(128, 0)
    assert fr.is_distance_to_goal_processed()
    d, _ = fr.channels()
    z, x = np.mgrid[0:H, 0:W]
    want = np.sqrt(((128 - x) ** 2 + (0 - z) ** 2).astype(np.float32))  # sqrtf of the int sum
    assert np.array_equal(d.view(np.uint32), want.view(np.uint32))


def test_safe_zone_bits_only_where_every_heading_is_feasible(gpu, ref):
    cls, _, _ = synth.c0_request(22)
    fr = gpu.SearchFrame(class_ids=cls, class_costs=COSTS)
    fr.process_safe_distance_zone((22, 40))
    assert fr.is_safe_zone_checked()
    _, trav = fr.channels()
    safe = (trav & 0x100) != 0
    # the definition: no obstacle within the Chebyshev radius that bounds
    # every probe of the 23 x 41 footprint
    rc = int(math.floor(math.sqrt(11 ** 2 + 20 ** 2))) + 2
    obst = COSTS[cls] < 0
    pad = np.pad(obst, rc)
    near = np.zeros_like(obst)
    for dz in range(-rc, rc + 1):
        for dx in range(-rc, rc + 1):
            near |= pad[rc + dz:rc + dz + H, rc + dx:rc + dx + W]
    assert np.array_equal(safe, ~near)
    assert 0.05 < safe.mean() < 0.95
    # soundness against the reference's footprint check at 16 headings
    zs, xs = np.nonzero(safe)
    pick = np.random.default_rng(1).choice(len(xs), 2000, replace=False)
    rc_ = ref.RefCase(ref.Frame(cls, COSTS), mdx=11, mdz=20)
    for a in np.linspace(-math.pi, math.pi, 16, endpoint=False):
        ang = np.full(len(pick), a, np.float32)
        assert rc_.feasible(xs[pick].astype(np.int32), zs[pick].astype(np.int32), ang, device=True).all()


@pytest.mark.parametrize("flags", [1, 2, 3])
def test_direct_connection_flags_bit_exact_vs_reference_kernel(gpu, ref, flags):
    cls, _, _ = synth.c0_request(23)
    rng = np.random.default_rng(flags)
    # safe-zone bits where the producer sets them; a distance channel that is
    # not the Euclidean one, so that reading it shows in the sample counts
    probe = gpu.SearchFrame(class_ids=cls, class_costs=COSTS)
    probe.process_safe_distance_zone((22, 40))
    _, trav = probe.channels()
    dist = rng.uniform(2.0, 90.0, (H, W)).astype(np.float32)
    xyz = np.zeros((H, W, 3), np.float32)
    xyz[..., 0] = cls
    xyz[..., 1] = dist
    xyz[..., 2] = trav
    fr = gpu.SearchFrame(class_costs=COSTS)
    fr.set_frame_data(xyz)
    ctx = gpu.Candidates(fr, min_dist=(22, 40), max_steering_rad=MS, lr_m=LR)
    x, z, lh, gx, gz, gh = synth.hermite_pairs(8192, W, H, 9, num_points=40)
    out, _ = ctx.hermite(x, z, lh, gx, gz, gh, 0.8, safe=flags)
    rcase = ref.RefCase(ref.Frame(cls, COSTS, trav=trav, dist=dist), mdx=11, mdz=20)
    r = rcase.direct(0.8, x, z, lh, gx, gz, gh, safe=flags, device=True)
    assert np.array_equal(out.view(np.uint32), r.view(np.uint32))
    # the flags change the answers on these inputs
    plain = rcase.direct(0.8, x, z, lh, gx, gz, gh, safe=0, device=True)
    assert not np.array_equal(plain.view(np.uint32), r.view(np.uint32))


def planner(F, fr, seed):
    return F.FastRRT(search_frame=fr, perception_width_m=34.56, perception_height_m=34.56,
                     max_steering_angle_deg=40, vehicle_length_m=5.4, timeout_ms=-1,
                     min_dist_x=22, min_dist_z=40, path_costs=COSTS, seed=seed)


def plan(p, fr, start, goal, loops=200):
    p.set_plan_data(fr, start, goal, 2.0)
    p.search_init()
    n = 0
    while not p.goal_reached() and n < loops:
        n += 1
        if not p.loop(False):
            break
    return n, p.get_planned_path_array() if p.goal_reached() else None


def test_planner_with_processed_distance_plans_the_same(gpu):
    # the produced distance is the one the planner computes: following the
    # frame's flags changes nothing
    for seed in (2, 6):
        cls, start, goal = synth.c0_request(seed)
        fr = gpu.SearchFrame(class_ids=cls, class_costs=COSTS)
        fr.process_distance_to_goal(goal[0], goal[1])
        a = planner(gpu, fr, seed)
        n1, p1 = plan(a, fr, start, goal)
        b = planner(gpu, fr, seed)
        b.set_frame_preprocessing(True)
        n2, p2 = plan(b, fr, start, goal)
        assert n1 == n2 and (p1 is None) == (p2 is None)
        if p1 is not None:
            assert np.array_equal(p1, p2)


def test_planner_with_safe_zone_bits_matches_oracle(gpu, orc):
    """The goal search always skips footprints from safe-zone cells
    (findBestGoalDirectConnection is called with safeZoneChecked = true,
    fastrrt.cpp:143); the planner on a frame with the bits plans as the
    oracle does on the same bits."""
    orc.set_fp_mode(orc.FP_DEVICE)
    try:
        for seed in (3, 8):
            cls, start, goal = synth.c0_request(seed)
            fr = gpu.SearchFrame(class_ids=cls, class_costs=COSTS)
            fr.process_safe_distance_zone((22, 40))
            _, trav = fr.channels()
            n, path = plan(planner(gpu, fr, seed), fr, start, goal)
            op = orc.Planner(orc.Frame(cls, COSTS, trav=trav), 34.56, 34.56, 40.0, 5.4)
            op.set_plan_data(start, goal, 2.0, (22, 40), seed=seed)
            ok, m = op.plan(False, n)
            assert m == n and ok == (path is not None)
            if path is not None:
                assert np.array_equal(path[:, :2], op.path()[:, :2])
    finally:
        orc.set_fp_mode(orc.FP_HOST)
