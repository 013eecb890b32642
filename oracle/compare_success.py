"""Whole-planner statistics against the reference's own planner (test
infrastructure; needs oracle/_ref and a GPU): success rate, path length and
path cost of C0 plans (or of the batched workload's generator, --workload c2) over a
range of seeds, for the reference's FastRRT
(src/fastrrt.cpp through its C ABI, its clock-seeded curand) and for this
library's drop-in FastRRT (the same seeds through the reference API), both
capped at the same number of loop() calls and without a timeout.

Path cost is the accumulated node cost the planner's own graph holds at the
last waypoint before the goal (the goal-connected cell): the parent's cost
plus (intrinsic + 1) per cell along the curves (kinematics.cu:184-221,
graph_direct_goal_connection.cu:16-167), with the base-cost addition of the
goal connection (fastrrt.cpp:145-167).  It is read from each planner's graph
dump (CudaGraph::dumpGraph, graph.cu:496-520: the same text format on both
sides).  The reference runs in several processes on the GPU at once.

    python -m oracle.compare_success [--seeds N] [--loops L] [--workers W] [--out file.json]
"""
import argparse
import json
import math
import os
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
W = H = 256


def path_length(p):
    p = np.asarray(p, np.float64)
    if len(p) < 2:
        return 0.0
    return float(np.sqrt(((p[1:, :2] - p[:-1, :2]) ** 2).sum(1)).sum())


def dump_cost(filename, x, z, width=W):
    """the cost column of cell (x, z) in a graph dump"""
    with open(filename) as f:
        for k, line in enumerate(f):
            if k == z * width + x:
                return float(line.split()[5])
    return float("nan")


def path_cost(planner_dump, path, width=W):
    """accumulated cost at the goal-connected cell (the waypoint before the goal)"""
    if len(path) < 2:
        return float("nan")
    with tempfile.TemporaryDirectory() as d:
        f = os.path.join(d, "graph.txt")
        planner_dump(f)
        return dump_cost(f, int(path[-2][0]), int(path[-2][1]), width)


def request(workload, s):
    """(class ids, start, goal, steering limit deg) of seed s"""
    from fastrrt_b200 import synth
    if workload == "c2":
        cls, st, gl, steer, _ = synth.batch_request(s)
        return cls, st, gl, steer
    cls, st, gl = synth.c0_request(s)
    return cls, st, gl, 40.0


def run_mine(seeds, loops, workload="c0"):
    import fastrrt_b200 as F
    from fastrrt_b200 import synth
    out = []
    for s in seeds:
        cls, st, gl, steer = request(workload, s)
        size_m = cls.shape[1] * synth.M_PER_PX
        fr = F.SearchFrame(class_ids=cls, class_costs=synth.CLASS_COSTS)
        p = F.FastRRT(search_frame=fr, perception_width_m=size_m, perception_height_m=size_m,
                      max_steering_angle_deg=steer, vehicle_length_m=5.4, timeout_ms=-1,
                      min_dist_x=22, min_dist_z=40, path_costs=synth.CLASS_COSTS, seed=s)
        p.set_plan_data(fr, st, gl, 2.0)
        p.search_init()
        n = 0
        while not p.goal_reached() and n < loops:
            n += 1
            if not p.loop(False):
                break
        ok = bool(p.goal_reached())
        path = p.get_planned_path_array() if ok else np.zeros((0, 3), np.float32)
        valid = ok and p.validate_path(path)
        out.append((int(ok and valid), path_length(path) if ok else float("nan"),
                    path_cost(p.save_current_graph_state, path, cls.shape[1]) if ok else float("nan")))
    return out


def run_reference(seeds, loops, workload="c0"):
    """the reference planner on `seeds` (a worker process)"""
    from fastrrt_b200 import synth
    from oracle import oracle as O
    out = []
    for s in seeds:
        cls, st, gl, steer = request(workload, s)
        size_m = cls.shape[1] * synth.M_PER_PX
        rp = O.RefPlanner(cls, synth.CLASS_COSTS, size_m, size_m, steer, 5.4)
        rp.set_plan_data(st, gl, 2.0, (22, 40))
        ok, _ = rp.plan(False, loops)
        path = rp.path() if ok else np.zeros((0, 3), np.float32)
        out.append((int(ok), path_length(path) if ok else float("nan"),
                    path_cost(rp.save_graph, path, cls.shape[1]) if ok else float("nan")))
        del rp
    return out


def _ref_worker(args):
    return run_reference(*args)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--seeds", type=int, default=1000)
    ap.add_argument("--loops", type=int, default=50)
    ap.add_argument("--seed0", type=int, default=0)
    ap.add_argument("--workers", type=int, default=4)
    ap.add_argument("--workload", default="c0", choices=("c0", "c2"),
                    help="c0: the single-instance 256x256 layout; c2: the batched workload's "
                         "generator (128/256/512 frames, 5-30 %% obstacles, steering 30-45 deg)")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    import concurrent.futures as cf
    import multiprocessing as mp
    seeds = list(range(a.seed0, a.seed0 + a.seeds))
    t0 = time.time()
    # the reference in spawned processes (started before this process uses the GPU)
    parts = [seeds[k::a.workers] for k in range(a.workers)]
    ex = cf.ProcessPoolExecutor(a.workers, mp_context=mp.get_context("spawn"))
    futs = [ex.submit(_ref_worker, (p, a.loops, a.workload)) for p in parts]
    mine = run_mine(seeds, a.loops, a.workload)
    t_mine = time.time() - t0
    ref_parts = [f.result() for f in futs]
    ex.shutdown()
    t_ref = time.time() - t0
    ref = [None] * len(seeds)
    for k, part in enumerate(ref_parts):
        for j, r in enumerate(part):
            ref[k + j * a.workers] = r
    mo, ml, mc = (np.array([m[i] for m in mine], np.float64) for i in range(3))
    ro, rl, rc = (np.array([r[i] for r in ref], np.float64) for i in range(3))

    def ci(p, n):
        return 1.96 * math.sqrt(max(p * (1 - p), 1e-12) / n)

    both = (mo > 0) & (ro > 0)
    res = {"seeds": [a.seed0, a.seed0 + a.seeds - 1], "loop_cap": a.loops, "timeout": "none",
           "workload": ("C0: seeded 256x256 frames, start (128,128,0), goal (128,0,0), 40 deg, 5.4 m, "
                        "min_dist 22x40 px, 2 m/s" if a.workload == "c0" else
                        "C2 generator: 128/256/512 frames, 5-30% obstacles, start near the bottom centre, "
                        "goal on the top band, steering U(30,45) deg, 5.4 m, min_dist 22x40 px, 2 m/s"),
           "success_mine": float(mo.mean()), "success_reference": float(ro.mean()),
           "success_ci95": [ci(mo.mean(), len(mo)), ci(ro.mean(), len(ro))],
           "success_diff_points": 100 * float(mo.mean() - ro.mean()),
           "mean_path_len_mine": float(np.nanmean(ml)), "mean_path_len_reference": float(np.nanmean(rl)),
           "mean_path_cost_mine": float(np.nanmean(mc)), "mean_path_cost_reference": float(np.nanmean(rc)),
           "path_cost_rel_diff": float(np.nanmean(mc) / np.nanmean(rc) - 1),
           "path_len_rel_diff": float(np.nanmean(ml) / np.nanmean(rl) - 1),
           "both_solved": int(both.sum()),
           "mean_path_len_both_solved": [float(ml[both].mean()), float(rl[both].mean())],
           "mean_path_cost_both_solved": [float(mc[both].mean()), float(rc[both].mean())],
           "mine_validated_by": "the device path validator (fastrrt_validate_path)",
           "seconds": {"mine": t_mine, "reference_wall": t_ref, "reference_workers": a.workers}}
    print(json.dumps(res))
    if a.out:
        json.dump(res, open(a.out, "w"), indent=1)


if __name__ == "__main__":
    main()
