"""Times the reference's own CPU planner on C0 frames: tests/cpu_tests/cpu_rrt.py
(RRT.loop_rrt(kinematic=True) with the MIN_DIST_CPU footprint check, on the
NodeGrid of node_grid.py).  TEST INFRASTRUCTURE and a reported baseline only:
it imports the reference tree, so it runs only on a machine that has that
tree, never where the bench runs; the record it writes is committed beside
it.

cpu_rrt.py imports model.waypoint.Waypoint, which is not in the reference
tree; a stand-in with the members the planner uses (x, z, heading and
distance_between) is installed under that name.  Every plan has the C0
parameters: seeded 256x256 frames (class id in channel 0 of an H x W x 3
image), start (128, 128, 0), goal (128, 0, 0), 40 deg, 5.4 m, min_dist
22 x 40 px, 2 m/s, max path 40 px, goal tolerance 20 px, and the timeout
(100 ms by default, the workload's); one process per host core.

    python -m oracle.cpu_rrt_baseline [--seeds N] [--timeout-ms T] [--workers W] [--out file]
"""
import argparse
import json
import math
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)


class Waypoint:
    """stand-in for the missing model.waypoint.Waypoint"""

    def __init__(self, x, z, heading=0.0):
        self.x, self.z, self.heading = int(x), int(z), float(heading)

    @staticmethod
    def distance_between(p1, p2):
        return math.hypot(p2.x - p1.x, p2.z - p1.z)


def _import_cpu_rrt():
    from oracle import build_oracle
    ref = build_oracle.reference_root()
    model = types.ModuleType("model")
    waypoint = types.ModuleType("model.waypoint")
    waypoint.Waypoint = Waypoint
    model.waypoint = waypoint
    sys.modules.setdefault("model", model)
    sys.modules.setdefault("model.waypoint", waypoint)
    for p in (os.path.join(ref, "tests", "cpu_tests"), ref):
        if p not in sys.path:
            sys.path.insert(0, p)
    import cpu_rrt
    return cpu_rrt


def plan_seeds(args):
    """plans of `seeds` (a worker process): (seed, solved, ms, loops)"""
    seeds, timeout_ms = args
    import random

    from fastrrt_b200 import synth
    cpu_rrt = _import_cpu_rrt()
    out = []
    for s in seeds:
        cls, st, gl = synth.c0_request(s)
        img = np.zeros((cls.shape[0], cls.shape[1], 3), np.float32)
        img[..., 0] = cls
        random.seed(s)
        r = cpu_rrt.RRT(256, 256, 256 * synth.M_PER_PX, 256 * synth.M_PER_PX, 40.0, 5.4, timeout_ms,
                        22, 40, -1, -1, -1, -1, 40.0, 20.0, [float(c) for c in synth.CLASS_COSTS])
        r.set_plan_data(img, Waypoint(*st), Waypoint(*gl), 2.0)
        t0 = time.perf_counter()
        r.search_init(cpu_rrt.MIN_DIST_CPU)
        loops = 0
        while not r.goal_reached():
            loops += 1
            if not r.loop_rrt(True):
                break
        out.append((s, int(r.goal_reached()), (time.perf_counter() - t0) * 1e3, loops))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--seeds", type=int, default=1000)
    ap.add_argument("--seed0", type=int, default=0)
    ap.add_argument("--timeout-ms", type=int, default=100)
    ap.add_argument("--workers", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--out", default=os.path.join(HERE, "cpu_rrt_baseline_c0.json"))
    a = ap.parse_args()
    import concurrent.futures as cf
    import multiprocessing as mp
    seeds = list(range(a.seed0, a.seed0 + a.seeds))
    parts = [seeds[k::a.workers] for k in range(a.workers)]
    t0 = time.time()
    with cf.ProcessPoolExecutor(a.workers, mp_context=mp.get_context("spawn")) as ex:
        res = [r for part in ex.map(plan_seeds, [(p, a.timeout_ms) for p in parts]) for r in part]
    wall = time.time() - t0
    ok = np.array([r[1] for r in res])
    ms = np.array([r[2] for r in res])
    rec = {"planner": "reference tests/cpu_tests/cpu_rrt.py RRT.loop_rrt(kinematic=True), MIN_DIST_CPU",
           "workload": "C0 seeds %d..%d, 256x256, timeout %d ms" % (seeds[0], seeds[-1], a.timeout_ms),
           "host_threads": a.workers, "host": os.uname().machine,
           "success_rate": float(ok.mean()), "plans_per_s": float(ok.sum()) / wall,
           "wall_s": wall, "plan_ms_p50": float(np.percentile(ms, 50)),
           "plan_ms_p99": float(np.percentile(ms, 99)),
           "solved_plan_ms_p50": float(np.percentile(ms[ok > 0], 50)) if ok.any() else None,
           "mean_loops": float(np.mean([r[3] for r in res]))}
    print(json.dumps(rec))
    json.dump(rec, open(a.out, "w"), indent=1)


if __name__ == "__main__":
    main()
