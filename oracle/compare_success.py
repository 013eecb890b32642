"""Whole-planner statistics against the reference's own planner (test
infrastructure; needs oracle/_ref and a GPU): success rate and coarse path
length of C0 plans over a range of seeds, for the reference's FastRRT
(src/fastrrt.cpp through its C ABI, its clock-seeded curand) and for this
library's batched planner, both capped at the same number of loop() calls.

    python -m oracle.compare_success [--seeds N] [--loops L] [--out file.json]
"""
import argparse
import json
import math
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def path_length(p):
    p = np.asarray(p, np.float64)
    if len(p) < 2:
        return 0.0
    return float(np.sqrt(((p[1:, :2] - p[:-1, :2]) ** 2).sum(1)).sum())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--seeds", type=int, default=1000)
    ap.add_argument("--loops", type=int, default=50)
    ap.add_argument("--seed0", type=int, default=0)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    import fastrrt_b200 as F
    from fastrrt_b200 import synth
    from oracle import oracle as O
    seeds = list(range(a.seed0, a.seed0 + a.seeds))
    # this library, batched
    B = F.BatchPlanner(256, 256, 256)
    mine_ok, mine_len = [], []
    t0 = time.time()
    for b0 in range(0, len(seeds), 256):
        chunk = seeds[b0:b0 + 256]
        reqs = [F.make_request(*[synth.c0_request(s)[0], synth.CLASS_COSTS, *synth.c0_request(s)[1:]],
                               seed=s, max_iterations=a.loops) for s in chunk]
        v, length, _, _ = B.plan(reqs, max_launches=a.loops + 8, check_every=4)
        for k in range(len(chunk)):
            mine_ok.append(int(v[k]))
            mine_len.append(path_length(B.path(k)) if v[k] else float("nan"))
    t_mine = time.time() - t0
    # the reference's planner
    ref_ok, ref_len = [], []
    t0 = time.time()
    for s in seeds:
        cls, st, gl = synth.c0_request(s)
        rp = O.RefPlanner(cls, synth.CLASS_COSTS, 34.56, 34.56, 40.0, 5.4)
        rp.set_plan_data(st, gl, 2.0, (22, 40))
        ok, _ = rp.plan(False, a.loops)
        ref_ok.append(int(ok))
        ref_len.append(path_length(rp.path()) if ok else float("nan"))
        del rp
    t_ref = time.time() - t0
    mo, ro = np.array(mine_ok), np.array(ref_ok)
    ml, rl = np.array(mine_len), np.array(ref_len)

    def ci(p, n):
        return 1.96 * math.sqrt(max(p * (1 - p), 1e-12) / n)

    both = (mo > 0) & (ro > 0)
    res = {"seeds": a.seeds, "loop_cap": a.loops,
           "success_mine": float(mo.mean()), "success_reference": float(ro.mean()),
           "success_ci95": [ci(mo.mean(), len(mo)), ci(ro.mean(), len(ro))],
           "mean_path_len_mine": float(np.nanmean(ml)), "mean_path_len_reference": float(np.nanmean(rl)),
           "mean_path_len_both_solved": [float(ml[both].mean()), float(rl[both].mean())],
           "seconds": {"mine": t_mine, "reference": t_ref}}
    print(json.dumps(res))
    if a.out:
        json.dump(res, open(a.out, "w"), indent=1)


if __name__ == "__main__":
    main()
