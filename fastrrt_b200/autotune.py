"""Autotuner of the served planner's shapes: measures validated plans/s of
served C0 planning (256x256, 100 ms timeout) for each combination of slots
per GPU, harvest interval (graph launches between checks) and launch shape
(blocks per SM of the sweep kernels and of the persistent expansion kernel),
and writes the best with every trial to a JSON file that bench.py reads.

    python -m fastrrt_b200.autotune [--requests N] [--out PATH]
"""
import argparse
import itertools
import json
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "tuned.json")
GRID = {"slots": (256, 512, 768), "check_every": (1, 2, 4), "sweep_blocks_per_sm": (4, 8, 16),
        "work_blocks_per_sm": (1, 2, 4)}


def load(path=DEFAULT_OUT):
    """the tuned shape, or None"""
    try:
        with open(path) as f:
            return json.load(f)["best"]
    except (OSError, ValueError, KeyError):
        return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=2048)
    ap.add_argument("--out", default=DEFAULT_OUT)
    a = ap.parse_args()
    import torch

    import fastrrt_b200 as F
    from fastrrt_b200 import synth
    frames, starts, goals, seeds = [], [], [], []
    for k in range(a.requests):
        cls, st, gl = synth.c0_request(3_000_000 + k)
        frames.append(cls)
        starts.append(st)
        goals.append(gl)
        seeds.append(3_000_000 + k)
    dev = torch.from_numpy(np.stack(frames)).cuda()
    reqs = [F.batch.device_request(F.make_request(frames[k], synth.CLASS_COSTS, starts[k], goals[k],
                                                  seed=seeds[k], timeout_ms=100),
                                   dev[k].data_ptr()) for k in range(a.requests)]
    trials = []
    for slots in GRID["slots"]:
        planner = F.BatchPlanner(slots, 256, 256)
        for sweep, work in itertools.product(GRID["sweep_blocks_per_sm"], GRID["work_blocks_per_sm"]):
            planner.set_launch(sweep, work)
            for ce in GRID["check_every"]:
                planner.serve(reqs[:slots], timeout_ms=100, check_every=ce)  # warm-up, graph capture
                out = planner.serve(reqs, timeout_ms=100, check_every=ce)
                v = out["valid"] > 0
                trials.append({"slots": slots, "check_every": ce, "sweep_blocks_per_sm": sweep,
                               "work_blocks_per_sm": work,
                               "plans_per_s": float(v.sum()) / (out["device_ms"] / 1e3),
                               "success_rate": float(v.mean()),
                               "service_p50_ms": float(np.percentile(out["service_ms"][v], 50))})
                print(json.dumps(trials[-1]), flush=True)
        del planner
    best = max(trials, key=lambda t: t["plans_per_s"])
    json.dump({"best": best, "trials": trials, "requests": a.requests,
               "when": time.strftime("%Y-%m-%d")}, open(a.out, "w"), indent=1)
    print("best", json.dumps(best))


if __name__ == "__main__":
    main()
