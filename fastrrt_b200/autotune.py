"""Autotuner of the served planner's operating point: measures validated
plans/s and the success rate of served C0 planning (256x256, 100 ms timeout
per request) for each combination of slots per GPU, harvest interval (graph
launches between checks) and expansion proposal (uniform draws, or the
learned network sampled with probability `mix`), and keeps the fastest
combination whose success rate is at least `--min-success` (97.9 %, the
planner's success rate over 1000 C0 seeds with a 50-loop cap, minus one
point; the reference's own planner solves 97.3 % of them); then the
harvest interval with the lowest p99 latency of Poisson arrivals at 1000
req/s through that operating point (the interval of the served benchmark's
Poisson legs); then the launch shape (blocks per SM of the sweep and
persistent kernels) of the batched workload (512 instances of mixed 128 /
256 / 512 frames).  The best and every trial go to a JSON file that
bench.py reads.

    python -m fastrrt_b200.autotune [--requests N] [--min-success S] [--out PATH]
"""
import argparse
import itertools
import json
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "tuned.json")
GRID = {"slots": (256, 384, 512, 640, 768, 1024), "check_every": (1, 2, 3, 4),
        "mix": (None, 0.8, 1.0)}
SERVING = {"rate": 1000.0, "requests": 2000, "check_every": (1, 2, 3, 4)}
LAUNCH = {"sweep_blocks_per_sm": 16, "work_blocks_per_sm": 2}
C2_GRID = {"sweep_blocks_per_sm": (4, 8, 16), "work_blocks_per_sm": (1, 2, 4)}
MIN_SUCCESS = 0.969


def load(path=DEFAULT_OUT):
    """the tuned operating point, or None"""
    try:
        with open(path) as f:
            return json.load(f)["best"]
    except (OSError, ValueError, KeyError):
        return None


def pick(trials, min_success):
    """the trial with the most validated plans/s among those whose success
    rate meets the bar (None when none does)"""
    ok = [t for t in trials if t["success_rate"] >= min_success]
    return max(ok, key=lambda t: t["plans_per_s"]) if ok else None


def serving_sweep(F, net, best, reqs):
    """the harvest interval for latency: Poisson arrivals at 1000 req/s
    through the chosen slots and proposal, p99 latency until the validated
    path is on the host for each interval"""
    serving_trials = []
    planner = F.BatchPlanner(best["slots"], 256, 256)
    planner.set_launch(LAUNCH["sweep_blocks_per_sm"], LAUNCH["work_blocks_per_sm"])
    planner.set_proposal(net if best["mix"] is not None else None, mix=best["mix"] or 0.0)
    rng = np.random.default_rng(99)
    arrival = np.cumsum(rng.exponential(1e3 / SERVING["rate"], SERVING["requests"]))
    sreqs = reqs[:SERVING["requests"]]
    for ce in SERVING["check_every"]:
        planner.serve(sreqs[:256], timeout_ms=100, check_every=ce)
        out = planner.serve(sreqs, arrival_ms=arrival, timeout_ms=100, check_every=ce)
        v = out["valid"] > 0
        serving_trials.append({"check_every": ce, "rate": SERVING["rate"],
                               "p50_ms": float(np.percentile(out["result_ms"][v], 50)),
                               "p99_ms": float(np.percentile(out["result_ms"][v], 99)),
                               "finish_p99_ms": float(np.percentile(out["latency_ms"][v], 99)),
                               "success_rate": float(v.mean())})
        print(json.dumps(serving_trials[-1]), flush=True)
    planner.set_proposal(None)
    del planner
    return serving_trials


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=8192)
    ap.add_argument("--min-success", type=float, default=MIN_SUCCESS)
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--serving-only", action="store_true",
                    help="keep the recorded operating point; measure only the latency harvest interval")
    a = ap.parse_args()
    import torch

    import fastrrt_b200 as F
    from fastrrt_b200 import proposal as P
    from fastrrt_b200 import synth
    from fastrrt_b200 import train_proposal as TP
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
    net = P.ProposalNet(seed=0, max_batch=512)
    have_net = TP.load(net)
    if a.serving_only:
        with open(a.out) as f:
            record = json.load(f)
        best = record["best"]
        record["serving_trials"] = serving_sweep(F, net, best, reqs)
        best["serving_check_every"] = min(record["serving_trials"], key=lambda t: t["p99_ms"])["check_every"]
        json.dump(record, open(a.out, "w"), indent=1)
        print("best", json.dumps(best))
        return
    trials = []
    for slots in GRID["slots"]:
        planner = F.BatchPlanner(slots, 256, 256)
        planner.set_launch(LAUNCH["sweep_blocks_per_sm"], LAUNCH["work_blocks_per_sm"])
        for mix, ce in itertools.product(GRID["mix"], GRID["check_every"]):
            if mix is not None and not have_net:
                continue
            planner.set_proposal(net if mix is not None else None, mix=mix or 0.0)
            planner.serve(reqs[:slots], timeout_ms=100, check_every=ce)  # warm-up, graph capture
            out = planner.serve(reqs, timeout_ms=100, check_every=ce)
            v = out["valid"] > 0
            trials.append({"slots": slots, "check_every": ce, "mix": mix, **LAUNCH,
                           "plans_per_s": float(v.sum()) / (out["device_ms"] / 1e3),
                           "success_rate": float(v.mean()),
                           "service_p50_ms": float(np.percentile(out["service_ms"][v], 50)),
                           "service_p99_ms": float(np.percentile(out["service_ms"][v], 99))})
            print(json.dumps(trials[-1]), flush=True)
        planner.set_proposal(None)
        del planner
    best = pick(trials, a.min_success)
    if best is None:  # nothing meets the bar: the most successful trial
        best = max(trials, key=lambda t: (t["success_rate"], t["plans_per_s"]))
    serving_trials = serving_sweep(F, net, best, reqs)
    best["serving_check_every"] = min(serving_trials, key=lambda t: t["p99_ms"])["check_every"]
    # the batched workload (512 instances of 128 / 256 / 512 frames in one
    # batch): the launch shape with the most validated plans/s
    c2_trials = []
    n = 512
    c2 = []
    keep = []
    for k in range(n):
        cls, st, gl, steer, _ = synth.batch_request(40_000_000 + k)
        d = torch.from_numpy(np.ascontiguousarray(cls)).cuda()
        keep.append(d)
        c2.append(F.batch.device_request(F.make_request(cls, synth.CLASS_COSTS, st, gl, max_steering_deg=steer,
                                                        seed=40_000_000 + k, timeout_ms=100), d.data_ptr()))
    planner = F.BatchPlanner(n, 512, 512)
    for sweep, work in itertools.product(C2_GRID["sweep_blocks_per_sm"], C2_GRID["work_blocks_per_sm"]):
        planner.set_launch(sweep, work)
        planner.plan(c2, 100000, 2)  # warm-up, graph capture
        v, _, _, ms = planner.plan(c2, 100000, 2)
        c2_trials.append({"sweep_blocks_per_sm": sweep, "work_blocks_per_sm": work,
                          "plans_per_s": float(v.sum()) / (ms / 1e3), "success_rate": float(v.mean())})
        print(json.dumps(c2_trials[-1]), flush=True)
    del planner
    c2_best = max(c2_trials, key=lambda t: t["plans_per_s"])
    best["c2_launch"] = {k: c2_best[k] for k in ("sweep_blocks_per_sm", "work_blocks_per_sm")}
    json.dump({"best": best, "min_success": a.min_success, "trials": trials, "serving_trials": serving_trials,
               "c2_trials": c2_trials,
               "requests": a.requests, "when": time.strftime("%Y-%m-%d")}, open(a.out, "w"), indent=1)
    print("best", json.dumps(best))


if __name__ == "__main__":
    main()
