"""Benchmark of the B200 FastRRT planner: validated plans/s and plan latency
of served, continuously batched planning on 256x256 frames, beside the plain
single-instance GPU loop.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--requests R] [--slots S]
                    [--impl mine|reference]

Requests are the C0 workload: seeded 256x256 frames (road corridor, 12
rectangles and 6 disks of obstacles, low/high-cost classes elsewhere), start
(128,128,0), goal (128,0,0), 40 deg steering, 5.4 m vehicle, 22x40 px
footprint, 2 m/s, 100 ms timeout per request.  A step serves R fresh
requests through S slots with continuous batching: a request is admitted
when a slot frees up (frame masks, deferred goal connections, start node),
planned in the same graph launches as the others until it reaches its goal
or its timeout, then extracted and validated on the device.  Only validated
plans count.  The headline operating point is the autotuner's
(fastrrt_b200/tuned.json): the fastest slot count, harvest interval and
expansion proposal (the learned network or uniform draws) whose success
rate is at least 96.9 %.

  value   : validated plans/s with the frames already in HBM (device clock,
            CUDA events around each step, max over ranks)
  e2e     : the same through the C ABI with host frames (host -> device
            copies of the frames and device -> host copies of the results
            inside the timed region)
  serving : Poisson arrivals at the C3 rates; p50/p95/p99 latency from
            arrival until the validated path is on the host (and from
            arrival to the device-clock finish)
  serving_mixed_sizes / batched_mixed_sizes : the C3 and C2 workloads
            (60/30/10 % 256/128/512 frames under a 40 GB budget; 512
            instances of 128/256/512 frames per batch)
  roofline: the dominant kernel's footprint-probe rate against one probe per
            lane per cycle
  cpu_baseline / --impl reference : the CPU restatement of the same planner
            (oracle/, all host cores) on a bounded sample of the workload

Each step plans frames never planned before; the per-step working set (S
slots x ~8 MB of node grid and scratch) exceeds L2.  With --gpus N > 1 and
no torchrun environment the script starts N ranks itself (one process per
GPU); every rank serves its own requests (weak scaling, no collective on the
data path) and the time is the maximum over ranks.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

M_PER_PX = 0.135
SIZE = 256
TIMEOUT_MS = 100
METRIC = "validated plans/s, served + batched 256x256 planning"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--requests", type=int, default=8192, help="requests per step and GPU")
    ap.add_argument("--slots", type=int, default=None,
                    help="planning slots per GPU (default: the autotuned value, else 512)")
    ap.add_argument("--check-every", type=int, default=None,
                    help="graph launches between harvests (default: autotuned, else 2)")
    ap.add_argument("--rates", default="200,1000,5000", help="Poisson arrival rates (req/s)")
    ap.add_argument("--rate-requests", type=int, default=2000)
    ap.add_argument("--mix", type=float, default=None,
                    help="learned-proposal sampling probability (default: the autotuned one; "
                         "< 0: uniform draws only)")
    ap.add_argument("--candidates", type=int, default=1 << 20, help="per-candidate microbench size")
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the mixed-size legs (C2 batched, C3 served) for short runs")
    ap.add_argument("--plain", type=int, default=256, help="plans of the plain single-instance loop")
    ap.add_argument("--ref-plans", type=int, default=None,
                    help="plans per step of the reference arm (default: one per host core)")
    return ap.parse_args()


def spawn_ranks(n, argv):
    """starts this script as n ranks on this node (torch.distributed.run,
    rendezvous on 127.0.0.1) and returns their exit status"""
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + argv
    return subprocess.call(cmd)


def dist_setup(gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        # NCCL over the GPUs; gloo where there is no GPU (the CPU tests)
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def reduce_over_ranks(v, world, op="max"):
    """max or sum of a per-rank scalar (NCCL on the GPUs, gloo on the CPU)"""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(v, world):
    return reduce_over_ranks(v, world, "max")


def sum_over_ranks(v, world):
    return reduce_over_ranks(v, world, "sum")


def request_seeds(rank, step, B):
    """seeds of the B requests of one step on one rank; ranks never share one"""
    return [(rank * 1000003 + step * B + k) & 0xFFFFFFFF for k in range(B)]


def _c0_frames(seeds):
    """C0 requests of `seeds` (a pool worker): (frames, starts, goals)"""
    from fastrrt_b200 import synth
    out = [synth.c0_request(seed, SIZE) for seed in seeds]
    return np.stack([o[0] for o in out]), [o[1] for o in out], [o[2] for o in out]


def workload(rank, step, B):
    """seeded requests of one step: (frames, starts, goals, seeds)"""
    seeds = request_seeds(rank, step, B)
    frames, starts, goals = _c0_frames(seeds)
    return frames, starts, goals, seeds


def workloads(rank, steps, B, world=1):
    """the requests of `steps` steps, generated by a process pool (spawned,
    so it is independent of this process's CUDA state)"""
    import concurrent.futures as cf
    import multiprocessing as mp
    seeds = [request_seeds(rank, s, B) for s in range(steps)]
    flat = [x for ss in seeds for x in ss]
    chunk = 256
    parts = [flat[i:i + chunk] for i in range(0, len(flat), chunk)]
    workers = max(1, min(32, (os.cpu_count() or 1) // max(1, world), len(parts)))
    if workers == 1:
        res = [_c0_frames(p) for p in parts]
    else:
        with cf.ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
            res = list(ex.map(_c0_frames, parts))
    frames = np.concatenate([r[0] for r in res])
    starts = [x for r in res for x in r[1]]
    goals = [x for r in res for x in r[2]]
    return [(frames[s * B:(s + 1) * B], starts[s * B:(s + 1) * B], goals[s * B:(s + 1) * B], seeds[s])
            for s in range(steps)]


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def start(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

        def run():
            while not self._stop.is_set():
                try:
                    out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits"], capture_output=True,
                                         text=True, timeout=5).stdout.strip()
                    if out:
                        self.rows.append([c.strip() for c in out.split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)

        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 3 + i and r[3 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def cpu_baseline(B_sample=None, threads=None, timeout_ms=30000):
    """the CPU restatement of the planner (oracle/, OpenMP over plans, one
    plan per thread) on a bounded sample of the workload.  The restatement
    follows the reference's eager goal precompute (every cell of the frame,
    seconds per frame on one core), so at the workload's 100 ms timeout no
    CPU plan would finish; the sample runs with a 30 s cap instead."""
    from fastrrt_b200 import synth
    from oracle import oracle as O
    cores = threads or os.cpu_count() or 1
    n = B_sample or max(8, min(64, 2 * cores))
    frames, sg, seeds = [], [], []
    for k in range(n):
        seed = 7_000_000 + k
        cls, st, gl = synth.c0_request(seed, SIZE)
        frames.append(cls)
        sg.append([st[0], st[1], int(st[2] * 1e6), gl[0], gl[1], int(gl[2] * 1e6)])
        seeds.append(seed)
    t0 = time.time()
    ok, iters, cost, ms = O.plan_batch(
        np.stack(frames), synth.CLASS_COSTS, np.array(sg, np.int32), np.array(seeds, np.uint64),
        pw_m=SIZE * M_PER_PX, ph_m=SIZE * M_PER_PX, max_steer_deg=40.0, vehicle_len=5.4,
        min_dist=(22, 40), velocity=2.0, max_path=40.0, dist_tol=20.0,
        heading_tol=float(np.float32(math.radians(10))), timeout_ms=timeout_ms, max_iter=0,
        smart=False, threads=cores)
    wall = time.time() - t0
    return {"value": float(ok.sum()) / wall, "unit": "plans/s", "cores": cores, "kind": "port",
            "sample": f"{n} seeded 256x256 C0 plans (same generator and parameters; "
                      f"{timeout_ms / 1e3:.0f} s cap per plan instead of 100 ms), "
                      f"{int(ok.sum())} validated, {wall:.1f} s wall on {cores} threads",
            "success_rate": float(ok.mean()), "median_plan_s": float(np.median(ms) / 1e3)}


def run_reference(args, rank, world):
    """--impl reference: the CPU planner (oracle port) on the host cores"""
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    per_step = args.ref_plans or cores
    for _ in range(args.warmup):
        cpu_baseline(per_step, cores)
    vals, walls = [], []
    for _ in range(args.steps):
        t0 = time.time()
        r = cpu_baseline(per_step, cores)
        walls.append(time.time() - t0)
        vals.append(r["value"])
    value = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "plans/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * float(np.mean(walls)), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"C0 plans of seeded {SIZE}x{SIZE} frames, {per_step} per step",
                       "parallelism": f"{cores} host threads"},
            "cpu_baseline": {"value": value, "unit": "plans/s", "cores": cores, "kind": "port",
                             "sample": f"{per_step} plans per step, 30 s cap per plan"},
            "e2e": {"value": value, "unit": "plans/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def plain_loop(n, rank):
    """the drop-in single-instance API (FastRRT + loop) on n fresh frames,
    100 ms timeout per plan as in the workload"""
    import fastrrt_b200 as F
    from fastrrt_b200 import synth
    ok = 0
    lat = []
    frames = [synth.c0_request(9_000_000 + rank * 1000 + k, SIZE) for k in range(n)]
    p = F.FastRRT(F.EgoParams.init(SIZE, SIZE).with_search_physical_size(SIZE * M_PER_PX, SIZE * M_PER_PX)
                  .with_max_steering_angle(F.angle.new_deg(40.0)).with_vehicle_length(5.4)
                  .with_segmentation_class_costs(synth.CLASS_COSTS).build(),
                  min_dist_x=22, min_dist_z=40, timeout_ms=TIMEOUT_MS)
    # one untimed plan first (library load, first launches)
    fr = F.SearchFrame(class_ids=frames[0][0], class_costs=synth.CLASS_COSTS)
    p.set_plan_data(fr, frames[0][1], frames[0][2], 2.0)
    p.search_init()
    p.loop(False)
    t0 = time.time()
    for k, (cls, st, gl) in enumerate(frames):
        t1 = time.time()
        fr = F.SearchFrame(class_ids=cls, class_costs=synth.CLASS_COSTS)
        p.set_seed(k)
        p.set_plan_data(fr, st, gl, 2.0)
        p.search_init()
        while not p.goal_reached():
            if not p.loop(False):
                break
        path = p.get_planned_path_array()
        lat.append((time.time() - t1) * 1e3)
        ok += int(p.goal_reached() and len(path) >= 2)
    wall = time.time() - t0
    return {"plans_per_s": ok / wall, "plans": n, "ok": ok,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "note": "one FastRRT object, set_plan_data + search_init + loop() until the goal or "
                    "the 100 ms timeout, per plan through the reference API, host wall clock"}


def candidate_microbench(n, cpu=True):
    """Per-candidate kernels on 256x256 C0-generator frames at 5/15/30%
    obstacles: n kinematic candidates (parent uniform, heading U(-pi, pi),
    steering U(-40, 40) deg, length U(5, 40) px) and 65,536 Hermite pairs of
    64 samples, through the device entry points (device clock, synchronised);
    the CPU restatement on a bounded sample beside them."""
    import torch

    import fastrrt_b200 as F
    from fastrrt_b200 import synth
    from oracle import oracle as O
    res = {}
    ms = math.radians(40.0)
    for cov in (0.05, 0.15, 0.30):
        cls = synth.make_frame(11, SIZE, coverage=cov)
        heading, sx, sz, steer, seg = synth.candidates(n, SIZE, SIZE, 1)
        fr = F.SearchFrame(class_ids=cls, class_costs=synth.CLASS_COSTS)
        ctx = F.Candidates(fr, min_dist=(22, 40), max_steering_rad=ms, lr_m=2.7, heading_grid=heading)
        d = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (sx, sz, steer, seg)]
        out = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
        pr = torch.zeros(1, dtype=torch.int64, device="cuda")
        ctx.kinematic_device(*d, 2.0, out, pr)
        torch.cuda.synchronize()
        reps = 3
        pr.zero_()
        t0 = time.perf_counter()
        for _ in range(reps):
            ctx.kinematic_device(*d, 2.0, out, pr)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / reps
        entry = {"candidates_per_s": n / dt, "reference_probes_per_s": float(pr.item()) / reps / dt,
                 "feasible_fraction": float((out[:, 0] >= 0).float().mean().item())}
        if cpu:
            m = min(n, 20000)
            g = O.Graph(SIZE, SIZE, SIZE * M_PER_PX, SIZE * M_PER_PX, 40.0, 5.4, -1.0, (22, 40))
            g.g.pp.lr, g.g.pp.max_steer_rad = 2.7, ms
            g.heading[:] = heading
            t0 = time.perf_counter()
            g.kinematic_batch(O.Frame(cls, synth.CLASS_COSTS), sx[:m], sz[:m], steer[:m], seg[:m], 2.0)
            entry["cpu_candidates_per_s"] = m / (time.perf_counter() - t0)
            entry["cpu_cores"] = os.cpu_count()
        res[f"kinematic_{int(cov * 100)}pct"] = entry
    cls = synth.make_frame(11, SIZE, coverage=0.15)
    x, z, lh, gx, gz, gh = synth.hermite_pairs(65536, SIZE, SIZE, 5, num_points=64)
    fr = F.SearchFrame(class_ids=cls, class_costs=synth.CLASS_COSTS)
    ctx = F.Candidates(fr, min_dist=(22, 40), max_steering_rad=ms, lr_m=2.7)
    d = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (x, z, lh, gx, gz, gh)]
    out = torch.zeros(65536, dtype=torch.float32, device="cuda")
    pr = torch.zeros(1, dtype=torch.int64, device="cuda")
    ctx.hermite_device(*d, 0.8, out, pr)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(3):
        ctx.hermite_device(*d, 0.8, out, pr)
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / 3
    res["hermite_64_samples"] = {"pairs_per_s": 65536 / dt,
                                 "connected_fraction": float((out >= 0).float().mean().item())}
    return res


def pct(a, q):
    return float(np.percentile(a, q)) if len(a) else None


def _mixed_frames(args):
    """requests of the batched workload (a pool worker): seeds and sizes ->
    (class ids, start, goal, steering limit) per request"""
    from fastrrt_b200 import synth
    out = []
    for seed, sizes in args:
        cls, st, gl, steer, _ = synth.batch_request(seed, sizes=sizes)
        out.append((cls, st, gl, steer))
    return out


def mixed_requests(specs, world=1):
    """batched-workload requests for (seed, sizes) specs, generated by a
    spawned process pool"""
    import concurrent.futures as cf
    import multiprocessing as mp
    parts = [specs[i:i + 64] for i in range(0, len(specs), 64)]
    workers = max(1, min(32, (os.cpu_count() or 1) // max(1, world), len(parts)))
    if workers == 1:
        res = [_mixed_frames(p) for p in parts]
    else:
        with cf.ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
            res = list(ex.map(_mixed_frames, parts))
    return [r for part in res for r in part]


# frame sizes of the served mixed workload and their shares
C3_SIZES = ((256, 0.6), (128, 0.3), (512, 0.1))
C3_BUDGET = 40 << 30  # node-grid budget of the served mixed workload (bytes)


def c2_batched(args, rank, world, tuned):
    """Batched planning of 512 instances in one go (frame sizes 128, 256 and
    512 drawn uniformly, obstacle coverage U(5, 30) %, start near the bottom
    centre, goal on the top band, steering limit U(30, 45) deg), 100 ms
    timeout per instance: validated plans/s of whole batches (device clock),
    success rate, per-kernel shares of one batch (kernel-timing replay)."""
    import torch

    import fastrrt_b200 as F
    from fastrrt_b200 import synth
    n = 512
    steps = max(1, min(args.steps, 3))
    specs = [(20_000_000 + rank * 1_000_003 + s * n + k, (128, 256, 512)) for s in range(steps + 1)
             for k in range(n)]
    data = mixed_requests(specs, world)
    launch = (tuned or {}).get("c2_launch") or {"sweep_blocks_per_sm": 16, "work_blocks_per_sm": 2}
    planner = F.BatchPlanner(n, 512, 512)
    planner.set_launch(launch["sweep_blocks_per_sm"], launch["work_blocks_per_sm"])
    keep = []

    def batch(s):
        reqs = []
        for k in range(n):
            cls, st, gl, steer = data[s * n + k]
            d = torch.from_numpy(np.ascontiguousarray(cls)).cuda()
            keep.append(d)
            reqs.append(F.batch.device_request(
                F.make_request(cls, synth.CLASS_COSTS, st, gl, max_steering_deg=steer,
                               seed=specs[s * n + k][0], m_per_px=M_PER_PX, timeout_ms=TIMEOUT_MS),
                d.data_ptr()))
        return reqs

    batches = [batch(s) for s in range(steps + 1)]
    torch.cuda.synchronize()
    planner.plan(batches[0], 100000, 2)  # warm-up, graph capture
    valid, dev_ms = 0, 0.0
    for s in range(1, steps + 1):
        v, _, _, ms = planner.plan(batches[s], 100000, 2)
        valid += int(v.sum())
        dev_ms += ms
    planner.profile(True)
    planner.plan(batches[1], 100000, 2)
    kt = planner.kernel_times()
    planner.profile(False)
    tot = sum(t[0] for t in kt.values()) or 1.0
    t_max = max_over_ranks(dev_ms, world)
    return {"workload": f"{n} instances per batch, frames 128/256/512 uniformly, obstacle coverage "
                        f"U(5,30)%, steering U(30,45) deg, {TIMEOUT_MS} ms timeout per instance, "
                        f"one CUDA graph launch per iteration over all instances",
            "batches": steps, "value": sum_over_ranks(valid, world) / (t_max / 1e3), "unit": "plans/s",
            "success_rate": valid / float(n * steps), "ms_per_batch": t_max / steps,
            "launch_shape": launch,
            "kernel_share": {k: round(t[0] / tot, 4) for k, t in
                             sorted(kt.items(), key=lambda kv: -kv[1][0]) if t[0] > 0}}


def c3_serving(args, rank, world, tuned, attach_net):
    """Served planning of the mixed workload: Poisson arrivals at the C3
    rates, frames 60 % 256x256, 30 % 128x128, 10 % 512x512 (the batched
    workload's generator), admission by device memory against a 40 GB
    node-grid budget (each request takes storage sized by its frame), 100
    ms timeout per request, latency from arrival to finish."""
    import torch

    import fastrrt_b200 as F
    from fastrrt_b200 import synth
    n = args.rate_requests
    rng = np.random.default_rng(4321 + rank)
    sizes = rng.choice([c[0] for c in C3_SIZES], size=n, p=[c[1] for c in C3_SIZES])
    specs = [(30_000_000 + rank * 1_000_003 + k, (int(sizes[k]),)) for k in range(n)]
    data = mixed_requests(specs, world)
    slots = args.slots
    planner = F.BatchPlanner(slots, 512, 512, budget_bytes=C3_BUDGET)
    launch = (tuned or {})
    if launch:
        planner.set_launch(launch["sweep_blocks_per_sm"], launch["work_blocks_per_sm"])
    attach_net(planner)
    keep, reqs = [], []
    for k in range(n):
        cls, st, gl, steer = data[k]
        d = torch.from_numpy(np.ascontiguousarray(cls)).cuda()
        keep.append(d)
        reqs.append(F.batch.device_request(
            F.make_request(cls, synth.CLASS_COSTS, st, gl, max_steering_deg=steer, seed=specs[k][0],
                           m_per_px=M_PER_PX, timeout_ms=TIMEOUT_MS), d.data_ptr()))
    torch.cuda.synchronize()
    planner.serve(reqs[:min(n, 64)], timeout_ms=TIMEOUT_MS, check_every=args.check_every)
    res = {"workload": "Poisson arrivals, frames 60% 256x256 / 30% 128x128 / 10% 512x512, "
                       f"{TIMEOUT_MS} ms timeout, admission by device memory against a "
                       f"{C3_BUDGET >> 30} GB node-grid budget, at most {slots} requests at once",
           "requests_per_rate": n, "size_counts": {str(c[0]): int((sizes == c[0]).sum()) for c in C3_SIZES},
           "slot_bytes": {str(c[0]): F.batch.slot_bytes(c[0], c[0]) for c in C3_SIZES}}
    rates = [float(x) for x in args.rates.split(",") if x]
    arrivals = {rate: np.cumsum(rng.exponential(1e3 / rate, n)) for rate in rates}

    def rates_block():
        out_rates = {}
        for rate in rates:
            out = planner.serve(reqs, arrival_ms=arrivals[rate], timeout_ms=TIMEOUT_MS,
                                check_every=args.serving_check_every)
            v = out["valid"] > 0
            lat = out["result_ms"][v]     # arrival -> validated path on the host
            out_rates[f"{rate:g}_req_s"] = {
                "offered": rate, "achieved_plans_per_s": float(v.sum()) / (out["wall_ms"] / 1e3),
                "success_rate": float(v.mean()), "p50_ms": pct(lat, 50), "p95_ms": pct(lat, 95),
                "p99_ms": pct(lat, 99), "mean_loops": float(out["loops"].mean()),
                "success_by_size": {str(c[0]): float(v[sizes == c[0]].mean()) for c in C3_SIZES
                                    if (sizes == c[0]).any()}}
        return out_rates

    # the headline's proposal, then uniform draws on the same arrivals
    res.update(rates_block())
    res["proposal"] = "learned" if planner.proposal_attached() else "uniform"
    if planner.proposal_attached():
        planner.set_proposal(None)
        planner.serve(reqs[:min(n, 64)], timeout_ms=TIMEOUT_MS, check_every=args.check_every)
        res["uniform"] = rates_block()
    budget, used, peak = planner.memory()
    res["memory"] = {"budget_bytes": budget, "peak_bytes_held": peak, "bytes_held_after": used}
    planner.set_proposal(None)
    return res


def issue_peak(peaks):
    """lane-issue peak of the footprint-probe roofline: SMs x 32 lanes x the
    measured maximum SM clock (probe lanes per second)"""
    import torch
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    mhz = float(peaks.get("sm_max_mhz", 1965.0))
    return sms * 32 * mhz * 1e6, sms, mhz


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one captured
# launch of the dominant search kernel (profiles/k_gd_eval_served_first_iterations.txt:
# a launch of the first iterations of 256 fresh 256x256 requests, 17.16 MB
# read + 0.06 MB written).  The masks and summed-area tables it probes stay
# in L2, so its DRAM bytes follow the frames it touches, not its probes: the
# figure is reported as captured, not scaled by probe count.
NCU_DRAM_BYTES_PER_LAUNCH = {
    "k_gd_eval": {"bytes": 17.22e6, "captured": "one launch of the first iterations of "
                  "256 fresh 256x256 C0 requests, 256 slots (ncu --set full)"},
}


def run_mine(args, rank, world, local):
    import torch

    import fastrrt_b200 as F
    from fastrrt_b200 import autotune, synth
    from fastrrt_b200 import proposal as P
    from fastrrt_b200 import train_proposal as TP
    F._lib.require_cuda()
    torch.cuda.set_device(local)
    tuned = autotune.load()
    if tuned and args.slots is None:
        args.slots = tuned["slots"]
    if tuned and args.check_every is None:
        args.check_every = tuned["check_every"]
    # the Poisson (latency) legs harvest at the interval tuned for latency
    args.serving_check_every = (tuned or {}).get("serving_check_every") or args.check_every
    if args.mix is None:
        args.mix = tuned.get("mix") if tuned else 0.8
        if args.mix is None:
            args.mix = -1.0
    args.slots = args.slots or 512
    args.check_every = args.check_every or 1
    R = args.requests
    total_steps = args.warmup + args.steps
    t_gen = time.time()
    work = workloads(rank, total_steps, R, world)
    gen_s = time.time() - t_gen
    planner = F.BatchPlanner(args.slots, SIZE, SIZE)
    if tuned:
        planner.set_launch(tuned["sweep_blocks_per_sm"], tuned["work_blocks_per_sm"])
    costs = synth.CLASS_COSTS
    net = P.ProposalNet(seed=0, max_batch=512)
    have_net = TP.load(net)
    learned = args.mix >= 0 and have_net

    def attach(use_net):
        planner.set_proposal(net if use_net else None, mix=args.mix if use_net else 0.0)

    def requests(frames, starts, goals, seeds, device_frames=None):
        reqs = []
        for k in range(len(seeds)):
            r = F.make_request(frames[k], costs, starts[k], goals[k], seed=seeds[k],
                               m_per_px=M_PER_PX, timeout_ms=TIMEOUT_MS)
            if device_frames is not None:
                r = F.batch.device_request(r, device_frames[k].data_ptr())
            reqs.append(r)
        return reqs

    def serve(reqs, arrival=None):
        ce = args.serving_check_every if arrival is not None else args.check_every
        return planner.serve(reqs, arrival_ms=arrival, timeout_ms=TIMEOUT_MS, check_every=ce)

    def timed_steps(reqs_of_step, clocks=None):
        """the timed steps: (device ms summed, validated plans, service ms, loops, lengths)"""
        barrier(world)
        torch.cuda.synchronize()
        if clocks:
            clocks.start()
        dev_ms, valid, service, loops, lengths = 0.0, 0, [], [], []
        for s in range(args.warmup, total_steps):
            out = serve(reqs_of_step(s))
            dev_ms += out["device_ms"]
            v = out["valid"] > 0
            valid += int(v.sum())
            service.extend(out["service_ms"][v].tolist())
            lengths.extend(out["length"][v].tolist())
            loops.extend(out["loops"].tolist())
        torch.cuda.synchronize()
        barrier(world)
        return dev_ms, valid, service, loops, lengths

    # frames resident in HBM for `value`
    dev = [torch.from_numpy(work[s][0]).cuda() for s in range(total_steps)]
    reqs_dev = [requests(*work[s], device_frames=dev[s]) for s in range(total_steps)]
    torch.cuda.synchronize()
    attach(learned)
    for s in range(args.warmup):
        serve(reqs_dev[s])
    sampler = ClockSampler(local)
    dev_ms, valid_total, service, loops, lengths = timed_steps(lambda s: reqs_dev[s], sampler)
    clocks = sampler.stop()
    t_max = max_over_ranks(dev_ms, world)
    plans = sum_over_ranks(valid_total, world)
    value = plans / (t_max / 1e3)

    # e2e: host frames through the C ABI (H2D of frames, D2H of results inside)
    e2e_ms, e2e_valid, _, _, _ = timed_steps(lambda s: requests(*work[s]))
    e2e_t = max_over_ranks(e2e_ms, world)
    e2e_plans = sum_over_ranks(e2e_valid, world)
    h2d = R * (SIZE * SIZE + 4 * len(costs))
    d2h = R * (4 * 5 + 3 * 4 * 1024)

    # served at the C3 Poisson rates (latency from arrival to finish)
    n_rate = args.rate_requests
    rate_work = workload(rank, 10_000, n_rate)
    rate_dev = torch.from_numpy(rate_work[0]).cuda()
    rate_reqs = requests(*rate_work, device_frames=rate_dev)

    def poisson():
        res = {}
        rng = np.random.default_rng(1234 + rank)
        for rate in [float(x) for x in args.rates.split(",") if x]:
            arrival = np.cumsum(rng.exponential(1e3 / rate, n_rate))
            out = serve(rate_reqs, arrival)
            v = out["valid"] > 0
            lat = out["result_ms"][v]     # arrival -> validated path on the host
            fin = out["latency_ms"][v]    # arrival -> finish on the device clock
            res[f"{rate:g}_req_s"] = {
                "offered": rate, "requests": n_rate,
                "achieved_plans_per_s": float(v.sum()) / (out["wall_ms"] / 1e3),
                "success_rate": float(v.mean()),
                "p50_ms": pct(lat, 50), "p95_ms": pct(lat, 95), "p99_ms": pct(lat, 99),
                "finish_p50_ms": pct(fin, 50), "finish_p99_ms": pct(fin, 99)}
        return res

    serving = poisson()

    # the same served workload with the other proposal (uniform draws when
    # the headline uses the network, the network when it does not)
    other = None
    if have_net:
        attach(not learned)
        serve(reqs_dev[0])
        o_ms, o_valid, o_service, o_loops, _ = timed_steps(lambda s: reqs_dev[s])
        o_serving = poisson()
        o_t = max_over_ranks(o_ms, world)
        other = {"proposal": "uniform" if learned else f"learned (mix {max(args.mix, 0.8):g})",
                 "value": sum_over_ranks(o_valid, world) / (o_t / 1e3), "unit": "plans/s",
                 "success_rate": o_valid / float(R * args.steps),
                 "service_p50_ms": pct(o_service, 50), "service_p99_ms": pct(o_service, 99),
                 "mean_loops": float(np.mean(o_loops)) if o_loops else None,
                 "serving": o_serving}
        attach(learned)

    def attach_to(pl):
        pl.set_proposal(net if learned else None, mix=args.mix if learned else 0.0)

    c3 = None if args.no_mixed else c3_serving(args, rank, world, tuned, attach_to)
    c2 = None if args.no_mixed else c2_batched(args, rank, world, tuned)

    # kernel timing replay of one step (same inputs, kernels launched one by one)
    planner.profile(True)
    serve(reqs_dev[args.warmup])
    ktimes = planner.kernel_times()
    probes = planner.probes()
    planner.profile(False)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    total_k = sum(v[0] for v in ktimes.values())
    dom = max(ktimes.items(), key=lambda kv: kv[1][0])
    name, (kms, kn) = dom
    per_launch_ms = kms / max(kn, 1)
    # the probe-issue roofline of the dominant search kernel: reference
    # footprint probes per second against one probe per lane per cycle
    peak, sms, mhz = issue_peak(peaks)
    alg = probes.get(name.split("(")[0], 0)
    achieved = (alg / max(kn, 1)) / (per_launch_ms * 1e-3) if alg else 0.0
    hbm = float(peaks.get("hbm_gbs", 6650.0))

    line = None
    if rank == 0:
        plain = plain_loop(args.plain, rank)
        cpu = None if args.no_cpu_baseline else cpu_baseline()
        micro = candidate_microbench(args.candidates, cpu=not args.no_cpu_baseline)
        proposal = (f"learned network (mix {args.mix:g}, fastrrt_b200/proposal_weights.npz)"
                    if learned else "uniform draws")
        line = {
            "metric": METRIC, "value": value, "unit": "plans/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"served C0 planning: {R} requests of seeded {SIZE}x{SIZE} "
                                   f"frames per step and GPU, continuous batching over "
                                   f"{args.slots} slots, {TIMEOUT_MS} ms timeout per request, "
                                   f"expansion proposal: {proposal}",
                       "requests_per_step_per_gpu": R, "slots_per_gpu": args.slots,
                       "check_every": args.check_every,
                       "serving_check_every": args.serving_check_every, "proposal": proposal,
                       "launch_shape": ({k: tuned[k] for k in ("sweep_blocks_per_sm", "work_blocks_per_sm")}
                                        if tuned else "default"),
                       "frame": f"{SIZE}x{SIZE} @ {M_PER_PX} m/px",
                       "parallelism": f"request sharding x{world}",
                       "l2": "fresh frames every step; per-step working set > L2"},
            "success_rate": valid_total / float(R * args.steps),
            "service_p50_ms": pct(service, 50), "service_p99_ms": pct(service, 99),
            "mean_loops": float(np.mean(loops)) if loops else None,
            "mean_path_len_px": float(np.mean(lengths)) if lengths else None,
            "serving": serving,
            "serving_mixed_sizes": c3,
            "batched_mixed_sizes": c2,
            "other_proposal": other,
            "candidate_kernels": micro,
            "plain_gpu_loop": plain,
            "served_over_plain": value / plain["plans_per_s"] if plain["plans_per_s"] else None,
            "e2e": {"value": e2e_plans / (e2e_t / 1e3), "unit": "plans/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": int(sum(v[1] for v in ktimes.values()) * args.steps),
            "roofline": {"bound": "issue", "kernel": name, "achieved": achieved / 1e9, "peak": peak / 1e9,
                         "unit": "Gprobe/s", "frac": achieved / peak if peak else None,
                         "traffic": (NCU_DRAM_BYTES_PER_LAUNCH[name]["bytes"]
                                     if name in NCU_DRAM_BYTES_PER_LAUNCH else None),
                         "traffic_captured": (NCU_DRAM_BYTES_PER_LAUNCH[name]["captured"]
                                              if name in NCU_DRAM_BYTES_PER_LAUNCH else None),
                         "probes_per_launch": alg / max(kn, 1),
                         "algorithmic": "reference footprint probes (class lookups of "
                                        "__computeFeasibleForAngle) the kernel's work stands for, "
                                        f"against one per lane per cycle ({sms} SMs x 32 lanes x "
                                        f"{mhz:g} MHz, of measured clock)",
                         "avg_launch_ms": per_launch_ms, "launches": kn,
                         "share_of_device_time": kms / total_k if total_k else None,
                         "probe_bytes_gbs": alg / max(kn, 1) / (per_launch_ms * 1e-3) / 1e9,
                         "hbm_gbs_of_measured": hbm},
            "kernel_ms": {k: round(v[0], 3) for k, v in ktimes.items()},
            "clocks": clocks,
            "cpu_baseline": cpu,
            "workload_generation_s": gen_s,
        }
        print(json.dumps(line), flush=True)
    barrier(world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return line


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args.gpus, sys.argv[1:]))
    rank, world, local = dist_setup(args.gpus)
    if args.impl == "reference":
        run_reference(args, rank, world)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    run_mine(args, rank, world, local)


if __name__ == "__main__":
    main()
