"""The multi-GPU path shards requests by rank with no collective on the data
path: two gloo ranks on the CPU check that their request seeds never
overlap, that each rank's plans are its own (the oracle planner run per
rank equals the same requests planned in one process), and that the timing
and result reductions are the maximum and the sum over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    import datetime
    import sys

    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    from oracle import build_oracle, oracle as O
    from fastrrt_b200 import synth
    build_oracle.build_oracle()
    seeds = bench.request_seeds(rank, 1, 3)
    ok = []
    for s in seeds[:2]:
        cls, st, gl = synth.make_frame(s, 128, start=(64, 64), goal=(64, 0)), (64, 64, 0.0), (64, 0, 0.0)
        p = O.Planner(O.Frame(cls, synth.CLASS_COSTS), 128 * 0.135, 128 * 0.135, 40.0, 5.4)
        p.set_plan_data(st, gl, 2.0, (22, 40), seed=s)
        good, it = p.plan(False, 30)
        ok.append([s, int(good), it, len(p.path())])
    gathered = [None] * world
    dist.all_gather_object(gathered, {"seeds": seeds, "plans": ok})
    mx = bench.max_over_ranks(float(rank + 1), world)
    sm = bench.sum_over_ranks(float(rank + 1), world)
    if rank == 0:
        np.save(os.path.join(out_dir, "result.npy"),
                np.array([gathered, mx, sm], dtype=object), allow_pickle=True)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_shard_requests(tmp_path, orc):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    gathered, mx, sm = np.load(tmp_path / "result.npy", allow_pickle=True)
    s0, s1 = set(gathered[0]["seeds"]), set(gathered[1]["seeds"])
    assert not (s0 & s1)
    assert mx == 2.0 and sm == 3.0
    # each rank's plans equal the same requests planned here
    from fastrrt_b200 import synth
    for r in range(world):
        for s, good, it, n in gathered[r]["plans"]:
            cls = synth.make_frame(s, 128, start=(64, 64), goal=(64, 0))
            p = orc.Planner(orc.Frame(cls, synth.CLASS_COSTS), 128 * 0.135, 128 * 0.135, 40.0, 5.4)
            p.set_plan_data((64, 64, 0.0), (64, 0, 0.0), 2.0, (22, 40), seed=s)
            g2, it2 = p.plan(False, 30)
            assert (int(g2), it2, len(p.path())) == (good, it, n)


def test_bench_starts_its_own_ranks():
    """`bench.py --gpus 2` without a torchrun environment starts two ranks
    itself (torch.distributed.run on 127.0.0.1, gloo without a GPU); the
    reference arm runs on rank 0 alone and prints one line for both ranks,
    the other rank exits 0 without work."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--gpus", "2", "--impl",
                        "reference", "--steps", "1", "--warmup", "0", "--ref-plans", "1"],
                       capture_output=True, text=True, timeout=600, env=env, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    assert lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2
