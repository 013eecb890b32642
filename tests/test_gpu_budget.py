"""Admission by device memory: a batched planner with a memory budget gives
each admitted request storage sized by its frame, refuses a request the
arena has no room for and admits it once a finished request gives its
storage back; plans are the same as in a planner whose slots hold the
largest frame, and served requests wait for memory instead of failing."""
import numpy as np
import pytest

from fastrrt_b200 import synth

pytestmark = pytest.mark.gpu
COSTS = synth.CLASS_COSTS


def request(F, seed, size, **kw):
    cls, start, goal, steer, _ = synth.batch_request(seed, sizes=(size,))
    return F.make_request(cls, COSTS, start, goal, max_steering_deg=steer, seed=seed, **kw)


def test_slot_bytes_follow_the_frame(gpu):
    b128, b256, b512 = (gpu.batch.slot_bytes(s, s) for s in (128, 256, 512))
    assert 0 < b128 < b256 < b512
    # the node grid and scratch scale with the cells
    assert 3.5 < b512 / b256 < 4.5 and 3.5 < b256 / b128 < 4.5


def test_budget_refuses_then_admits(gpu):
    b128, b512 = gpu.batch.slot_bytes(128, 128), gpu.batch.slot_bytes(512, 512)
    budget = 2 * b512 + b128
    B = gpu.BatchPlanner(4, 512, 512, budget_bytes=budget)
    assert B.memory()[0] >= budget and B.memory()[1] == 0
    big = [request(gpu, 3000 + k, 512, max_iterations=80) for k in range(3)]
    small = request(gpu, 3100, 128, max_iterations=80)
    B.admit(0, big[0])
    B.admit(1, big[1])
    with pytest.raises(gpu.FastRRTError, match="budget exhausted"):
        B.admit(2, big[2])
    B.admit(2, small)  # the room left fits a 128 x 128 frame
    assert B.memory()[1] == 2 * b512 + b128
    B.run(200, 4)
    B.release(0)
    assert B.memory()[1] == b512 + b128
    B.admit(3, big[2])  # admitted once memory freed
    B.run(200, 4)
    done, goal, loops = B.status()
    valid, _, _ = B.collect(np.array([1, 2, 3]))
    # the same requests in a planner whose slots hold the largest frame
    A = gpu.BatchPlanner(1, 512, 512)
    for slot, r in ((1, big[1]), (2, small), (3, big[2])):
        A.admit(0, r)
        A.run(200, 4)
        _, g1, l1 = A.status()
        v1, _, _ = A.collect(np.array([0]))
        assert (int(goal[slot]), int(loops[slot])) == (int(g1[0]), int(l1[0])), slot
        assert np.array_equal(B.path([1, 2, 3].index(slot)), A.path(0)), slot
    assert B.memory()[2] == 2 * b512 + b128


def test_served_requests_wait_for_memory(gpu):
    """24 mixed-size requests through 8 slots and a budget of two 512 x 512
    frames: requests wait for memory in arrival order, every one is served,
    and each result is the one it gives served alone."""
    rng = np.random.default_rng(11)
    sizes = [int(rng.choice([256, 128, 512], p=[0.6, 0.3, 0.1])) for _ in range(24)]
    sizes[0] = sizes[5] = sizes[9] = 512
    reqs = [request(gpu, 4000 + k, s, max_iterations=60) for k, s in enumerate(sizes)]
    budget = 2 * gpu.batch.slot_bytes(512, 512)
    B = gpu.BatchPlanner(8, 512, 512, budget_bytes=budget)
    mix = B.serve(reqs, arrival_ms=np.cumsum(rng.exponential(0.3, len(reqs))), timeout_ms=0,
                  check_every=2)
    assert B.memory()[1] == 0  # every slot's storage is back in the arena
    assert B.memory()[2] <= budget
    A = gpu.BatchPlanner(1, 512, 512)
    for k in range(len(reqs)):
        one = A.serve([reqs[k]], timeout_ms=0, check_every=2)
        got = (int(mix["valid"][k]), int(mix["loops"][k]), float(mix["length"][k]))
        assert got == (int(one["valid"][0]), int(one["loops"][0]), float(one["length"][0])), k
    assert mix["valid"].sum() >= 1
