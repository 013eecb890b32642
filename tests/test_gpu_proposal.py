"""The learned expansion proposal inside the planner: with the network
attached at mix 0 every expansion is the uniform draw, so plans are those of
the planner without it; training rows logged from solves are well formed;
and a network trained on the planner's own solves raises the success rate
on held-out requests under the same loop budget."""
import numpy as np
import pytest

from fastrrt_b200 import synth

pytestmark = pytest.mark.gpu
COSTS = synth.CLASS_COSTS


@pytest.fixture(scope="module")
def torch_gpu(gpu):
    import torch
    return torch


def requests(F, seeds, max_iterations=40):
    out = []
    for s in seeds:
        cls, start, goal, steer, _ = synth.batch_request(s)
        out.append(F.make_request(cls, COSTS, start, goal, max_steering_deg=steer, seed=s,
                                  max_iterations=max_iterations))
    return out


def test_mix_zero_is_the_uniform_planner(gpu):
    from fastrrt_b200.proposal import ProposalNet
    reqs = requests(gpu, range(3000, 3024))
    A = gpu.BatchPlanner(24, 512, 512)
    va, la, _, _ = A.plan(reqs, 60, 4)
    _, _, loops_a = A.status()
    B = gpu.BatchPlanner(24, 512, 512)
    B.set_proposal(ProposalNet(seed=5), mix=0.0)
    vb, lb, _, _ = B.plan(reqs, 60, 4)
    _, _, loops_b = B.status()
    assert np.array_equal(va, vb) and np.array_equal(la, lb) and np.array_equal(loops_a, loops_b)
    for k in range(24):
        assert np.array_equal(A.path(k), B.path(k)), k


def test_logged_rows(gpu, torch_gpu):
    torch = torch_gpu
    from fastrrt_b200 import proposal as P
    X, L, solved = P.collect_dataset(256, seed0=700_000, max_rows=20_000, max_iterations=60)
    assert solved > 0 and len(L) >= solved  # at least one expansion per solved path
    lab = L.cpu().numpy()
    assert lab.min() >= 0 and lab.max() < 128
    x = X.float().cpu().numpy()
    patch = x[:, :1024]
    assert set(np.unique(patch)).issubset({0.0, 0.5, 1.0})
    assert np.all(x[:, 1030:] == 0)
    assert np.all(np.abs(x[:, 1027] ** 2 + x[:, 1028] ** 2 - 1) < 2e-2)  # sin, cos of the heading
    # every accepted expansion of the same (deterministic) solves: more rows,
    # the same form
    Xn, Ln, solved_n = P.collect_dataset(256, seed0=700_000, max_rows=200_000, max_iterations=60,
                                         source="nodes")
    assert solved_n == solved and len(Ln) > len(L)
    lab = Ln.cpu().numpy()
    assert lab.min() >= 0 and lab.max() < 128
    xn = Xn.float().cpu().numpy()
    assert set(np.unique(xn[:, :1024])).issubset({0.0, 0.5, 1.0}) and np.all(xn[:, 1030:] == 0)


def test_trained_proposal_raises_success(gpu, torch_gpu):
    from fastrrt_b200 import proposal as P
    X, L, _ = P.collect_dataset(2048, seed0=500_000, max_rows=200_000)
    net = P.ProposalNet(seed=1, max_batch=512)
    net.train(X, L, len(L), epochs=12, batch=512, lr=1e-3, seed=1)
    r = P.evaluate(net, 1024, seed0=900_000, mix=0.8)
    su = float((r["uniform"]["valid"] > 0).mean())
    sl = float((r["learned"]["valid"] > 0).mean())
    print(f"held-out success: uniform {su:.3f}, learned {sl:.3f}")
    assert sl > su


def test_learned_plans_same_alone_and_in_a_batch(gpu):
    """With the shipped network attached (mix 1.0) a request's plan does not
    depend on the other requests of its batch: its candidates' rows,
    features, logits and draws are its own."""
    from fastrrt_b200 import proposal as P
    from fastrrt_b200 import train_proposal as TP
    net = P.ProposalNet(seed=0, max_batch=512)
    assert TP.load(net)
    reqs = requests(gpu, range(5000, 5012))
    B = gpu.BatchPlanner(12, 512, 512)
    B.set_proposal(net, mix=1.0)
    vb, lb, _, _ = B.plan(reqs, 60, 4)
    _, _, loops_b = B.status()
    A = gpu.BatchPlanner(1, 512, 512)
    A.set_proposal(net, mix=1.0)
    for k in range(len(reqs)):
        va, la, _, _ = A.plan([reqs[k]], 60, 4)
        _, _, loops_a = A.status()
        assert (int(va[0]), float(la[0]), int(loops_a[0])) == (int(vb[k]), float(lb[k]), int(loops_b[k])), k
        assert np.array_equal(A.path(0), B.path(k)), k
