"""The proposal network's GPU kernels (tensor-core GEMMs, softmax
cross-entropy, bias reductions, Adam) against the CPU oracle."""
import numpy as np
import pytest

from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-12))


@pytest.fixture
def net(gpu):
    from fastrrt_b200.proposal import ProposalNet
    return ProposalNet(seed=3, max_batch=512)


def test_forward_matches_oracle(net):
    rng = np.random.default_rng(1)
    ws = M.random_weights(rng)
    for w in ws[1::2]:
        w[:] = rng.standard_normal(w.shape).astype(np.float32) * 0.1
    net.set_weights(ws)
    X = (rng.random((300, 1030)) < 0.3).astype(np.float32)
    X[:, 1024:] = rng.standard_normal((300, 6))
    got = net.forward(X)
    _, _, _, want = M.forward(ws, X)
    # bf16 hidden activations: a summation order that differs may move a
    # value across a rounding boundary, so compare in norm
    assert rel(got, want) < 1e-2
    assert np.abs(got - want).max() < 0.05 * np.abs(want).max()


def test_gradients_match_oracle(net):
    rng = np.random.default_rng(2)
    ws = M.random_weights(rng)
    net.set_weights(ws)
    X = (rng.random((256, 1030)) < 0.3).astype(np.float32)
    labels = rng.integers(0, 128, 256).astype(np.int32)
    gs, loss = net.gradients(X, labels)
    want, want_loss = M.gradients(ws, X, labels)
    assert abs(loss - want_loss) < 1e-3 * max(1.0, abs(want_loss))
    for t, (g, w) in enumerate(zip(gs, want)):
        assert rel(g, w) < 3e-2, (t, rel(g, w))
    # padding inputs get no gradient
    assert np.all(gs[0][:, 1030:] == 0)


def test_training_reduces_loss(net, torch_gpu):
    torch = torch_gpu
    rng = np.random.default_rng(4)
    n = 4096
    X = (rng.random((n, 1030)) < 0.2).astype(np.float32)
    # a learnable rule: the label is set by two patch cells and the goal side
    labels = (X[:, 0] * 64 + X[:, 500] * 32 + (X[:, 1024] > 0.1) * 16).astype(np.int32)
    Xp = M.pad_inputs(X)
    Xd = torch.from_numpy(Xp).to(torch.bfloat16).cuda().contiguous()
    Ld = torch.from_numpy(labels).cuda()
    _, l0 = net.gradients(X[:512], labels[:512])
    l1 = net.train(Xd, Ld, n, epochs=6, batch=256, lr=2e-3, seed=1)
    assert l1 < 0.5 * l0, (l0, l1)
    logits = net.forward(X[:512])
    assert (logits.argmax(1) == labels[:512]).mean() > 0.9


@pytest.fixture(scope="module")
def torch_gpu(gpu):
    import torch
    return torch
