"""The CPU oracle of the proposal network: its backward pass equals finite
differences of its float64 loss, and bf16 rounding behaves as the GPU's."""
import numpy as np

from oracle import mlp_oracle as M


def test_bf16_rounding_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0, 0.0], np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0          # exactly half an ulp: ties to even
    assert r[2] == 1.0078125    # above half: up
    assert abs(r[3] + 3.140625) < 1e-6
    assert r[5] == 0.0


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    ws = [w.astype(np.float64) for w in M.random_weights(rng, 0.5)]
    for w in ws[1::2]:
        w[:] = rng.standard_normal(w.shape) * 0.1
    X = rng.random((6, 1030))
    labels = rng.integers(0, 128, 6)
    gs, loss = M.gradients(ws, X, labels, round=False)
    assert abs(loss - M.loss_only(ws, X, labels)) < 1e-9
    eps = 1e-6
    for t, idxs in ((0, [(3, 7), (100, 1029)]), (1, [(5,)]), (2, [(9, 200)]), (3, [(17,)]),
                    (4, [(0, 0), (127, 255)]), (5, [(64,)])):
        for ix in idxs:
            wp = [w.copy() for w in ws]
            wm = [w.copy() for w in ws]
            wp[t][ix] += eps
            wm[t][ix] -= eps
            num = (M.loss_only(wp, X, labels) - M.loss_only(wm, X, labels)) / (2 * eps)
            assert abs(num - gs[t][ix]) < 1e-6 + 1e-4 * abs(num), (t, ix, num, gs[t][ix])


def test_shipped_weights_fit_the_network():
    """fastrrt_b200/proposal_weights.npz: the network's shapes (1040 -> 256
    -> 256 -> 128), finite values, the training record it was made from, and
    finite logits through the oracle's bf16 forward pass"""
    import os

    from fastrrt_b200 import proposal as P
    path = os.path.join(os.path.dirname(P.__file__), "proposal_weights.npz")
    d = np.load(path)
    ws = [d[k] for k in ["w1", "b1", "w2", "b2", "w3", "b3"]]
    assert [w.shape for w in ws] == [tuple(s) for s in P.SHAPES]
    assert all(np.isfinite(w).all() for w in ws)
    # the padded input columns past the 1030 features never see a nonzero
    # input, whatever their weights
    assert P.N_IN == 1030 and P.N_IN_PAD == ws[0].shape[1]
    assert int(d["rows"]) > 100000 and int(d["solved"]) <= int(d["plans"])
    assert str(d["source"]) == "paths"
    rng = np.random.default_rng(3)
    X = rng.random((64, P.N_IN)).astype(np.float32)
    X[:, :1024] = rng.random((64, 1024)) < 0.2
    _, _, _, logits = M.forward(ws, X)
    assert logits.shape == (64, P.N_OUT) and np.isfinite(logits).all()
    assert logits.std(axis=1).min() > 0
