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
