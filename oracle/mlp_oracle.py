"""CPU oracle of the learned proposal's network (test infrastructure only):
the forward pass and the mean cross-entropy gradients of the BF16 MLP in
numpy, with bf16 rounding (round to nearest even) at the points where the GPU
kernels round: inputs, weights, hidden activations and their gradients, the
logit gradients.  With round=False the same network runs in float64, which a
finite-difference test pins."""
import numpy as np


def bf16(x):
    """round float32 values to bfloat16 (nearest even), returned as float32"""
    x = np.ascontiguousarray(x, np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).reshape(x.shape)


def pad_inputs(X, width=1040):
    X = np.asarray(X, np.float32)
    out = np.zeros((len(X), width), np.float32)
    out[:, :X.shape[1]] = X
    return out


def forward(ws, X, round=True):
    w1, b1, w2, b2, w3, b3 = ws
    r = bf16 if round else (lambda a: np.asarray(a, np.float64))
    X = r(pad_inputs(X))
    h1 = r(np.maximum(X @ r(w1).T + b1, 0))
    h2 = r(np.maximum(h1 @ r(w2).T + b2, 0))
    logits = h2 @ r(w3).T + b3
    return X, h1, h2, logits


def gradients(ws, X, labels, round=True):
    w1, b1, w2, b2, w3, b3 = ws
    r = bf16 if round else (lambda a: np.asarray(a, np.float64))
    Xp, h1, h2, logits = forward(ws, X, round)
    n = len(labels)
    z = logits - logits.max(1, keepdims=True)
    p = np.exp(z)
    p /= p.sum(1, keepdims=True)
    loss = float(-np.log(np.maximum(p[np.arange(n), labels], 1e-30)).mean())
    y = np.zeros_like(p)
    y[np.arange(n), labels] = 1
    dl = r((p - y) / n)
    gw3 = dl.T @ h2
    gb3 = dl.sum(0)
    dh2 = r((dl @ r(w3)) * (h2 > 0))
    gw2 = dh2.T @ h1
    gb2 = dh2.sum(0)
    dh1 = r((dh2 @ r(w2)) * (h1 > 0))
    gw1 = dh1.T @ Xp
    gb1 = dh1.sum(0)
    return [gw1, gb1, gw2, gb2, gw3, gb3], loss


def loss_only(ws, X, labels):
    _, _, _, logits = forward(ws, X, round=False)
    z = logits - logits.max(1, keepdims=True)
    lp = z - np.log(np.exp(z).sum(1, keepdims=True))
    return float(-lp[np.arange(len(labels)), labels].mean())


def random_weights(rng, scale=1.0):
    shapes = [(256, 1040), (256,), (256, 256), (256,), (128, 256), (128,)]
    ws = []
    for s in shapes:
        fan = s[1] if len(s) == 2 else 1
        ws.append((rng.standard_normal(s) * scale * np.sqrt(2.0 / fan)).astype(np.float32))
    ws[0][:, 1030:] = 0
    return ws
