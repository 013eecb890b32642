"""The learned expansion proposal: a BF16 MLP (1030 -> 256 -> 256 -> 128)
trained with the library's own kernels on expansions the planner accepted on
its solution paths (fastrrt_mlp_* in the C ABI)."""
import ctypes as C

import numpy as np

from . import _lib

N_IN = 1030
N_IN_PAD = 1040
HIDDEN = 256
N_OUT = 128
STEER_BINS = 16
LEN_BINS = 8
SHAPES = [(HIDDEN, N_IN_PAD), (HIDDEN,), (HIDDEN, HIDDEN), (HIDDEN,), (N_OUT, HIDDEN), (N_OUT,)]
# GEMM FLOPs of one training row: forward (3 layers) + backward (the weight
# gradients of all three layers, the input gradients of layers 2 and 3)
FWD_FLOP_PER_ROW = 2 * (HIDDEN * N_IN_PAD + HIDDEN * HIDDEN + N_OUT * HIDDEN)
TRAIN_FLOP_PER_ROW = FWD_FLOP_PER_ROW + 2 * (HIDDEN * N_IN_PAD + 2 * HIDDEN * HIDDEN + 2 * N_OUT * HIDDEN)


class ProposalNet:
    def __init__(self, seed=0, max_batch=4096):
        h = _lib.lib().fastrrt_mlp_create(int(seed), int(max_batch))
        if not h:
            raise _lib.FastRRTError("mlp_create: " + _lib.last_error())
        self._h = h
        self.max_batch = max_batch

    def __del__(self):
        try:
            if getattr(self, "_h", None) and _lib._lib is not None:
                _lib.lib().fastrrt_mlp_destroy(self._h)
                self._h = None
        except (AttributeError, TypeError):
            pass  # interpreter shutdown

    @property
    def handle(self):
        return self._h

    def get_weights(self):
        ws = [np.zeros(s, np.float32) for s in SHAPES]
        _lib.check(_lib.lib().fastrrt_mlp_get_weights(self._h, *[w.reshape(-1) for w in ws]),
                   "mlp_get_weights")
        return ws

    def set_weights(self, ws):
        ws = [np.ascontiguousarray(w, np.float32).reshape(-1) for w in ws]
        _lib.check(_lib.lib().fastrrt_mlp_set_weights(self._h, *ws), "mlp_set_weights")

    def forward(self, X):
        X = np.ascontiguousarray(X, np.float32).reshape(-1, N_IN)
        out = np.zeros((len(X), N_OUT), np.float32)
        _lib.check(_lib.lib().fastrrt_mlp_forward(self._h, len(X), X.reshape(-1), out.reshape(-1)),
                   "mlp_forward")
        return out

    def gradients(self, X, labels):
        X = np.ascontiguousarray(X, np.float32).reshape(-1, N_IN)
        labels = np.ascontiguousarray(labels, np.int32)
        gs = [np.zeros(s, np.float32) for s in SHAPES]
        loss = C.c_float(0)
        _lib.check(_lib.lib().fastrrt_mlp_gradients(self._h, len(X), X.reshape(-1), labels,
                                                     *[g.reshape(-1) for g in gs], C.byref(loss)),
                   "mlp_gradients")
        return gs, loss.value

    def train(self, X_dev, labels_dev, n, epochs=4, batch=1024, lr=1e-3, seed=0):
        """Adam on a device dataset (X_dev: n x 1040 bf16, labels_dev: n int32,
        e.g. torch tensors); returns the mean loss of the last batch."""
        loss = C.c_float(0)
        _lib.check(_lib.lib().fastrrt_mlp_train(self._h, X_dev.data_ptr(), labels_dev.data_ptr(), int(n),
                                                int(epochs), int(batch), float(lr), int(seed),
                                                C.byref(loss)), "mlp_train")
        return loss.value


def collect_dataset(n_plans, seed0=500_000, max_rows=200_000, slots=256, max_iterations=100,
                    sizes=(128, 256, 512), c0_share=0.0, net=None, mix=0.8, source="paths"):
    """Training rows from the planner's own solves of seeded batched requests
    (mixed frame sizes, 5-30% obstacles; a share `c0_share` of them the
    single-instance 256 x 256 layout, start at the centre, goal top centre),
    with `net` attached at `mix` when given.  source "paths": one row per
    expansion on every validated path; "nodes": one row per accepted
    expansion (node of the final graph) of every solved request; "both":
    the two sets (a path's expansions then appear twice).  Stops at max_rows.
    Returns device tensors (X: rows x 1040 bf16, labels: int32) and the
    number of plans solved."""
    import torch

    from . import synth
    from .batch import BatchPlanner, make_request
    size_max = max(sizes)
    planner = BatchPlanner(slots, size_max, size_max)
    if net is not None:
        planner.set_proposal(net, mix=mix)
    X = torch.zeros((max_rows, N_IN_PAD), dtype=torch.bfloat16, device="cuda")
    labels = torch.zeros(max_rows, dtype=torch.int32, device="cuda")
    rows = solved = 0
    for b0 in range(0, n_plans, slots):
        reqs = []
        for k in range(b0, min(n_plans, b0 + slots)):
            if (k % 100) < int(round(100 * c0_share)):
                cls, start, goal = synth.c0_request(seed0 + k)
                steer = 40.0
            else:
                cls, start, goal, steer, _ = synth.batch_request(seed0 + k, sizes=sizes)
            reqs.append(make_request(cls, synth.CLASS_COSTS, start, goal, max_steering_deg=steer,
                                     seed=seed0 + k, max_iterations=max_iterations))
        valid, _, _, _ = planner.plan(reqs, max_launches=max_iterations + 8, check_every=4)
        solved += int(valid.sum())
        if source in ("paths", "both"):
            rows += planner.log_paths(X, labels, rows, max_rows)
        if source in ("nodes", "both") and rows < max_rows:
            rows += planner.log_nodes(X, labels, rows, max_rows)
        if rows >= max_rows:
            break
    return X[:rows], labels[:rows], solved


def evaluate(net, n_plans, seed0, mix=0.5, slots=256, max_iterations=60, sizes=(128, 256, 512)):
    """Solve seeded requests with and without the network attached; returns
    per-request validity and loop counts for both."""
    from . import synth
    from .batch import BatchPlanner, make_request
    size_max = max(sizes)
    out = {}
    for name, use in (("uniform", False), ("learned", True)):
        planner = BatchPlanner(slots, size_max, size_max)
        if use:
            planner.set_proposal(net, mix=mix)
        valid, loops = [], []
        for b0 in range(0, n_plans, slots):
            reqs = []
            for k in range(b0, min(n_plans, b0 + slots)):
                cls, start, goal, steer, _ = synth.batch_request(seed0 + k, sizes=sizes)
                reqs.append(make_request(cls, synth.CLASS_COSTS, start, goal, max_steering_deg=steer,
                                         seed=seed0 + k, max_iterations=max_iterations))
            v, _, _, _ = planner.plan(reqs, max_launches=max_iterations + 8, check_every=4)
            _, _, lp = planner.status()
            valid.extend(v.tolist())
            loops.extend(lp[:len(reqs)].tolist())
        out[name] = {"valid": np.array(valid), "loops": np.array(loops)}
    return out


def gemm(A, B, trans_a=False, trans_b=False, bias=None, relu=False, mask=None, out=None, M=None,
         d_count=None, split_ws=None):
    """The network's tcgen05 GEMM on torch CUDA tensors (bf16 A, B; see
    fastrrt_gemm_bf16): out (M x N, f32 or bf16) = epilogue(A(m, k) B(k, n))
    with A (M x K), or (K x M) when trans_a; B (N x K) -- a weight matrix --,
    or (K x N) when trans_b.  Row strides are the tensors' own.  split_ws: an
    f32 CUDA tensor for the split over K of a raw f32 product."""
    import torch
    assert A.dtype == torch.bfloat16 and B.dtype == torch.bfloat16 and A.is_cuda and B.is_cuda
    K = A.shape[0] if trans_a else A.shape[1]
    Mx = A.shape[1] if trans_a else A.shape[0]
    N = B.shape[1] if trans_b else B.shape[0]
    M = Mx if M is None else M
    if out is None:
        out = torch.empty((M, N), dtype=torch.float32, device=A.device)
    cf = out.data_ptr() if out.dtype == torch.float32 else None
    cb = out.data_ptr() if out.dtype == torch.bfloat16 else None
    _lib.check(_lib.lib().fastrrt_gemm_bf16(
        M, N, K, A.data_ptr(), A.stride(0), int(trans_a), B.data_ptr(), B.stride(0), int(trans_b),
        None if bias is None else bias.data_ptr(), int(relu), None if mask is None else mask.data_ptr(),
        0 if mask is None else mask.stride(0), cf, cb, out.stride(0),
        None if d_count is None else d_count.data_ptr(), None if split_ws is None else split_ws.data_ptr(),
        0 if split_ws is None else split_ws.numel(), torch.cuda.current_stream().cuda_stream), "gemm")
    return out
