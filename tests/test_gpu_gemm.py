"""The proposal network's tcgen05 GEMM (TMA-fed shared-memory ring, TMEM
accumulator) against a float64 reference of the same op on the same bf16
inputs, for every operand layout the network uses (forward: both K-major;
dH = dY W: B MN-major; dW = dY^T X: both MN-major), ragged M / N / K, strides
wider than the extent, the epilogues and the device-side row count.

Tolerance: f32 results within 3e-5 of sum_k |A(m,k)| |B(k,n)| (+1e-6), the
order of FP32 accumulation being the only difference; bf16 results within
one bf16 rounding (2^-8 relative) on top of that."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def T(gpu):
    import torch
    return torch


def operands(T, rng, M, N, K, trans_a, trans_b, pad=0):
    a = T.from_numpy(rng.standard_normal((K, M + pad) if trans_a else (M, K + pad)).astype(np.float32))
    b = T.from_numpy(rng.standard_normal((K, N + pad) if trans_b else (N, K + pad)).astype(np.float32))
    A = a.to(T.bfloat16).cuda()
    B = b.to(T.bfloat16).cuda()
    if pad:
        A = A[:, :M] if trans_a else A[:, :K]
        B = B[:, :N] if trans_b else B[:, :K]
    a64 = A.float().cpu().double()
    b64 = B.float().cpu().double()
    Am = a64.T if trans_a else a64          # M x K
    Bm = b64 if trans_b else b64.T          # K x N
    return A, B, Am, Bm


def check(got, want, bound, bf16):
    got = got.float().cpu().double()
    tol = 3e-5 * bound + 1e-6
    if bf16:
        tol = tol + 2.0 ** -8 * want.abs()
    err = (got - want).abs()
    assert bool((err <= tol).all()), float((err - tol).max())


CASES = [
    # M, N, K, trans_a, trans_b
    (1000, 256, 1040, 0, 0),     # layer 1 forward (K ragged: 16 x 64 + 16)
    (300, 128, 256, 0, 0),       # layer 3 forward
    (1, 8, 16, 0, 0),            # smallest
    (700, 256, 128, 0, 1),       # dH2 = dL W3
    (513, 256, 256, 0, 1),       # dH1 = dH2 W2
    (256, 1040, 512, 1, 1),      # dW1 = dH1^T X (N ragged)
    (128, 256, 300, 1, 1),       # dW3 = dL^T H2 (K ragged)
    (200, 200, 200, 1, 0),       # MN-major A, K-major B
]


@pytest.mark.parametrize("M,N,K,ta,tb", CASES)
def test_gemm_f32_matches_float64(T, M, N, K, ta, tb):
    from fastrrt_b200.proposal import gemm
    rng = np.random.default_rng(M * 7 + N * 3 + K)
    A, B, Am, Bm = operands(T, rng, M, N, K, ta, tb)
    got = gemm(A, B, trans_a=bool(ta), trans_b=bool(tb))
    check(got, Am @ Bm, Am.abs() @ Bm.abs(), False)


@pytest.mark.parametrize("M,N,K,ta,tb", [(1000, 256, 1040, 0, 0), (513, 256, 256, 0, 1),
                                         (256, 1040, 512, 1, 1)])
def test_gemm_epilogues(T, M, N, K, ta, tb):
    from fastrrt_b200.proposal import gemm
    rng = np.random.default_rng(K)
    A, B, Am, Bm = operands(T, rng, M, N, K, ta, tb, pad=8)   # row strides wider than the extent
    bias = T.from_numpy(rng.standard_normal(N).astype(np.float32)).cuda()
    mask = T.from_numpy((rng.random((M, N)) < 0.5).astype(np.float32)).to(T.bfloat16).cuda()
    ref = Am @ Bm
    bound = Am.abs() @ Bm.abs()
    b64 = bias.cpu().double()
    # bias + ReLU, bf16 out
    out = T.empty((M, N), dtype=T.bfloat16, device="cuda")
    gemm(A, B, trans_a=bool(ta), trans_b=bool(tb), bias=bias, relu=True, out=out)
    check(out, (ref + b64).clamp(min=0), bound, True)
    # ReLU-mask (the backward pass's), bf16 out
    gemm(A, B, trans_a=bool(ta), trans_b=bool(tb), mask=mask, out=out)
    check(out, ref * (mask.float().cpu().double() > 0), bound, True)
    # bias, f32 out into a wider destination
    wide = T.full((M, N + 24), 7.0, dtype=T.float32, device="cuda")
    gemm(A, B, trans_a=bool(ta), trans_b=bool(tb), bias=bias, out=wide[:, :N])
    check(wide[:, :N], ref + b64, bound, False)
    assert bool((wide[:, N:] == 7.0).all())


def test_gemm_device_row_count(T):
    """rows at and beyond *d_count are not written (the planner's proposal
    rows are a device count below the buffer's capacity)"""
    from fastrrt_b200.proposal import gemm
    rng = np.random.default_rng(5)
    M, N, K = 4096, 256, 1040
    A, B, Am, Bm = operands(T, rng, M, N, K, 0, 0)
    for cnt in (0, 1, 777, 4096, 9999):
        d = T.tensor([cnt], dtype=T.int32, device="cuda")
        out = T.full((M, N), -3.0, dtype=T.float32, device="cuda")
        gemm(A, B, out=out, d_count=d)
        c = min(cnt, M)
        if c:
            check(out[:c], Am[:c] @ Bm, Am[:c].abs() @ Bm.abs(), False)
        assert bool((out[c:] == -3.0).all())


def test_gemm_rejects_unaligned_strides(T, gpu):
    from fastrrt_b200.proposal import gemm
    A = T.zeros((64, 104), dtype=T.bfloat16, device="cuda")[:, :99]   # 208-byte rows: a TMA stride
    B = T.zeros((32, 99), dtype=T.bfloat16, device="cuda")             # 198-byte rows: not a TMA stride
    with pytest.raises(gpu.FastRRTError):
        gemm(A, B)


@pytest.mark.parametrize("M,N,K", [(256, 1040, 4096), (128, 256, 4096), (256, 256, 1000)])
def test_gemm_split_over_k(T, M, N, K):
    """weight-gradient shapes (both operands MN-major, few output tiles, long
    K) split over K into the workspace and reduced in a fixed order: the
    float64 bound holds and two runs are bit-identical"""
    from fastrrt_b200.proposal import gemm
    rng = np.random.default_rng(M + N + K)
    A, B, Am, Bm = operands(T, rng, M, N, K, 1, 1)
    ws = T.empty(16 * M * N, dtype=T.float32, device="cuda")
    got = gemm(A, B, trans_a=True, trans_b=True, split_ws=ws)
    check(got, Am @ Bm, Am.abs() @ Bm.abs(), False)
    again = gemm(A, B, trans_a=True, trans_b=True, split_ws=ws)
    assert T.equal(got, again)
    # too small a workspace: the unsplit product, within the same bound
    small = gemm(A, B, trans_a=True, trans_b=True, split_ws=ws[:M * N])
    check(small, Am @ Bm, Am.abs() @ Bm.abs(), False)


def test_fused_forward_equals_the_layer_gemms(T, gpu):
    """The network's one-kernel forward pass (activations kept in shared
    memory between the layers) against three single GEMM launches with the
    same epilogues on the same bf16 operands: bit-identical logits."""
    from fastrrt_b200 import proposal as P
    from oracle import mlp_oracle as M
    rng = np.random.default_rng(9)
    ws = M.random_weights(rng)
    for w in ws[1::2]:
        w[:] = rng.standard_normal(w.shape).astype(np.float32) * 0.1
    net = P.ProposalNet(seed=1, max_batch=512)
    net.set_weights(ws)
    for n in (1, 129, 300, 512):
        X = (rng.random((n, 1030)) < 0.3).astype(np.float32)
        X[:, 1024:] = rng.standard_normal((n, 6))
        got = T.from_numpy(net.forward(X))
        Xp = np.zeros((n, 1040), np.float32)
        Xp[:, :1030] = X
        xb = T.from_numpy(Xp).to(T.bfloat16).cuda()
        w1, b1, w2, b2, w3, b3 = [T.from_numpy(np.ascontiguousarray(w)).cuda() for w in ws]
        h1 = P.gemm(xb, w1.to(T.bfloat16), bias=b1, relu=True, out=T.empty((n, 256), dtype=T.bfloat16, device="cuda"))
        h2 = P.gemm(h1, w2.to(T.bfloat16), bias=b2, relu=True, out=T.empty((n, 256), dtype=T.bfloat16, device="cuda"))
        want = P.gemm(h2, w3.to(T.bfloat16), bias=b3).cpu()
        assert T.equal(got, want), (n, float((got - want).abs().max()))
