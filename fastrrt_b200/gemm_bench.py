"""Throughput of the proposal network's tcgen05 GEMM on the network's own
shapes at the planner's row capacity (layers 1-3 forward, an input gradient,
the largest weight gradient) and on an 8192^3 product, by CUDA events over 20
launches after 3 warm-up launches; one JSON line per shape with the error
against torch's f32 product of the same bf16 inputs.

    python -m fastrrt_b200.gemm_bench
"""
import json

import torch

from fastrrt_b200.proposal import gemm


def main():
    torch.manual_seed(0)
    res = []
    ws = torch.empty(16 * 256 * 1040, device="cuda", dtype=torch.float32)
    shapes = [(131072, 256, 1040, 0, 0, "fwd L1", None), (131072, 256, 256, 0, 0, "fwd L2", None),
              (131072, 128, 256, 0, 0, "fwd L3", None), (131072, 256, 128, 0, 1, "dH2", None),
              (256, 1040, 131072, 1, 1, "dW1", None), (256, 1040, 4096, 1, 1, "dW1, 4096 rows", None),
              (256, 1040, 4096, 1, 1, "dW1, 4096 rows, split over K", ws),
              (8192, 8192, 8192, 0, 0, "square 8k", None)]
    for (M, N, K, ta, tb, name, split) in shapes:
        A = (torch.randn((K, M) if ta else (M, K), device="cuda") * 0.1).to(torch.bfloat16)
        B = (torch.randn((K, N) if tb else (N, K), device="cuda") * 0.1).to(torch.bfloat16)
        out = torch.empty((M, N), device="cuda", dtype=torch.float32)
        for _ in range(3):
            gemm(A, B, trans_a=bool(ta), trans_b=bool(tb), out=out, split_ws=split)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n = 20
        e0.record()
        for _ in range(n):
            gemm(A, B, trans_a=bool(ta), trans_b=bool(tb), out=out, split_ws=split)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / n
        ref = (A.float().T if ta else A.float()) @ (B.float() if tb else B.float().T)
        err = float((out - ref).abs().max() / ref.abs().max())
        res.append({"shape": name, "M": M, "N": N, "K": K, "ms": ms, "tflops": 2 * M * N * K / ms / 1e9,
                    "gbs_min_bytes": (2 * (M * K + N * K) + 4 * M * N) / ms / 1e6, "rel_err": err})
        print(json.dumps(res[-1]), flush=True)


if __name__ == "__main__":
    main()
