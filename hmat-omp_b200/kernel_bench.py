"""Kernel micro-benchmark of the library's batched dense kernels through the C ABI
(hm_gemm_batched_*_device, hm_inverse_batched_device), on batches shaped like the
headline factorization's (Coulomb 2-D, N = 2^18, leaf 256, ranks 96).

    python hmat-omp_b200/kernel_bench.py gemm --dtype f32 --kernel fma
    python hmat-omp_b200/kernel_bench.py gemm --dtype f64 --kernel tc      # FP64 MMA
    python hmat-omp_b200/kernel_bench.py inverse --order 256 --count 1024

Default GEMM batch: the factorization's basis correction W -= Q delta at one level:
`count` problems of m x n x k = 1024 x 96 x 96 with beta = 1 (C read and written).
Prints one JSON line: per-launch CUDA-event time (mean of --iters launches after
--warmup), algorithmic flops (2 m n k per problem) and bytes (A, B, C read, C written),
and the rates.  A target for ncu captures of one kernel on a headline-sized batch.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["gemm", "inverse"])
    ap.add_argument("--dtype", default="f32", choices=["f32", "f64"])
    ap.add_argument("--kernel", default="fma", choices=["fma", "tc", "auto"])
    ap.add_argument("--count", type=int, default=2048)
    ap.add_argument("--m", type=int, default=1024)
    ap.add_argument("--n", type=int, default=96)
    ap.add_argument("--k", type=int, default=96)
    ap.add_argument("--beta", type=float, default=1.0)
    ap.add_argument("--opa", type=int, default=0, choices=[0, 1],
                    help="1: op(A) = A^T with A stored k x m (the projections V^T x: m = rank, k = node rows)")
    ap.add_argument("--ksplit", type=int, default=1, help="k slices per problem (0: the library's choice)")
    ap.add_argument("--order", type=int, default=256, help="inverse: matrix order")
    ap.add_argument("--iters", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    a = ap.parse_args()
    import numpy as np
    import torch

    import hmat_b200 as H
    dev = torch.device("cuda", 0)
    torch.cuda.set_stream(torch.cuda.Stream(device=dev))
    stream = torch.cuda.current_stream()
    d = H.Dense()
    d.set_stream(stream.cuda_stream)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if a.what == "gemm":
        dt = torch.float32 if a.dtype == "f32" else torch.float64
        w = 4 if a.dtype == "f32" else 8
        # each problem column-major: m x k (opa 0) or k x m (opa 1)
        A = torch.randn(a.count, a.k, a.m, dtype=dt, device=dev) if a.opa == 0 else \
            torch.randn(a.count, a.m, a.k, dtype=dt, device=dev)
        B = torch.randn(a.count, a.n, a.k, dtype=dt, device=dev)     # k x n
        C = torch.randn(a.count, a.n, a.m, dtype=dt, device=dev)     # m x n
        flags = {"fma": H.GEMM_FMA, "tc": H.GEMM_TENSOR_CORES, "auto": H.GEMM_AUTO}[a.kernel]
        args = ([a.m] * a.count, [a.n] * a.count, [a.k] * a.count, 1.0, [A[i].data_ptr() for i in range(a.count)],
                [a.m if a.opa == 0 else a.k] * a.count, a.opa, [B[i].data_ptr() for i in range(a.count)], [a.k] * a.count, 0, a.beta,
                [C[i].data_ptr() for i in range(a.count)], [a.m] * a.count)

        def run():
            d.gemm(*args, ksplit=a.ksplit, flags=flags, dtype=a.dtype)
        flops = 2.0 * a.m * a.n * a.k * a.count
        nbytes = w * a.count * (a.m * a.k + a.k * a.n + a.m * a.n * (2 if a.beta != 0 else 1))
    else:
        n = a.order
        rng = np.random.default_rng(0)
        M = rng.standard_normal((a.count, n, n)) / np.sqrt(n) + 2.0 * np.eye(n)
        A = torch.from_numpy(M).to(dev)
        X = torch.empty_like(A)
        args = None

        def run():
            d.inverse([n] * a.count, [A[i].data_ptr() for i in range(a.count)], [n] * a.count,
                      [X[i].data_ptr() for i in range(a.count)], [n] * a.count)
        flops = 2.0 * n ** 3 * a.count
        nbytes = 16.0 * n * n * a.count
    for _ in range(a.warmup):
        run()
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(a.iters):
        run()
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / a.iters
    print(json.dumps({"what": a.what, "dtype": a.dtype, "kernel": a.kernel, "count": a.count, "m": a.m, "n": a.n,
                      "k": a.k, "beta": a.beta, "opa": a.opa, "ksplit": a.ksplit, "ms_per_launch_incl_host": ms, "flops": flops, "bytes": nbytes,
                      "tflops": flops / ms / 1e9, "gbs": nbytes / ms / 1e6,
                      "note": "each call also plans and uploads its tables (synchronising): the time includes that"}))


if __name__ == "__main__":
    main()
