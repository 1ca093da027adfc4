"""Measures the FP64 complex GEMM kernels per shape bucket and writes the
kernel table the library uses (``rcwa_set_gemm_table``).

    python -m rcwa_b200.tune            (from rcwa-cuda_b200/, on the GPU)

The solve path multiplies matrices of very different shapes: rank-32 updates
of the blocked LU and Hessenberg reductions (k = 32), the recursive
triangular solves (k up to n / 2) and the S-matrix algebra (k = n), for n
from 50 to 2000.  Four FP64 kernels compete: the FP64 tensor-core (DMMA)
kernel with cp.async tile loads on 64 x 64 and on 32 x 64 complex tiles, the
64 x 64 DMMA kernel fed by the tensor memory accelerator (TMA) through an
mbarrier ring, and the CUDA-core kernel.  For every bucket -- k in (<= 16, <= 32,
<= 64, <= 128, larger) by min(m, n) in (<= 64, <= 128, <= 256, <= 512,
larger) -- the tuner times both kernels on a representative square shape,
in both forms the solver issues (C = A B and the update C = C - A B), with a
batch that gives each launch a few GFLOP, and keeps the fastest.  The
table is written next to this file (``gemm_tuning_b200.json``); the Python
binding applies it when the first context is created.
"""
from __future__ import annotations

import json
import os
import time

PKG = os.path.dirname(os.path.abspath(__file__))
TABLE_PATH = os.path.join(PKG, "gemm_tuning_b200.json")

K_BUCKETS = [16, 32, 64, 128, 450]          # representative k of each k bucket
SIZE_BUCKETS = [48, 98, 200, 450, 900]      # representative m = n of each size bucket
K_LIMITS = ["k<=16", "k<=32", "k<=64", "k<=128", "k>128"]
SIZE_LIMITS = ["mn<=64", "mn<=128", "mn<=256", "mn<=512", "mn>512"]


def _time_kernel(ctx, lib, torch, stream, choice, s, k, batch, reps=5):
    """Median ms of C = A B plus C = C - A B with every bucket forced to
    `choice` (0 = DMMA with cp.async, 1 = CUDA cores, 2 = DMMA fed by TMA,
    3 = DMMA with cp.async on 32 x 64 tiles)."""
    import ctypes as C
    arr = (C.c_int * 25)(*([choice] * 25))
    assert lib.rcwa_set_gemm_table(arr) == 0
    A = torch.randn(batch, k, s, dtype=torch.complex128, device="cuda")   # column-major s x k
    B = torch.randn(batch, s, k, dtype=torch.complex128, device="cuda")   # column-major k x s
    Cm = torch.randn(batch, s, s, dtype=torch.complex128, device="cuda")
    args = (A.data_ptr(), B.data_ptr(), Cm.data_ptr(), s, s, k, batch)
    times = []
    for rep in range(reps + 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.gemm_device(*args)
        ctx.gemm_device(*args, alpha=-1.0, beta=1.0)
        e1.record(stream)
        torch.cuda.synchronize()
        if rep:
            times.append(e0.elapsed_time(e1))
    times.sort()
    return times[len(times) // 2]


def tune(path: str = TABLE_PATH) -> dict:
    import torch
    from . import lib as L
    lib = L.load()
    ctx = L.Context(0)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    table, rows = [], []
    try:
        for k in K_BUCKETS:
            for s in SIZE_BUCKETS:
                flops = 2 * 8.0 * s * s * k
                batch = int(max(1, min(4096, 4e9 / flops)))
                t = [_time_kernel(ctx, lib, torch, stream, c, s, k, batch) for c in (0, 1, 2, 3)]
                choice = min(range(4), key=lambda c: t[c])
                table.append(choice)
                rows.append({"k": k, "m=n": s, "batch": batch,
                             "dmma_tflops": flops * batch / (t[0] / 1e3) / 1e12,
                             "cuda_core_tflops": flops * batch / (t[1] / 1e3) / 1e12,
                             "dmma_tma_tflops": flops * batch / (t[2] / 1e3) / 1e12,
                             "dmma_32x64_tflops": flops * batch / (t[3] / 1e3) / 1e12,
                             "choice": ("dmma", "cuda_core", "dmma_tma", "dmma_32x64")[choice]})
    finally:
        lib.rcwa_set_gemm_table(None)
        ctx.close()
    out = {"device": torch.cuda.get_device_name(0), "date": time.strftime("%Y-%m-%d"),
           "k_buckets": K_LIMITS, "size_buckets": SIZE_LIMITS,
           "choice": table, "measurements": rows,
           "note": "choice[5 * k_bucket + size_bucket]: 0 = FP64 tensor-core (DMMA) kernel fed by cp.async, 1 = CUDA-core kernel, 2 = DMMA kernel fed by TMA, 3 = DMMA kernel (cp.async) on 32 x 64 tiles"}
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    return out


def load_table(path: str = TABLE_PATH):
    """The tuned choices (25 ints), or None when no table has been written."""
    if not os.path.exists(path):
        return None
    with open(path) as f:
        t = json.load(f)
    ch = t.get("choice")
    if not isinstance(ch, list) or len(ch) != 25 or any(c not in (-1, 0, 1, 2, 3) for c in ch):
        return None
    return ch


if __name__ == "__main__":
    import sys
    dst = sys.argv[1] if len(sys.argv) > 1 else TABLE_PATH
    res = tune(dst)
    for r in res["measurements"]:
        print(r)
    print("written", dst)
