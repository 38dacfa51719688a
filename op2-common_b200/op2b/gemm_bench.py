"""Time op2b_gemm_bf16 on the learned warm start's edge-MLP shapes.

    python -m op2b.gemm_bench [--rows 635000] [--reps 20]

M = rows (messages of 8 copies of the 200x100 cell graph by default), N = 128,
K and epilogue as the network's products use them.  Each product runs on
engine 2 with the persistent kernel (16 epilogue warps storing whole rows
through shared memory, and each lane its own row; 8 epilogue warps), engine 2
one CTA per tile, and engine 0; one JSON line per run with the mean CUDA-event
time of `reps` launches after 3 untimed, and GB/s over the bytes of A, B and
the outputs (C, and Z for bias+SiLU).
"""
import argparse
import json

import torch

from . import gnn as G
from . import lib as L


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rows", type=int, default=635000)
    ap.add_argument("--reps", type=int, default=20)
    a = ap.parse_args()
    L.load()
    L.op_init()
    M, N = a.rows, 128
    s = torch.cuda.current_stream().cuda_stream
    cases = ((384, G.EPI_BIAS_SILU_BF16), (128, G.EPI_BIAS_SILU_BF16), (128, G.EPI_BIAS_BF16),
             (8, G.EPI_BIAS_SILU_BF16), (384, G.EPI_STORE_F32))
    for K, epi in cases:
        A = (torch.randn(M, K, device="cuda") * 0.2).to(torch.bfloat16)
        B = (torch.randn(N, K, device="cuda") * 0.2).to(torch.bfloat16)
        bias = torch.randn(N, device="cuda")
        f32 = epi == G.EPI_STORE_F32
        C = torch.zeros(M, N, device="cuda", dtype=torch.float32 if f32 else torch.bfloat16)
        Z = None if f32 or epi != G.EPI_BIAS_SILU_BF16 else torch.zeros_like(C)
        out_bytes = M * N * (4 if f32 else 2) * (2 if Z is not None else 1)
        for engine, pers, rows in ((2, 2, 1), (2, 2, 0), (2, 1, 0), (2, 0, 0), (0, 0, 0)):
            L.set_option("gemm_persistent", pers)
            L.set_option("gemm_rows", rows)

            def run():
                rc = G._lib().op2b_gemm_bf16(M, N, K, A.data_ptr(), K, 1, B.data_ptr(), K, 1,
                                             C.data_ptr(), N, epi, bias.data_ptr(),
                                             None if Z is None else Z.data_ptr(), None, 0, 1,
                                             engine, s)
                if rc != 0:
                    raise RuntimeError(L.last_error())

            for _ in range(3):
                run()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(a.reps):
                run()
            e1.record()
            torch.cuda.synchronize()
            us = e0.elapsed_time(e1) * 1e3 / a.reps
            byts = M * K * 2 + N * K * 2 + out_bytes
            print(json.dumps({"M": M, "N": N, "K": K, "epi": epi, "engine": engine,
                              "gemm_persistent": pers, "gemm_rows": rows, "us": round(us, 1),
                              "gbs": round(byts / us / 1e3)}), flush=True)
    L.set_option("gemm_persistent", 2)
    L.set_option("gemm_rows", 1)
    torch.cuda.synchronize()
    if G._lib().op2b_gemm_error(1) != 0:
        raise RuntimeError("a GEMM wait timed out")
    L.op_exit()


if __name__ == "__main__":
    main()
