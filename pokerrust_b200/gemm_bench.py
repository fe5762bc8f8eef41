"""Throughput of the library's tcgen05 BF16 GEMM against torch.matmul (cuBLAS), and of the
value network's training step with either GEMM form.

    python -m pokerrust_b200.gemm_bench

For each shape (M x N x K, operands K-major, f32 output) it times, with CUDA events over 20
launches after 3 warm-up launches: the per-tile form with 256- and 128-wide tiles
(pr_gemm_bf16_async), the persistent form (pr_gemm_bf16_persistent_async) and torch.matmul
of the same BF16 operands (BF16 output). Prints one JSON line per shape in TFLOP/s, then the
training step at batch 4096 in ms for the per-tile and the persistent GEMM forms.
"""
import json
import sys
import time

SHAPES = [(8192, 8192, 4096), (4096, 4096, 4096), (4096, 1024, 1024), (4096, 1024, 2816), (4096, 2816, 1024)]


def _time(fn, reps=20):
    import torch
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def gemm_rows():
    import torch
    from . import interface as P
    L = P.lib()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rows = []
    for (M, N, K) in SHAPES:
        g = torch.Generator(device="cuda").manual_seed(1)
        A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
        B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
        D = torch.zeros(M, N, device="cuda")
        flop = 2.0 * M * N * K
        row = {"shape": [M, N, K]}
        cands = [("tile256", lambda: L.pr_gemm_bf16_async(A.data_ptr(), B.data_ptr(), D.data_ptr(), M, N, K, 256,
                                                           err.data_ptr(), None)),
                 ("tile128", lambda: L.pr_gemm_bf16_async(A.data_ptr(), B.data_ptr(), D.data_ptr(), M, N, K, 128,
                                                           err.data_ptr(), None)),
                 ("persistent256", lambda: L.pr_gemm_bf16_persistent_async(A.data_ptr(), B.data_ptr(), D.data_ptr(),
                                                                            M, N, K, 256, err.data_ptr(), None)),
                 ("persistent128", lambda: L.pr_gemm_bf16_persistent_async(A.data_ptr(), B.data_ptr(), D.data_ptr(),
                                                                            M, N, K, 128, err.data_ptr(), None)),
                 ("torch", lambda: torch.matmul(A, B.t()))]
        for name, fn in cands:
            if name.endswith("256") and N % 256:
                continue
            ms = _time(fn)
            row[name + "_tflops"] = round(flop / ms / 1e9, 1)
        want = A.float() @ B.float().T
        L.pr_gemm_bf16_async(A.data_ptr(), B.data_ptr(), D.data_ptr(), M, N, K, 256 if N % 256 == 0 else 128,
                             err.data_ptr(), None)
        torch.cuda.synchronize()
        row["max_rel_err"] = float((D - want).abs().max() / want.abs().max())
        rows.append(row)
    if int(err.item()):
        raise P.PokerLibError(f"a GEMM wait timed out (bits {int(err.item())})")
    return rows


def train_step_ms():
    import torch
    from . import interface as P
    net = P.ValueNet(rows=4096, seed=11)
    g = torch.Generator(device="cuda").manual_seed(5)
    r = torch.rand((4096, 2, 1326), device="cuda", generator=g) / 600.0
    b = torch.randint(0, 1 << 20, (4096,), device="cuda", dtype=torch.int64, generator=g)
    s = torch.rand((4096, 2), device="cuda", generator=g)
    t = torch.randn((4096, 2652), device="cuda", generator=g) * 0.1
    out = {}
    for pers in (False, True):
        net.set_persistent(pers)
        for _ in range(3):
            net.train_step(r, b, s, t, 1e-4)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(20):
            net.train_step(r, b, s, t, 1e-4)
        out["persistent" if pers else "per_tile"] = (time.perf_counter() - t0) / 20 * 1e3
    net.close()
    return out


def main():
    for row in gemm_rows():
        print(json.dumps(row), flush=True)
    print(json.dumps({"train_step_ms": train_step_ms()}), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
