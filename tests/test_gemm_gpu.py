"""The tcgen05 BF16 GEMM (pr_gemm_bf16) against an FP32 product of the same BF16 operands.

Products of two bf16 values are exact in f32, so the only difference is the order of the
f32 sums: 1e-5 of the output's scale."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K,bn", [(128, 128, 64, 128), (128, 256, 64, 256), (256, 512, 320, 256),
                                      (384, 384, 1024, 128), (1024, 1024, 2752, 256)])
def test_gemm_matches_fp32(M, N, K, bn):
    import torch
    import pokerrust_b200 as P
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    D = torch.full((M, N), float("nan"), device="cuda", dtype=torch.float32)
    torch.cuda.synchronize()
    st = P.lib().pr_gemm_bf16(A.data_ptr(), B.data_ptr(), D.data_ptr(), M, N, K, bn, None)
    assert st == 0
    want = A.float() @ B.float().T
    err = (D - want).abs().max().item()
    assert err <= 1e-5 * want.abs().max().item(), err


@pytest.mark.parametrize("a_mn,b_mn", [(0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("M,N,K,bn", [(128, 256, 64, 256), (256, 512, 320, 256), (1024, 2816, 4096, 256),
                                      (384, 384, 1024, 128)])
def test_gemm_mn_major_operands(M, N, K, bn, a_mn, b_mn):
    """Operands stored MN-major ([K][M] for A, [K][N] for B), read by the tensor cores without
    a transpose in memory: the same product."""
    import torch
    import pokerrust_b200 as P
    g = torch.Generator(device="cuda").manual_seed(M * 5 + N + K + 7 * a_mn + 3 * b_mn)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    As = A.T.contiguous() if a_mn else A
    Bs = B.T.contiguous() if b_mn else B
    D = torch.full((M, N), float("nan"), device="cuda", dtype=torch.float32)
    torch.cuda.synchronize()
    st = P.lib().pr_gemm_bf16_major(As.data_ptr(), Bs.data_ptr(), D.data_ptr(), M, N, K, bn, a_mn, b_mn, None)
    assert st == 0
    want = A.float() @ B.float().T
    err = (D - want).abs().max().item()
    assert err <= 1e-5 * want.abs().max().item(), err


def test_gemm_rejects_bad_shapes():
    import torch
    import pokerrust_b200 as P
    A = torch.zeros(100, 64, device="cuda", dtype=torch.bfloat16)
    B = torch.zeros(128, 64, device="cuda", dtype=torch.bfloat16)
    D = torch.zeros(100, 128, device="cuda")
    assert P.lib().pr_gemm_bf16(A.data_ptr(), B.data_ptr(), D.data_ptr(), 100, 128, 64, 128, None) == 2


def test_gemm_bounded_wait_runs_out_and_recovers():
    """The GEMM's mbarrier waits are bounded: with one tile load of the first CTA armed but
    never issued (test hook) and a 20 ms limit, the MMA warp's wait for it runs out, the
    kernel sets its error bit and returns, and the context stays usable: the next product on
    the same buffers is correct. The failure is made by withholding work, not by a fault."""
    import torch
    import pokerrust_b200 as P
    M, N, K = 256, 256, 512  # 8 k tiles, more than the 4-stage ring
    g = torch.Generator(device="cuda").manual_seed(3)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    D = torch.zeros((M, N), device="cuda", dtype=torch.float32)
    torch.cuda.synchronize()
    L = P.lib()
    # without a withheld load every wait is met
    assert L.pr_gemm_bf16_wait_test(A.data_ptr(), B.data_ptr(), D.data_ptr(), M, N, K, 128, 20_000_000, -1, None) == 0
    want = A.float() @ B.float().T
    assert (D - want).abs().max().item() <= 1e-5 * want.abs().max().item()
    # the withheld load: the MMA wait (bit 2) and the producer's wait for the stage (bit 1) run out
    bits = L.pr_gemm_bf16_wait_test(A.data_ptr(), B.data_ptr(), D.data_ptr(), M, N, K, 128, 20_000_000, 0, None)
    assert bits & 2 and bits & 1, bits
    torch.cuda.synchronize()  # the context is still usable
    # bad shapes for the hook are refused before any launch
    assert L.pr_gemm_bf16_wait_test(A.data_ptr(), B.data_ptr(), D.data_ptr(), M, N, 256, 128, 20_000_000, 0, None) == -2
    D.zero_()
    assert L.pr_gemm_bf16(A.data_ptr(), B.data_ptr(), D.data_ptr(), M, N, K, 128, None) == 0
    assert (D - want).abs().max().item() <= 1e-5 * want.abs().max().item()


@pytest.mark.parametrize("M,N,K,bn,a_mn,b_mn,splits", [
    (128, 128, 64, 128, 0, 0, 1),          # one tile
    (4096, 1024, 1024, 128, 0, 1, 1),      # 256 tiles: more than one per SM, both accumulators in turn
    (4096, 1024, 2816, 256, 0, 0, 1),      # the network's first layer
    (1024, 1024, 4096, 256, 1, 1, 4),      # split-K weight gradient, both operands MN-major
    (2048, 2048, 512, 256, 1, 0, 1),
])
def test_persistent_gemm_matches_fp32(M, N, K, bn, a_mn, b_mn, splits):
    """The persistent form (one CTA per SM over all tiles, epilogues overlapping the next
    tile's main loop through a double-buffered accumulator): the sum of its split-K parts is
    the FP32 product of the same BF16 operands to 1e-5 of the output's scale."""
    import torch
    import pokerrust_b200 as P
    g = torch.Generator(device="cuda").manual_seed(M + 3 * N + 7 * K + splits)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    As = A.T.contiguous() if a_mn else A
    Bs = B.T.contiguous() if b_mn else B
    D = torch.full((splits, M, N), float("nan"), device="cuda", dtype=torch.float32)
    torch.cuda.synchronize()
    st = P.lib().pr_gemm_bf16_persistent(As.data_ptr(), Bs.data_ptr(), D.data_ptr(), M, N, K, bn, a_mn, b_mn,
                                         splits, None)
    assert st == 0
    want = A.float() @ B.float().T
    err = (D.sum(0) - want).abs().max().item()
    assert err <= 1e-5 * want.abs().max().item(), err
