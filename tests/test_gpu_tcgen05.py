"""GPU tests of the hand-written tcgen05 GEMM (TMA-fed shared-memory ring, tcgen05.mma into
TMEM, TMEM loads in the epilogue) against torch's matmul on the same 16-bit operands.
Tolerance: FP32 accumulation in a different order, |diff| <= 1e-3 * sqrt(K) * max|C|."""
import math

import pytest

pytestmark = pytest.mark.gpu


def _run(pkg, ctx, M, N, K, dtype):
    import torch
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    tdt = torch.bfloat16 if dtype == 0 else torch.float16
    A = torch.randn(M, K, device="cuda", generator=g).to(tdt).contiguous()
    B = torch.randn(N, K, device="cuda", generator=g).to(tdt).contiguous()
    C = torch.full((M, N), float("nan"), device="cuda", dtype=torch.float32)
    torch.cuda.synchronize()
    pkg._lib.check(ctx.lib.scrna_debug_tc_gemm(ctx.h, A.data_ptr(), B.data_ptr(), C.data_ptr(), M, N, K, dtype))
    ref = A.float() @ B.float().T
    err = (C - ref).abs().max().item()
    return err, ref.abs().max().item()


@pytest.mark.parametrize("M,N,K,dtype", [(128, 256, 64, 0), (256, 512, 128, 0), (300, 600, 192, 0),
                                         (1000, 2000, 2112, 0), (257, 130, 128, 1)])
def test_tc_gemm_matches_torch(pkg, ctx, M, N, K, dtype):
    err, scale = _run(pkg, ctx, M, N, K, dtype)
    assert err <= 1e-3 * math.sqrt(K) * max(scale, 1.0), (err, scale)
