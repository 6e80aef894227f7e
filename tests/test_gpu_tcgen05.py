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


def test_pipeline_wait_timeout_returns_error_and_context_recovers(pkg, ctx):
    """Failure detection without a fault: the TMA producer withholds its first load in every
    CTA (no load or MMA is ever in flight), so the MMA issuer's and the epilogue's bounded
    waits (2 s) run out.  The call returns SCRNA_ETIMEOUT after the kernel left through its
    normal exit, which releases TMEM; the next GEMM on the same context (which allocates TMEM
    on the same SMs again) and a CLE run both succeed."""
    import time
    import torch
    M, N, K = 256, 512, 128
    A = torch.randn(M, K, device="cuda").to(torch.bfloat16).contiguous()
    B = torch.randn(N, K, device="cuda").to(torch.bfloat16).contiguous()
    C = torch.zeros((M, N), device="cuda", dtype=torch.float32)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rc = ctx.lib.scrna_debug_tc_gemm_withhold(ctx.h, A.data_ptr(), B.data_ptr(), C.data_ptr(), M, N, K, 0, 0)
    el = time.perf_counter() - t0
    assert rc == -4  # SCRNA_ETIMEOUT
    assert b"timed out" in ctx.lib.scrna_last_error()
    assert 1.5 < el < 60.0
    err, scale = _run(pkg, ctx, M, N, K, 0)
    assert err <= 1e-3 * math.sqrt(K) * max(scale, 1.0)
    net = pkg.sample_network(6, seed=3)
    out = pkg.simulate(net, pkg.CLE(0.01), pkg.WORKLOAD_KINETICS, cell_num=64, T=0.5, ctx=ctx)
    assert out.shape == (64, 6)
