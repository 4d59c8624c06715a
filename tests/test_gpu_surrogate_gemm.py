"""The surrogate's tensor-core GEMM (TMA + tcgen05.mma + TMEM, BF16 in, FP32
accumulate) against a plain PyTorch FP32 matmul of the same BF16 operands.

Tolerance: both sides accumulate the same BF16 products in FP32, in different
orders, so |C - C_ref| <= 1e-4 * sum_k |a_ik b_jk| + 1e-6."""

import ctypes as ct

import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,n,k,splits", [
    (128, 128, 64, 1),        # one tile, one k-block
    (1000, 256, 256, 1),      # ragged M (TMA zero-fill), 2 N-tiles, 4 k-blocks (ring wraps)
    (256, 256, 8192, 64),     # split-K slabs, as the weight-gradient GEMMs run
    (384, 64, 1024, 8),       # 64-wide N tile
    (8192, 128, 640, 1),      # many M-tiles, ring wraps 2.5 times
])
def test_umma_gemm_matches_torch_fp32(qk, m, n, k, splits):
    g = torch.Generator(device="cuda").manual_seed(m * 7 + n * 3 + k)
    a = torch.randn(m, k, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(n, k, device="cuda", generator=g).to(torch.bfloat16)
    c = torch.full((splits, m, n), float("nan"), device="cuda", dtype=torch.float32)
    rc = qk._lib.qk_sur_gemm_bf16(ct.c_void_p(a.data_ptr()), ct.c_void_p(b.data_ptr()),
                                  ct.c_void_p(c.data_ptr()), m, n, k, splits, None)
    assert rc == 0, qk.get_last_error()
    torch.cuda.synchronize()
    got = c.sum(0)
    ref = a.float() @ b.float().T
    bound = (a.float().abs() @ b.float().abs().T) * 1e-4 + 1e-6
    err = (got - ref).abs()
    assert torch.isfinite(got).all()
    assert bool((err <= bound).all()), float((err / bound).max())


def test_umma_gemm_rejects_bad_shapes(qk):
    a = torch.zeros(128, 64, device="cuda", dtype=torch.bfloat16)
    c = torch.zeros(128, 128, device="cuda")
    p = ct.c_void_p(a.data_ptr())
    assert qk._lib.qk_sur_gemm_bf16(p, p, ct.c_void_p(c.data_ptr()), 128, 128, 60, 1, None) == -2
    assert qk._lib.qk_sur_gemm_bf16(p, p, ct.c_void_p(c.data_ptr()), 128, 100, 64, 1, None) == -2
    assert qk._lib.qk_sur_gemm_bf16(None, p, ct.c_void_p(c.data_ptr()), 128, 128, 64, 1, None) == -1
