"""The tcgen05 bf16 GEMM (kf_gemm_bf16) against a plain PyTorch fp32 matmul
of the same bf16 operands."""

import ctypes as C

import numpy as np
import pytest

from kinectfusion_b200 import abi

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,n,k", [(128, 16, 64), (256, 32, 128), (300, 64, 96), (128, 200, 64), (1200, 32, 32),
                                   (64, 256, 1280), (32, 24, 8192), (256, 288, 4800),
                                   (38016, 300, 192)])
@pytest.mark.parametrize("epilogue", [False, True])
def test_gemm_matches_fp32_reference(m, n, k, epilogue):
    import torch
    g = torch.Generator(device="cpu").manual_seed(m * 7 + n * 3 + k)
    a = torch.randn(m, k, generator=g).to(torch.bfloat16).cuda()
    b = torch.randn(n, k, generator=g).to(torch.bfloat16).cuda()
    bias = torch.randn(n, generator=g).cuda() if epilogue else None
    c = torch.full((m, n), float("nan"), device="cuda")
    torch.cuda.synchronize()
    abi.check(abi.load().kf_gemm_bf16(C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()), C.c_void_p(c.data_ptr()),
                                      m, n, k, C.c_void_p(bias.data_ptr()) if epilogue else None,
                                      1 if epilogue else 0, None))
    ref = a.float() @ b.float().T
    if epilogue:
        ref = torch.relu(ref + bias)
    scale = float(ref.abs().max()) + 1.0
    # both sum exact bf16 products in FP32, in different orders
    assert float((c - ref).abs().max()) <= 1e-5 * scale * k ** 0.5
