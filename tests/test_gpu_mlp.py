"""The surrogate network's tensor-core kernels (include/sph_mlp.h) against a plain PyTorch
FP32 reference on the same bf16 operands."""
import ctypes

import numpy as np
import pytest
import torch

import sph_b200

pytestmark = pytest.mark.gpu

PF = ctypes.POINTER(ctypes.c_float)


def tc_gemm(A, B, heads, M, N, K):
    L = sph_b200.lib()
    L.sph_tc_gemm.argtypes = [ctypes.c_void_p, ctypes.c_void_p, PF, ctypes.c_int, ctypes.c_int,
                              ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    C = torch.full((heads, M, N), float("nan"), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    st = L.sph_tc_gemm(A.data_ptr(), B.data_ptr(), ctypes.cast(C.data_ptr(), PF), M, N, K,
                       heads, None)
    assert st == 0, sph_b200.STATUS.get(st, st)
    return C


@pytest.mark.parametrize("M,N,K,heads", [(128, 256, 64, 1), (256, 256, 256, 5),
                                         (128, 16, 128, 1), (256, 128, 1024, 2),
                                         (1024, 256, 256, 5)])
def test_tc_gemm_matches_fp32_reference(M, N, K, heads):
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K + heads)
    A = torch.randn(heads, M, K, generator=g, device="cuda").to(torch.bfloat16)
    B = torch.randn(heads, N, K, generator=g, device="cuda").to(torch.bfloat16)
    C = tc_gemm(A, B, heads, M, N, K)
    ref = torch.matmul(A.double(), B.double().transpose(1, 2))
    err = (C.double() - ref).abs().max().item()
    scale = ref.abs().max().item()
    # bf16 x bf16 products are exact in FP32; only the summation order differs
    assert err <= 1e-5 * scale, (err, scale)
