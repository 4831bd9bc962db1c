"""The tcgen05 tensor-core GEMM core (mms_diag_gemm_bf16) against a plain
PyTorch FP32 reference of the same op on the same BF16 inputs.  BF16 products
are exact in FP32, so only the summation order differs: rel-L2 <= 1e-5."""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K,bn", [(128, 128, 64, 128), (200, 100, 1000, 64), (64, 48, 8, 64),
                                      (1000, 300, 512, 128), (333, 257, 136, 64)])
def test_gemm_matches_torch(cuda, lib, M, N, K, bn):
    import mmsb200
    torch = cuda
    g = torch.Generator(device="cuda").manual_seed(M * N + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    C = torch.full((M, N), float("nan"), device="cuda")
    st = lib.mms_diag_gemm_bf16(ctypes.c_void_p(A.data_ptr()), K, ctypes.c_void_p(B.data_ptr()), K,
                                ctypes.c_void_p(C.data_ptr()), N, M, N, K, 0, bn, None)
    assert st == mmsb200.MMS_OK, lib.mms_last_error()
    ref = A.float() @ B.float().T
    assert rel_l2(C.cpu().numpy(), ref.cpu().numpy()) < 1e-5
    # accumulate mode: C += A B^T
    st = lib.mms_diag_gemm_bf16(ctypes.c_void_p(A.data_ptr()), K, ctypes.c_void_p(B.data_ptr()), K,
                                ctypes.c_void_p(C.data_ptr()), N, M, N, K, 1, bn, None)
    assert st == mmsb200.MMS_OK, lib.mms_last_error()
    assert rel_l2(C.cpu().numpy(), 2 * ref.cpu().numpy()) < 1e-5


def test_gemm_rejects_bad_shapes(cuda, lib):
    import mmsb200
    torch = cuda
    A = torch.zeros(16, 12, device="cuda", dtype=torch.bfloat16)
    C = torch.zeros(16, 16, device="cuda")
    st = lib.mms_diag_gemm_bf16(ctypes.c_void_p(A.data_ptr()), 12, ctypes.c_void_p(A.data_ptr()), 12,
                                ctypes.c_void_p(C.data_ptr()), 16, 16, 16, 12, 0, 64, None)
    assert st == mmsb200.MMS_ERR_ARG
