"""Learned initialiser: the tensor-core BF16 GEMM its layers run on, against an FP64
product of the same BF16 operands."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gemm(A, B):
    import torch
    from sitk_b200 import _lib
    from sitk_b200.metric import default_context
    L = _lib.load()
    L.mi_gemm_bf16_tn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                  ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
    L.mi_gemm_bf16_tn.restype = ctypes.c_int
    M, K = A.shape
    N = B.shape[0]
    C = torch.zeros((M, N), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    ctx = default_context()
    _lib.check(L.mi_gemm_bf16_tn(ctx.handle, M, N, K, A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0),
                                 C.data_ptr(), C.stride(0)), ctx.handle)
    return C


@pytest.mark.parametrize("M,N,K", [(128, 16, 64), (300, 48, 200), (1000, 128, 1000), (64, 12, 256),
                                   (257, 256, 130), (130, 40, 54)])
def test_tensor_core_gemm_matches_fp64(M, N, K):
    import torch
    g = torch.Generator(device="cpu").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn((M, K), generator=g).to(torch.bfloat16).cuda()
    B = torch.randn((N, K), generator=g).to(torch.bfloat16).cuda()
    C = _gemm(A, B).cpu().double().numpy()
    ref = A.cpu().double().numpy() @ B.cpu().double().numpy().T
    # FP32 accumulation of K exact BF16 products
    tol = 1e-5 * np.sqrt(K) * (np.abs(A.cpu().double().numpy()) @ np.abs(B.cpu().double().numpy()).T) + 1e-6
    assert np.all(np.abs(C - ref) <= tol), np.max(np.abs(C - ref))


def test_tensor_core_gemm_strided_operands():
    import torch
    g = torch.Generator(device="cpu").manual_seed(5)
    A = torch.randn((200, 96), generator=g).to(torch.bfloat16).cuda()[:, :80]   # lda 96
    B = torch.randn((24, 88), generator=g).to(torch.bfloat16).cuda()[:, :80]    # ldb 88
    C = _gemm(A, B).cpu().double().numpy()
    ref = A.cpu().double().numpy() @ B.cpu().double().numpy().T
    assert np.max(np.abs(C - ref)) < 1e-3
