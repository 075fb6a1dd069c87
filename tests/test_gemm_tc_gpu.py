"""GPU numerics of the surrogate network's BF16 GEMM paths through the C ABI
(rbc_gemm_bf16): the tcgen05 kernel (5th-generation tensor cores, TMEM accumulator) and the
mma.sync tiles against a float64 product of the same BF16 values. FP32 accumulation over
K <= 256 terms: bar 1e-5 of the largest |C| (both paths), and the two paths within 1e-5 of
each other. Shapes cover partial row tiles, N not a multiple of 32, K not a multiple of 16
and the largest N (256)."""
import ctypes

import numpy as np
import pytest

import sdc_b200

pytestmark = pytest.mark.gpu

SHAPES = [(256, 32, 32), (300, 48, 48), (1024, 128, 256), (128, 256, 64), (520, 40, 24), (4096, 16, 8),
          (640, 96, 200)]


def run(A, B, path):
    import torch
    M, K = A.shape
    N = B.shape[1]
    C = torch.zeros((M, N), dtype=torch.float32, device="cuda")
    st = sdc_b200.lib().rbc_gemm_bf16(0, ctypes.c_void_p(A.data_ptr()), ctypes.c_void_p(B.data_ptr()),
                                      ctypes.c_void_p(C.data_ptr()), M, N, K, path, None)
    assert st == 0, st
    return C.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("shape", SHAPES)
def test_gemm_paths_match_float64_product(shape):
    import torch
    M, N, K = shape
    g = torch.Generator().manual_seed(M * 7 + N * 3 + K)
    A = torch.randn((M, K), generator=g).to(torch.bfloat16).cuda()
    B = torch.randn((K, N), generator=g).to(torch.bfloat16).cuda()
    ref = A.cpu().double().numpy() @ B.cpu().double().numpy()
    scale = np.abs(ref).max()
    tc = run(A, B, 0)
    ms = run(A, B, 1)
    assert np.abs(tc - ref).max() <= 1e-5 * scale, np.abs(tc - ref).max() / scale
    assert np.abs(ms - ref).max() <= 1e-5 * scale, np.abs(ms - ref).max() / scale
    assert np.abs(tc - ms).max() <= 1e-5 * scale


def test_gemm_tc_consecutive_calls_and_bad_arguments():
    import torch
    A = torch.randn((384, 64)).to(torch.bfloat16).cuda()
    B = torch.randn((64, 64)).to(torch.bfloat16).cuda()
    ref = A.cpu().double().numpy() @ B.cpu().double().numpy()
    for _ in range(3):
        assert np.abs(run(A, B, 0) - ref).max() <= 1e-5 * np.abs(ref).max()
    C = torch.zeros((384, 64), dtype=torch.float32, device="cuda")
    bad = sdc_b200.lib().rbc_gemm_bf16(0, ctypes.c_void_p(A.data_ptr()), ctypes.c_void_p(B.data_ptr()),
                                       ctypes.c_void_p(C.data_ptr()), 384, 64, 64, 2, None)
    assert bad == 1
    # N above the tensor-core limit
    B2 = torch.randn((64, 272)).to(torch.bfloat16).cuda()
    C2 = torch.zeros((384, 272), dtype=torch.float32, device="cuda")
    bad2 = sdc_b200.lib().rbc_gemm_bf16(0, ctypes.c_void_p(A.data_ptr()), ctypes.c_void_p(B2.data_ptr()),
                                        ctypes.c_void_p(C2.data_ptr()), 384, 272, 64, 0, None)
    assert bad2 == 1
