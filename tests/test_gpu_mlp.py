"""Tensor-core kernels of the surrogate's MLP: operand encodings against host products."""

import ctypes

import numpy as np
import pytest

from grasph2_b200._abi import load_library

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("b_mn", [0, 1])
@pytest.mark.parametrize("a_mn", [0, 1])
@pytest.mark.parametrize("N,K", [(16, 16), (128, 32), (64, 128), (128, 128), (16, 128), (32, 64)])
def test_tc_gemm_check(N, K, a_mn, b_mn):
    import torch
    lib = load_library()
    g = torch.Generator().manual_seed(N * 1000 + K * 10 + 2 * a_mn + b_mn)
    A = torch.randn(128, K, generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, generator=g).to(torch.bfloat16)
    dA, dB = A.cuda(), B.cuda()
    D = torch.zeros(128, N, dtype=torch.float32, device="cuda")
    rc = lib.gsph_tc_gemm_check(ctypes.c_void_p(dA.data_ptr()), ctypes.c_void_p(dB.data_ptr()),
                                ctypes.c_void_p(D.data_ptr()), N, K, a_mn, b_mn)
    assert rc == 0, lib.gsph_last_error(None)
    want = A.double().numpy() @ B.double().numpy().T
    err = np.abs(D.cpu().numpy() - want).max() / np.abs(want).max()
    assert err < 1e-5, (N, K, a_mn, b_mn, err)
