"""Numerics of the tcgen05 GEMM (TMA + TMEM, bf16 / tf32 operands, fp32 accumulation)
against a plain PyTorch reference of the same op on the same (rounded) inputs.
Tolerance: 2e-5 relative to max|C| (fp32 accumulation over K <= 1024)."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def run(M, N, K, batch, tf32, bn, seed=0, mode=0):
    from miniafqmc_b200.afqmc import load_library
    lib = load_library()
    g = torch.Generator().manual_seed(seed)
    A = torch.randn(batch, M, K, generator=g)
    B = torch.randn(batch, N, K, generator=g)
    if tf32:   # make the inputs exactly tf32-representable (drop 13 low mantissa bits)
        A = (A.view(torch.int32) & ~0x1FFF).view(torch.float32)
        B = (B.view(torch.int32) & ~0x1FFF).view(torch.float32)
    elif mode < 5:   # split modes keep full fp32 inputs (hi + lo parts)
        A = A.bfloat16().float()
        B = B.bfloat16().float()
    C = np.zeros((batch, M, N), np.float32)
    err = ctypes.c_int(-1)
    An, Bn = A.numpy().copy(), B.numpy().copy()
    st = lib.afq_selftest_tc_gemm(M, N, K, batch, int(tf32), bn, mode,
                                  ctypes.c_void_p(An.ctypes.data),
                                  ctypes.c_void_p(Bn.ctypes.data), ctypes.c_void_p(C.ctypes.data),
                                  ctypes.byref(err))
    assert st == 0 and err.value == 0, (st, err.value)
    ref = torch.bmm(A.double(), B.double().transpose(1, 2)).numpy()
    return C, ref


@pytest.mark.parametrize("tf32", [False, True])
@pytest.mark.parametrize("shape", [(128, 128, 64, 1, 128), (300, 200, 768, 3, 128),
                                   (256, 192, 1024, 2, 192), (100, 64, 72, 1, 64),
                                   (384, 192, 768, 4, 192), (256, 512, 512, 2, 256)])
# per-tile, persistent x1 / x2 epilogue groups; per-tile and persistent with 64-byte K slabs
@pytest.mark.parametrize("mode", [0, 1, 2, 3, 4])
def test_tc_gemm_matches_reference(shape, tf32, mode):
    M, N, K, batch, bn = shape
    C, ref = run(M, N, K, batch, tf32, bn, mode=mode)
    scale = np.abs(ref).max()
    assert np.max(np.abs(C - ref)) / scale < 2e-5


@pytest.mark.parametrize("shape", [(128, 256, 512, 1, 256), (300, 512, 768, 2, 256),
                                   (256, 192, 1024, 2, 192), (256, 128, 256, 1, 128)])
def test_tc_gemm_split_matches_reference(shape):
    """Split bf16 (hi*hi + hi*lo + lo*hi of fp32 inputs) on the per-tile (modes 5, 6) and
    persistent (7, 8) kernels with 128- and 64-byte K slabs: within 1e-4 of the FP64
    product (bf16x3 carries about 16 bits per operand), and each 64-byte-slab result
    within 1e-6 of the 128-byte one (the same products in another fp32 summation order)."""
    M, N, K, batch, bn = shape
    out = {}
    for mode in (5, 6, 7, 8):
        C, ref = run(M, N, K, batch, False, bn, mode=mode)
        scale = np.abs(ref).max()
        out[mode] = C
        assert np.max(np.abs(C - ref)) / scale < 1e-4, mode
    assert np.max(np.abs(out[6] - out[5])) / scale < 1e-6
    assert np.max(np.abs(out[8] - out[7])) / scale < 1e-6
