"""The tcgen05 dense layer (csrc/pgm_tc.cuh) against an FP32 matrix product of the same BF16
operands (GPU): C = act(A W^T + bias) for every compiled (K, N), row counts that are and are not
multiples of the 128-row tile, FP32 and BF16 outputs, with and without SiLU."""

import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

SHAPES = [(16, 64), (64, 64), (64, 128), (80, 64), (64, 32), (128, 16)]


def _p(t):
    return C.c_void_p(t.data_ptr())


@pytest.mark.parametrize("K,N", SHAPES)
@pytest.mark.parametrize("M", [1, 128, 300, 4099])
def test_tc_gemm_matches_fp32_product(K, N, M):
    from pgm_jax_b200 import _lib

    lib = _lib.load()
    dev = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(K * 1000 + N + M)
    lda = K + 8  # rows padded past K: only the first K are read
    A = torch.randn((M, lda), generator=g).to(torch.bfloat16).to(dev)
    W = (torch.randn((N, K), generator=g) / K**0.5).to(torch.bfloat16).to(dev)
    bias = torch.randn(N, generator=g).to(dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    ref = A[:, :K].float() @ W.float().T + bias
    for act in (0, 1):
        want = ref if act == 0 else ref * torch.sigmoid(ref)
        for f32 in (1, 0):
            out = torch.full((M, N), float("nan"), dtype=torch.float32 if f32 else torch.bfloat16, device=dev)
            rc = lib.pgm_tc_gemm(None, K, N, act, f32, _p(A), lda, M, _p(W), _p(bias), _p(out), N, _p(err))
            assert rc == 0, lib.pgm_tc_last_error().decode()
            torch.cuda.synchronize()
            got = out.float()
            tol = 1e-5 if f32 else 8e-3  # FP32 accumulation order; BF16 rounding of the output
            assert torch.isfinite(got).all()
            assert (got - want).abs().max().item() <= tol * max(1.0, want.abs().max().item()), (act, f32)
    assert int(err.item()) == 0


def test_tc_gemm_rejects_an_uncompiled_shape():
    from pgm_jax_b200 import _lib

    lib = _lib.load()
    dev = torch.device("cuda", 0)
    A = torch.zeros((8, 48), dtype=torch.bfloat16, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    rc = lib.pgm_tc_gemm(None, 48, 48, 0, 1, _p(A), 48, 8, _p(A), None, _p(A), 48, _p(err))
    assert rc == 4 and b"not compiled" in lib.pgm_tc_last_error()
