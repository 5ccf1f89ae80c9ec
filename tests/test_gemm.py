"""BF16 tensor-core GEMM (tcgen05) of the warm-start surrogate against torch fp32.

The products of bf16 inputs are exact in fp32; only the accumulation order
differs from the fp32 reference, so the tolerance is a few fp32 ulps of the
row sums.
"""

from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


def _gemm(A, B, C, accumulate=0):
    import torch

    from curved_lbm import _native

    lib = _native.load()
    err = torch.zeros(1, dtype=torch.int32, device=A.device)
    M, K = A.shape
    N = B.shape[0]
    _native.check(lib.cvlbm_gemm_bf16(_native.ptr(A), _native.ptr(B), _native.ptr(C), M, N, K,
                                      A.stride(0), B.stride(0), C.stride(0), accumulate,
                                      _native.ptr(err),
                                      _native.stream_ptr(A.device)), "cvlbm_gemm_bf16")
    torch.cuda.synchronize()
    assert int(err.item()) == 0, "tensor-core MMAs did not complete"


@pytest.mark.parametrize("M,N,K", [(128, 64, 64), (384, 128, 320), (256, 192, 1024)])
def test_gemm_matches_fp32_reference(M, N, K):
    import torch

    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    C = torch.full((M, N), float("nan"), device="cuda")
    _gemm(A, B, C)
    ref = A.double() @ B.double().T
    scale = (A.double().abs() @ B.double().abs().T).max().item()
    assert torch.allclose(C.double(), ref, atol=1e-6 * scale, rtol=0), \
        float((C.double() - ref).abs().max())


def test_gemm_accumulates_and_respects_strides():
    import torch

    g = torch.Generator(device="cuda").manual_seed(3)
    A = torch.randn(128, 192, device="cuda", generator=g).to(torch.bfloat16)[:, :128]
    B = torch.randn(64, 128, device="cuda", generator=g).to(torch.bfloat16)
    C0 = torch.randn(128, 96, device="cuda", generator=g)
    C = C0.clone()
    _gemm(A, B, C[:, :64], accumulate=1)
    ref = C0[:, :64].double() + A.double() @ B.double().T
    assert torch.allclose(C[:, :64].double(), ref, atol=1e-4, rtol=1e-6)
    assert torch.equal(C[:, 64:], C0[:, 64:])
