"""BF16 tensor-core GEMM (tcgen05) of the warm-start surrogate against fp64.

The products of bf16 inputs are exact in fp32; only the accumulation order
differs from the reference, so the tolerance is a few fp32 ulps of the row
sums.  Both operand loaders run every case: TMA tensor copies into the
128-byte-swizzled layout (the default) and thread loads into the
no-swizzle layout (CVLBM_GEMM_LOADER=threads).
"""

from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["tma", "threads"], autouse=True)
def loader(request, monkeypatch):
    monkeypatch.setenv("CVLBM_GEMM_LOADER", request.param)
    return request.param


def _gemm(A, B, C, accumulate=0, split=True):
    import torch

    from curved_lbm import _native

    lib = _native.load()
    err = torch.zeros(1, dtype=torch.int32, device=A.device)
    M, K = A.shape
    N = B.shape[0]
    ws = torch.empty(int(lib.cvlbm_gemm_bf16_workspace(M, N, K)) // 4 if split else 1,
                     dtype=torch.float32, device=A.device)
    _native.check(lib.cvlbm_gemm_bf16(_native.ptr(A), _native.ptr(B), _native.ptr(C), M, N, K,
                                      A.stride(0), B.stride(0), C.stride(0), accumulate,
                                      _native.ptr(err), _native.ptr(ws) if split else 0,
                                      ws.numel() * 4 if split else 0,
                                      _native.stream_ptr(A.device)), "cvlbm_gemm_bf16")
    torch.cuda.synchronize()
    assert int(err.item()) == 0, "tensor-core MMAs did not complete"


@pytest.mark.parametrize("M,N,K,split", [(128, 64, 64, True), (384, 128, 320, True),
                                         (256, 192, 1024, True), (128, 256, 8192, True),
                                         (128, 256, 8192, False), (256, 128, 4096, True)])
def test_gemm_matches_fp32_reference(M, N, K, split):
    import torch

    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    C = torch.full((M, N), float("nan"), device="cuda")
    _gemm(A, B, C, split=split)
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
    A2 = torch.randn(128, 4096, device="cuda", generator=g).to(torch.bfloat16)
    B2 = torch.randn(128, 4096, device="cuda", generator=g).to(torch.bfloat16)
    C3 = torch.randn(128, 128, device="cuda", generator=g)
    C3c = C3.clone()
    _gemm(A2, B2, C3, accumulate=1)  # split K with accumulate
    ref3 = C3c.double() + A2.double() @ B2.double().T
    scale3 = (A2.double().abs() @ B2.double().abs().T).max().item()
    assert torch.allclose(C3.double(), ref3, atol=1e-6 * scale3 + 1e-5, rtol=0)
    ref = C0[:, :64].double() + A.double() @ B.double().T
    assert torch.allclose(C[:, :64].double(), ref, atol=1e-4, rtol=1e-6)
    assert torch.equal(C[:, 64:], C0[:, 64:])
