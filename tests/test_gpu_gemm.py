"""BF16 tensor-core GEMM (lbm_gemm_bf16, tcgen05) against a PyTorch float32 product (needs a B200).

Two kernels run the product: below 1024 rows or 128 columns the TMA-fed one-tile-per-CTA
pipeline (k_gemm_tma: a 3-stage ring of tensor-map loads, one thread issuing the MMAs), above
them the persistent warp-specialised k_gemm_ws (accumulator transposed in TMEM, two accumulator
buffers, tiles walked by one CTA per SM).  The shapes cover both, with M, N and K tails (zero
fill of the boxes), several tiles per CTA, strided operands, every epilogue, and the warm
start's largest shape.

A and B are bf16; the reference multiplies their exact float32 values, so the only
difference is the order of the float32 accumulation: relative 1e-5 of the row's sum of
|a b| is the bar.
"""
import pytest

from water_flow_simulation_b200 import _native as nat

pytestmark = pytest.mark.gpu

SHAPES = [(128, 32, 64), (300, 100, 72), (77, 200, 8), (1000, 256, 1728), (129, 129, 136), (128, 64, 8192),
          (2048, 512, 576), (32768, 128, 3456), (5000, 200, 200), (1024, 128, 64), (33000, 384, 136)]


def _require_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


def gemm(A, B, epilogue=0, bias=None, D=None):
    torch = _require_gpu()
    M, K = A.shape
    N = B.shape[0]
    if D is None:
        D = torch.zeros(M, N, dtype=torch.float32 if epilogue < 2 else torch.bfloat16, device=A.device)
    err = torch.zeros(1, dtype=torch.int32, device=A.device)
    lib = nat.load()
    nat.check(lib.lbm_gemm_bf16(A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0), M, N, K, D.data_ptr(),
                                D.stride(0), epilogue, None if bias is None else bias.data_ptr(), err.data_ptr(),
                                torch.cuda.current_stream().cuda_stream), "lbm_gemm_bf16")
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return D


@pytest.mark.parametrize("shape", SHAPES)
def test_gemm_matches_float32_product(shape):
    torch = _require_gpu()
    M, N, K = shape
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    ref = A.float() @ B.float().T
    scale = A.float().abs() @ B.float().abs().T
    D = gemm(A, B)
    assert float(((D - ref).abs() / scale.clamp(min=1e-30)).max()) < 1e-5


def test_gemm_epilogues_and_strides():
    torch = _require_gpu()
    g = torch.Generator(device="cuda").manual_seed(3)
    Abig = torch.randn(200, 96, device="cuda", generator=g).to(torch.bfloat16)
    A = Abig[:, :88]                                   # lda = 96, K = 88
    B = torch.randn(70, 88, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(70, device="cuda", generator=g)
    ref = A.float() @ B.float().T
    D = gemm(A, B, epilogue=2, bias=bias)
    assert torch.allclose(D.float(), (ref + bias).to(torch.bfloat16).float(), rtol=1e-2, atol=1e-2)
    D = gemm(A, B, epilogue=3, bias=bias)
    assert torch.allclose(D.float(), torch.relu(ref + bias).to(torch.bfloat16).float(), rtol=1e-2, atol=1e-2)
    acc = torch.ones(200, 70, device="cuda")
    gemm(A, B, epilogue=1, D=acc)
    assert torch.allclose(acc, ref + 1, rtol=1e-5, atol=1e-4)


def test_gemm_argument_errors():
    import ctypes
    lib = nat.load()
    assert lib.lbm_gemm_bf16(None, 8, None, 8, 8, 8, 8, None, 8, 0, None, None, None) == -1
    buf = (ctypes.c_uint16 * 4096)()
    p = ctypes.addressof(buf)
    assert lib.lbm_gemm_bf16(p, 12, p, 12, 8, 8, 12, p, 8, 0, None, p, None) == -1
    assert b"multiples of 8" in lib.lbm_last_error()


@pytest.mark.parametrize("rows", [200, 3000])
def test_gemm_epilogues_and_strides_both_kernels(rows):
    """Every epilogue with lda > K and ldd > N, on the one-tile kernel (200 rows) and on the
    persistent kernel (3000 rows, N = 130: a second column block of 2 channels)."""
    torch = _require_gpu()
    g = torch.Generator(device="cuda").manual_seed(rows)
    A = torch.randn(rows, 96, device="cuda", generator=g).to(torch.bfloat16)[:, :88]
    B = torch.randn(130, 88, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(130, device="cuda", generator=g)
    ref = A.float() @ B.float().T
    scale = (A.float().abs() @ B.float().abs().T).clamp(min=1e-30)
    Df = torch.full((rows, 136), 7.0, device="cuda")
    D = gemm(A, B, epilogue=0, D=Df[:, :130])
    assert float(((D - ref).abs() / scale).max()) < 1e-5
    assert bool((Df[:, 130:] == 7.0).all())                   # nothing written past N
    D = gemm(A, B, epilogue=4, bias=bias, D=torch.empty(rows, 136, device="cuda")[:, :130])
    assert float(((D - ref - bias).abs() / (scale + bias.abs())).max()) < 1e-5
    for epi, fn in ((2, lambda x: x), (3, torch.relu)):
        Db = torch.empty(rows, 136, dtype=torch.bfloat16, device="cuda")[:, :130]
        D = gemm(A, B, epilogue=epi, bias=bias, D=Db)
        assert torch.equal(D, fn(D.float()).to(torch.bfloat16))
        assert torch.allclose(D.float(), fn(ref + bias).to(torch.bfloat16).float(), rtol=1e-2, atol=1e-2)
    acc = torch.ones(rows, 130, device="cuda")
    gemm(A, B, epilogue=1, D=acc)
    assert float(((acc - ref - 1).abs() / (scale + 1)).max()) < 1e-5
