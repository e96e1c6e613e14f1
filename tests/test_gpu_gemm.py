"""The tcgen05 BF16 GEMM of the coarse assignment against an FP32 product of the same
BF16 inputs (torch, plain fp32 matmul of the bf16-rounded operands)."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("rows,cols,d", [(128, 128, 64), (300, 700, 128), (257, 576, 384), (5, 9, 8),
                                         (1000, 64, 128), (200, 300, 96), (4096, 4608, 128)])
def test_bf16_gemm_matches_fp32_reference(cuda, rows, cols, d):
    import torch
    import hdgrid_b200 as hg
    g = torch.Generator(device="cpu").manual_seed(rows * 131 + cols)
    a = torch.randn(rows, d, generator=g).to(cuda).to(torch.bfloat16)
    b = torch.randn(cols, d, generator=g).to(cuda).to(torch.bfloat16)
    out = torch.full((rows, cols), float("nan"), device=cuda)
    hg.bf16_gemm(a, b, out)
    torch.cuda.synchronize()
    ref = a.float() @ b.float().t()
    assert not torch.isnan(out).any()
    # fp32 accumulation of exact bf16 products: differences come from summation order only
    tol = 1e-5 * (a.float().abs() @ b.float().abs().t()) + 1e-6
    assert torch.all((out - ref).abs() <= tol), float((out - ref).abs().max())


def test_bf16_gemm_into_a_column_slice(cuda):
    # the coarse stage writes the list block at column C of a [q x (C + L)] matrix: the GEMM
    # writes only its own columns, with the wide matrix's row stride
    import torch
    import hdgrid_b200 as hg
    g = torch.Generator(device="cpu").manual_seed(7)
    q, c, lists, d = 700, 64, 512, 128
    a = torch.randn(q, d, generator=g).to(cuda).to(torch.bfloat16)
    b = torch.randn(lists, d, generator=g).to(cuda).to(torch.bfloat16)
    wide = torch.full((q, c + lists), float("nan"), device=cuda)
    hg.bf16_gemm(a, b, wide[:, c:])
    torch.cuda.synchronize()
    ref = a.float() @ b.float().t()
    tol = 1e-5 * (a.float().abs() @ b.float().abs().t()) + 1e-6
    assert torch.isnan(wide[:, :c]).all()
    assert torch.all((wide[:, c:] - ref).abs() <= tol)
