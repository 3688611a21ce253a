"""tcgen05 split-BF16 GEMM against an FP64 torch reference (GPU).

Tolerances: one bf16 piece per operand reproduces the fp32-accumulated
product of the bf16-rounded inputs (rel 1e-5); BF16x3 (two pieces, three
products) is within 3e-5 relative of the FP64 product; three pieces with six
products within 1e-5 (the FP32 accumulator is the floor; it grows with K).
"""

import pytest
import torch

from ad_afqmc_b200 import _lib

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float((a.double() - b).norm() / b.norm())


@pytest.mark.parametrize("M,N,K,batch", [(128, 128, 64, 1), (300, 200, 130, 3), (77, 45, 520, 2),
                                          (1024, 384, 1000, 1)])
def test_split_gemm_accuracy(M, N, K, batch):
    g = torch.Generator(device="cuda").manual_seed(M * N + K)
    Kp = (K + 7) // 8 * 8  # row strides must be multiples of 8 elements
    Ap = torch.zeros(batch, M, Kp, dtype=torch.float64, device="cuda")
    Bp = torch.zeros(batch, N, Kp, dtype=torch.float64, device="cuda")
    Ap[..., :K] = torch.randn(batch, M, K, dtype=torch.float64, device="cuda", generator=g)
    Bp[..., :K] = torch.randn(batch, N, K, dtype=torch.float64, device="cuda", generator=g)
    A, B = Ap[..., :K], Bp[..., :K]
    ref = A @ B.transpose(1, 2)

    def split(x, n):
        return [p[..., :K] for p in _lib.split_bf16(x, n)]

    a1 = split(Ap, 1)
    b1 = split(Bp, 1)
    c1 = _lib.gemm_split_bf16(a1, b1, ((0, 0),))
    ref1 = a1[0].double() @ b1[0].double().transpose(1, 2)
    assert _rel(c1, ref1) < 1e-5
    a2, b2 = split(Ap, 2), split(Bp, 2)
    c3 = _lib.gemm_split_bf16(a2, b2, _lib.BF16X3)
    assert _rel(c3, ref) < 3e-5
    a3, b3 = split(Ap, 3), split(Bp, 3)
    c6 = _lib.gemm_split_bf16(a3, b3, _lib.BF16X6)
    assert _rel(c6, ref) < 1e-5  # FP32 accumulation bounds the three-piece product


def test_split_pieces_reconstruct():
    x = torch.randn(10007, dtype=torch.float64, device="cuda") * 10
    p = _lib.split_bf16(x, 3)
    rec = p[0].double() + p[1].double() + p[2].double()
    assert float(((rec - x).abs() / x.abs()).max()) < 2 ** -22
