"""Complex FP32 products on the fifth-generation tensor cores
(negf_cgemm_tf32x3: tcgen05.mma kind::tf32 with TMEM accumulators, 3 x TF32
split) against a plain PyTorch FP32 reference of the same op (complex64
matmul with TF32 disabled), for every conjugation of the operands and block
orders 16 .. 128.  The 3 x TF32 split carries ~2^-22 relative error per
product term and the FP32 accumulation in Tensor Memory adds its own
rounding over K; the bound is 1e-5 of the largest entry."""

from __future__ import annotations

import pytest
import torch

pytestmark = pytest.mark.gpu

from negfpy_b200 import engine  # noqa: E402


@pytest.mark.parametrize("n", [16, 48, 96, 128])
@pytest.mark.parametrize("ca,cb", [(False, False), (True, False), (False, True), (True, True)])
def test_cgemm_matches_fp32_reference(n, ca, cb):
    gen = torch.Generator(device="cpu").manual_seed(n + 2 * ca + cb)
    P = 37
    a = torch.randn((P, n, n), dtype=torch.complex64, generator=gen).cuda()
    b = torch.randn((P, n, n), dtype=torch.complex64, generator=gen).cuda()
    c, st = engine.cgemm_tf32x3(a, b, ca, cb)
    assert bool((st == 0).all())
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        oa = a.conj().transpose(-1, -2) if ca else a
        ob = b.conj().transpose(-1, -2) if cb else b
        ref = oa @ ob
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    err = float((c - ref).abs().max() / ref.abs().max())
    assert err < 1e-5, err


def test_cgemm_rejects_unsupported_order():
    a = torch.zeros((1, 24, 24), dtype=torch.complex64)
    with pytest.raises(RuntimeError, match="multiple of 16"):
        engine.cgemm_tf32x3(a, a)
