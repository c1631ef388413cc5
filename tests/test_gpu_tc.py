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


def _slab_points(stride=64):
    import numpy as np

    from negfpy_b200 import workloads as W

    wl = W.slab_workload()
    wi = np.arange(0, wl.omegas.size, stride)
    K = len(wl.kpoints)
    s = engine.StackedSystem.from_arrays(wl.lead_l, wl.lead_l, wl.onsite, wl.coupling, wl.n_layers, same_leads=True)
    om = torch.as_tensor(np.repeat(wl.omegas[wi], K), device="cuda", dtype=torch.float64)
    ki = torch.as_tensor(np.tile(np.arange(K), len(wi)), device="cuda", dtype=torch.int32)
    return s, om, ki, torch.full_like(om, wl.eta)


def test_sweeps_on_tcgen05_tiles_match_f64():
    """The FP32 sweeps with their products on tcgen05 tiles (opt-in per block
    order): the mixed sweep within the FP32 bound of the mma.sync tiling
    (|dT| <= 1e-4 max(1, |T|) at n = 48) and the refined solve at the FP64
    parity bound (1e-10), the same bars as with the default tiling."""
    s, om, ki, eta = _slab_points()
    r64 = s.transmission(om, ki, eta)
    try:
        assert engine.set_fp32_product_path(s.n, 1) == 1
        rm = s.transmission(om, ki, eta, precision="mixed")
        rr = s.transmission(om, ki, eta, precision="refined")
    finally:
        engine.set_fp32_product_path(s.n, -1)
    t64 = r64["T"]
    assert bool((rm["status"] == 0).all()) and bool((rr["status"] == 0).all())
    err_m = float(((rm["T"] - t64).abs() / t64.abs().clamp_min(1.0)).max())
    err_r = float(((rr["T"] - t64).abs() / t64.abs().clamp_min(1.0)).max())
    assert err_m <= 1e-4, err_m
    assert err_r <= 1e-10, err_r


def test_product_path_tuner_sets_and_caches_a_path(tmp_path):
    from negfpy_b200.autotune import ProductPathTuner

    s, om, ki, eta = _slab_points(stride=256)
    tuner = ProductPathTuner(tmp_path / "tune.json")
    try:
        e1 = tuner.tune(s, om, ki, eta, precision="mixed", reps=1)
        assert e1["path"] in (0, 1) and not e1["cached"]
        assert set(e1["timings"]) == {"1/mma.sync", "1/tcgen05"}
        assert engine.set_fp32_product_path(s.n, e1["path"]) == e1["path"]
        e2 = ProductPathTuner(tmp_path / "tune.json").tune(s, om, ki, eta, precision="mixed")
        assert e2["cached"] and e2["path"] == e1["path"]
    finally:
        engine.set_fp32_product_path(s.n, -1)
