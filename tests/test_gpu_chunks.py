"""The stacked solve in chunks: every point's T, status and sweep counts are
bitwise the same whether the points go in one launch pair or in many chunks
(each point is solved independently), for the default chunk size and for
small explicit ones, with identical and with different leads."""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from negfpy_b200 import engine, spectrum, workloads as W  # noqa: E402


def _points(wl, stride):
    wi = np.arange(0, wl.omegas.size, stride)
    K = len(wl.kpoints)
    om_w = torch.tensor(wl.omegas[wi], dtype=torch.float64, device="cuda")
    w_idx, k_idx = spectrum.grid_points(len(wi), K, om_w.device)
    om = om_w[w_idx].contiguous()
    return om, k_idx, torch.full_like(om, wl.eta)


@pytest.mark.parametrize("same_leads", [True, False])
def test_chunked_solve_is_bitwise_the_single_launch(same_leads):
    wl = W.slab_workload(n_omega=64, n_k=8, n_layers=4, nz=4)
    s = engine.StackedSystem.from_arrays(wl.lead_l, wl.lead_l, wl.onsite, wl.coupling, wl.n_layers,
                                         same_leads=same_leads)
    om, ki, eta = _points(wl, 1)
    ref = s.transmission(om, ki, eta)
    assert int((ref["status"] != 0).sum()) == 0
    for chunk in (97, 256):
        r = s.transmission(om, ki, eta, chunk=chunk)
        for key in ("T", "status", "iters_left", "iters_right"):
            assert torch.equal(r[key], ref[key]), (chunk, key)
