"""The allocation-free device solve agrees with the allocating one.

negf_rgf_transmission_f64_noalloc exists for callers that cannot allocate
device memory when they call the library (a host program that fixed its GPU
memory budget up front, or a binding without a CUDA allocator): it keeps its
scratch in a static device array instead of a caller workspace.  This test
calls it through the C ABI twice in a row on two different systems -- an
order-48 slab with 48 points, then an order-24 slab with fewer points -- and
compares each result with negf_rgf_transmission_f64 on the same inputs, to
the FP64 tolerance of the parity tests (1e-10 relative, floor 1).  The second
call reuses the array: self-energies left over from the first call, or a
work counter that was not cleared (it would stand above the second call's
point count and leave its points unsolved, NaN), show up as a mismatch.  The
file is named to be collected last so that a run stopping at the first
failure has already run every other test; it also passes on its own in a
fresh process.
"""

import numpy as np
import pytest
import torch

from negfpy_b200 import _lib, engine
from negfpy_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _system(nz: int, omega_idx, k_idx):
    wl = W.subsample(W.slab_workload(n_omega=64, n_k=8, n_layers=6, nz=nz), omega_idx, k_idx)
    s = engine.StackedSystem.from_arrays(wl.lead_l, wl.lead_l, wl.onsite, wl.coupling, wl.n_layers)
    dev = _lib.require_cuda()
    K, Wn = len(wl.kpoints), len(wl.omegas)
    wi = torch.arange(Wn, device=dev).repeat_interleave(K)
    ki = torch.arange(K, device=dev, dtype=torch.int32).repeat(Wn)
    om = torch.tensor(wl.omegas, device=dev)[wi].contiguous()
    eta = torch.full_like(om, wl.eta)
    sr = engine.sgf_sr(*s.lead_l, om, eta, ki)
    return s, om, eta, ki, sr


def _noalloc(lib, s, om, eta, ki, sr):
    n, nl, nr = s.n, s.nl, s.nr
    K, Lo = s.onsite.shape[0], s.onsite.shape[1]
    P = int(om.shape[0])
    T = torch.full((P,), float("nan"), dtype=torch.float64, device=om.device)
    st = torch.full((P,), -7, dtype=torch.int32, device=om.device)
    cp = s.coupling
    rc = lib.negf_rgf_transmission_f64_noalloc(
        n, nl, nr, s.n_layers, P,
        s.onsite.data_ptr(), Lo * n * n if K > 1 else 0, 0 if Lo == 1 else n * n,
        cp.data_ptr(), cp.shape[1] * n * n if K > 1 else 0, 0 if cp.shape[1] == 1 else n * n,
        s.vl.data_ptr(), n * nl if s.vl.shape[0] > 1 else 0,
        s.vr.data_ptr(), n * nr if s.vr.shape[0] > 1 else 0,
        sr["g"].data_ptr(), nl * nl, sr["g"].data_ptr(), nr * nr,
        ki.data_ptr(), om.data_ptr(), eta.data_ptr(), sr["status"].data_ptr(),
        T.data_ptr(), st.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == 0, rc
    torch.cuda.synchronize()
    return T.cpu().numpy(), st.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_on_two_calls():
    lib = _lib.load()
    cases = [(8, list(range(0, 64, 4)), [0, 3, 5]),  # order 48, 48 points
             (4, [7, 21, 40, 55], [1, 6])]  # order 24, 8 points
    for nz, wi, ki_sel in cases:
        s, om, eta, ki, sr = _system(nz, wi, ki_sel)
        assert s.n == 6 * nz
        T_ref, st_ref = engine.rgf_transmission(s.onsite, s.coupling, s.n_layers, s.vl, s.vr, sr["g"], sr["g"], om,
                                                eta, ki, sr["status"])
        T_ref, st_ref = T_ref.cpu().numpy(), st_ref.cpu().numpy()
        assert np.all(st_ref == 0)
        T, st = _noalloc(lib, s, om, eta, ki, sr)
        assert np.array_equal(st, st_ref)
        err = np.abs(T - T_ref) / np.maximum(np.abs(T_ref), 1.0)
        assert err.max() <= TOL, (s.n, err.max())


def test_noalloc_rejects_unsupported_block_order():
    lib = _lib.load()
    dev = _lib.require_cuda()
    x = torch.zeros(8, dtype=torch.float64, device=dev)
    rc = lib.negf_rgf_transmission_f64_noalloc(
        64, 64, 64, 2, 1, x.data_ptr(), 0, 0, x.data_ptr(), 0, 0, x.data_ptr(), 0, x.data_ptr(), 0,
        x.data_ptr(), 0, x.data_ptr(), 0, None, x.data_ptr(), x.data_ptr(), None, x.data_ptr(), None,
        torch.cuda.current_stream().cuda_stream)
    assert rc == -2  # NEGF_EUNSUPPORTED
    msg = lib.negf_last_error().decode()
    assert msg.startswith("negf_rgf_transmission_f64_noalloc") and "48" in msg, msg
