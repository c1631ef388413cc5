"""ctypes binding of libnegfb200.so (the C ABI declared in include/negf_b200.h).

Every product call goes through this module into the CUDA library.  There is
no CPU fallback: without a CUDA device, or without the built library, calls
raise instead of computing anything.
"""

from __future__ import annotations

import ctypes as C
import threading

import torch

from . import _build

_lock = threading.Lock()
_lib = None

OK, MAXITER, NONFINITE, SINGULAR, REFINE_FAIL, BAD_ITEM, UNSTABLE = 0, 1, 2, 3, 4, 5, 6
STATUS_NAMES = {OK: "ok", MAXITER: "maxiter", NONFINITE: "non_finite", SINGULAR: "singular", REFINE_FAIL: "refine_failed",
                BAD_ITEM: "bad_item", UNSTABLE: "unstable"}

_P = C.c_void_p
_I = C.c_int
_LL = C.c_longlong
_D = C.c_double
_SZ = C.c_size_t

_SIGNATURES = {
    "negf_get_version": (_I, []),
    "negf_last_error": (C.c_char_p, []),
    "negf_max_order_f64": (_I, []),
    "negf_sgf_workspace_bytes": (_SZ, [_I]),
    "negf_sgf_sr_f64": (_I, [_I, _I, _P, _P, _P, _LL, _P, _P, _P, _D, _I, _P, _P, _P, _P, _P, _SZ, _P]),
    "negf_rgf_workspace_bytes": (_SZ, [_I, _I, _I]),
    "negf_rgf_transmission_f64": (
        _I,
        [_I, _I, _I, _I, _I, _P, _LL, _LL, _P, _LL, _LL, _P, _LL, _P, _LL, _P, _LL, _P, _LL, _P, _P, _P, _P, _P,
         _P, _P, _SZ, _P],
    ),
    "negf_rgf_transmission_f64_noalloc": (
        _I,
        [_I, _I, _I, _I, _I, _P, _LL, _LL, _P, _LL, _LL, _P, _LL, _P, _LL, _P, _LL, _P, _LL, _P, _P, _P, _P, _P,
         _P, _P],
    ),
    "negf_rgf_mixed_workspace_bytes": (_SZ, [_I, _I, _I]),
    "negf_rgf_transmission_mixed": (
        _I,
        [_I, _I, _I, _I, _I, _P, _LL, _LL, _P, _LL, _LL, _P, _LL, _P, _LL, _P, _LL, _P, _LL, _P, _P, _P, _P, _P,
         _P, _P, _SZ, _P],
    ),
    "negf_rgf_refined_workspace_bytes": (_SZ, [_I, _I, _I, _I]),
    "negf_rgf_transmission_refined": (
        _I,
        [_I, _I, _I, _I, _I, _P, _LL, _LL, _P, _LL, _LL, _P, _LL, _P, _LL, _P, _LL, _P, _LL, _P, _P, _P, _P, _D,
         _I, _P, _P, _P, _P, _SZ, _P],
    ),
    "negf_cgemm_tf32x3": (_I, [_I, _I, _P, _P, _P, _I, _I, _P, _P]),
    "negf_set_fp32_product_path": (_I, [_I, _I]),
    "negf_batch_max_grid": (_I, [_I, _I, _I]),
    "negf_batch_workspace_bytes": (_SZ, [_I, _I, _I, _I]),
    "negf_batch_system_bytes": (_SZ, []),
    "negf_batch_transmission": (
        _I, [_P, _I, _I, _P, _P, _P, _I, _D, _I, _I, _I, _I, _P, _P, _P, _P, _SZ, _P],
    ),
    "negf_device_green_workspace_bytes": (_SZ, [_I, _I, _I, _I]),
    "negf_device_green_f64": (
        _I,
        [_I, _I, _I, _I, _I, _P, _LL, _LL, _P, _LL, _LL, _P, _LL, _P, _LL, _P, _LL, _P, _LL, _P, _P, _P, _P, _P,
         _P, _P, _P, _P, _SZ, _P],
    ),
    "negf_adjoint_workspace_bytes": (_SZ, [_I, _I, _I, _I]),
    "negf_rgf_adjoint_f64": (
        _I,
        [_I, _I, _I, _I, _I, _P, _LL, _LL, _P, _LL, _LL, _P, _LL, _P, _LL, _P, _LL, _P, _LL, _P, _P, _P, _P, _P,
         _P, _P, _P, _P, _P, _SZ, _P],
    ),
    "negf_rgf_adjoint_sigma_f64": (
        _I,
        [_I, _I, _I, _I, _I, _P, _LL, _LL, _P, _LL, _LL, _P, _LL, _P, _LL, _P, _LL, _P, _LL, _P, _P, _P, _P, _P,
         _P, _P, _P, _P, _P, _P, _P, _SZ, _P],
    ),
    "negf_sgf_adjoint_workspace_bytes": (_SZ, [_I, _I]),
    "negf_sgf_adjoint_f64": (
        _I,
        [_I, _I, _I, _P, _P, _LL, _P, _LL, _P, _LL, _P, _P, _P, _D, _I, _P, _P, _P, _P, _P, _P, _P, _SZ, _P],
    ),
    "negf_sgf_adjoint_points_f64": (
        _I,
        [_I, _I, _I, _P, _P, _LL, _P, _LL, _P, _LL, _P, _P, _P, _D, _I, _P, _P, _P, _P, _P, _P, _P, _SZ, _P],
    ),
    "negf_rgf_adjoint_points_f64": (
        _I,
        [_I, _I, _I, _I, _I, _P, _LL, _LL, _P, _LL, _LL, _P, _LL, _P, _LL, _P, _LL, _P, _LL, _P, _P, _P, _P, _P,
         _P, _P, _P, _P, _P, _P, _P, _SZ, _P],
    ),
    "negf_kavg_f64": (_I, [_P, _I, _I, _P, _P]),
    "negf_heat_current_f64": (_I, [_P, _P, _I, _I, _D, _D, _P, _P]),
    "negf_kmoments_f64": (_I, [_P, _I, _I, _P, _P, _P]),
    "negf_kspace_blocks_f64": (_I, [_P, _P, _I, _P, _I, _I, _P, _P, _D, _P, _P]),
    "negf_fcs_cumulants_f64": (_I, [_P, _P, _P, _I, _D, _D, _P, _P]),
    "negf_kappa_f64": (_I, [_P, _P, _I, _P, _I, _D, _P, _P]),
}


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


def load(build_if_missing: bool = True):
    """Load (building first if needed) the shared library; does not need a GPU."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if build_if_missing and _build.needs_build():
            _build.build()
        if not _build.LIB.exists():
            raise RuntimeError(f"{_build.LIB} is missing; run negfpy_b200._build.build()")
        lib = C.CDLL(str(_build.LIB))
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("negfpy_b200 runs on a CUDA device only (no CPU fallback); no GPU is visible")
    return torch.device("cuda", torch.cuda.current_device())


def check(rc: int, what: str) -> None:
    if rc != 0:
        msg = load().negf_last_error().decode(errors="replace")
        raise RuntimeError(f"{what} failed (code {rc}): {msg}")


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def stream_handle(stream: torch.cuda.Stream | None = None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream
