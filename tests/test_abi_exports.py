"""The C-ABI library builds, loads without a GPU and exports every declared symbol."""

import re
from pathlib import Path

from negfpy_b200 import _build, _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "negf_b200.h"


def declared_symbols() -> set[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(negf_[a-z0-9_]+)\s*\(", text))


def test_library_loads_and_exports_header_symbols():
    lib = _lib.load()
    decl = declared_symbols()
    assert decl, "no declarations parsed"
    for name in decl:
        assert hasattr(lib, name), name
    assert decl == set(_lib.exported_symbols())
    assert lib.negf_get_version() == 1


def test_workspace_query_without_gpu_is_safe():
    lib = _lib.load()
    # size queries for unsupported orders return 0 rather than touching a device
    assert lib.negf_rgf_workspace_bytes(0, 1, 1) == 0
    assert lib.negf_rgf_workspace_bytes(1, 1, 1) == 256


def test_build_is_for_sm100a():
    assert "arch=compute_100a,code=sm_100a" in " ".join(_build.ARCH)


def test_fp32_product_path_switch_without_gpu():
    """The product-tiling switch is host state only: it validates the order
    and the path, refuses tcgen05 tiles above order 128 and reports the path
    in effect (padded orders share a setting)."""
    lib = _lib.load()
    assert lib.negf_set_fp32_product_path(48, 1) == 1
    assert lib.negf_set_fp32_product_path(40, 0) == 0  # pads to 48
    assert lib.negf_set_fp32_product_path(48, -1) in (0, 1)  # default: environment
    assert lib.negf_set_fp32_product_path(160, 1) == -2  # NEGF_EUNSUPPORTED
    assert "128" in lib.negf_last_error().decode()
    assert lib.negf_set_fp32_product_path(160, 0) == 0
    assert lib.negf_set_fp32_product_path(0, 0) == -1  # NEGF_EINVAL
    assert lib.negf_set_fp32_product_path(48, 2) == -1
    lib.negf_set_fp32_product_path(160, -1)


def test_product_path_tuner_keeps_mma_sync_above_order_128(tmp_path):
    """Orders above 128 have only the mma.sync tiling: the tuner sets it
    without timing anything (no GPU needed)."""
    from types import SimpleNamespace

    from negfpy_b200.autotune import ProductPathTuner

    system = SimpleNamespace(n=160, nl=160, nr=160, n_layers=4)
    e = ProductPathTuner(tmp_path / "tune.json").tune(system, None, None, None)
    assert e["path"] == 0 and e["order"] == "mma.sync" and e["timings"] == {}
    assert _lib.load().negf_set_fp32_product_path(160, -1) == 0


def test_per_point_adjoint_entries_validate_without_gpu():
    """The per-point adjoint entries reject bad sizes and missing pointers
    before touching a device, with messages naming the entry point."""
    lib = _lib.load()
    z = [None] * 40
    # negf_sgf_adjoint_points_f64(n_lead=0, ...)
    rc = lib.negf_sgf_adjoint_points_f64(0, 4, 1, None, None, 0, None, 0, None, 0, None, None, None, 1e-12, 10,
                                         *z[:6], None, 0, None)
    assert rc == -1 and lib.negf_last_error().decode().startswith("negf_sgf_adjoint_points_f64")
    # negf_rgf_adjoint_points_f64 with every pointer missing
    rc = lib.negf_rgf_adjoint_points_f64(4, 4, 4, 2, 1, None, 0, 0, None, 0, 0, None, 0, None, 0, None, 0, None, 0,
                                         *z[:11], None, 0, None)
    assert rc == -1
    msg = lib.negf_last_error().decode()
    assert msg.startswith("negf_rgf_adjoint_points_f64") and "null pointer" in msg
