"""negfpy's own transmission() on sampled points of a workload (CPU timing leg).

bench.py uses this to time the reference itself -- negfpy installed into
baseline/_ref by baseline/install_ref.sh -- beside the oracle restatement.
Each task builds negfpy's Device1D / LeadBlocks from a point's blocks and
calls ``negfpy.core.transmission(..., surface_gf_method="sancho_rubio")``
(``src/negfpy/core/negf.py:306-357``), as negfpy's workflow does per point.
Workers run in a spawn pool with one BLAS thread each.
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

REF = Path(__file__).resolve().parent / "_ref"


def available() -> bool:
    return (REF / "negfpy" / "core" / "negf.py").exists()


def _init():
    for v in ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[v] = "1"
    if str(REF) not in sys.path:
        sys.path.insert(0, str(REF))


def task(args) -> float:
    from negfpy.core import transmission
    from negfpy.core.types import Device1D, LeadBlocks

    ll, lr = args["lead_l"], args["lead_r"]
    dev = Device1D(onsite_blocks=list(args["onsite"]), coupling_blocks=list(args["coupling"]))
    try:
        return float(transmission(args["omega"], dev, LeadBlocks(*ll), LeadBlocks(*lr), eta=args["eta"],
                                  surface_gf_method="sancho_rubio"))
    except (RuntimeError, ValueError):
        return float("nan")


def make_pool(processes: int):
    import multiprocessing as mp

    saved = {v: os.environ.get(v) for v in ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS", "MKL_NUM_THREADS")}
    for v in saved:
        os.environ[v] = "1"
    try:
        return mp.get_context("spawn").Pool(processes, initializer=_init)
    finally:
        for v, old in saved.items():
            if old is None:
                os.environ.pop(v, None)
            else:
                os.environ[v] = old
