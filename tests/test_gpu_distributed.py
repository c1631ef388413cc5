"""The omega-sharded spectrum (distributed.transmission_grid_sharded) on one
NCCL rank: the gathered table equals transmission_grid's, and the shard is
the whole grid."""

from __future__ import annotations

import datetime
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import negfpy_b200 as nb  # noqa: E402
from negfpy_b200.models import ChainParams, device_perfect_chain, lead_blocks  # noqa: E402


def test_sharded_spectrum_one_nccl_rank():
    import torch.distributed as dist

    from negfpy_b200.distributed import transmission_grid_sharded

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        p = ChainParams(1.0, 1.0)
        dev, lead = device_perfect_chain(6, p), lead_blocks(p)
        om = (np.arange(37, dtype=float) + 0.5) * (2.0 / 37)
        res = transmission_grid_sharded(om, None, dev, lead, lead, eta=1e-8)
        ref = nb.transmission_grid(om, None, dev, lead, lead, eta=1e-8)
        assert np.array_equal(res["shard"], np.arange(om.size))
        assert np.array_equal(res["T"], ref["T"]) and np.array_equal(res["status"], ref["status"])
    finally:
        dist.destroy_process_group()
