"""Multi-rank plumbing of the benchmark on CPU: two gloo ranks (no GPU), the way torchrun launches bench.py.

Each rank steps its own scenes (independent units, no collective on the data path); the job's time is the slowest
rank's and its body-steps the sum over ranks. A rank that leaves before a collective is noticed by the other through
a short process-group timeout instead of a hang.
"""
import datetime
import os
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _init(rank, world, port, timeout_s=30):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=timeout_s))


def _combine_worker(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    import bench
    _init(rank, world, port)
    ms = [40.0, 55.0][rank]
    body_steps = [1.0e6, 3.0e6][rank]
    res = bench.combine(dist, ms, body_steps)
    dist.barrier()
    dist.destroy_process_group()
    out[rank] = res


def _dead_rank_worker(rank, world, port, out):
    _init(rank, world, port, timeout_s=3)
    if rank == 1:
        out[rank] = "left"
        os._exit(0)          # leaves between steps, before the next collective
    try:
        dist.barrier()
        out[rank] = "no error"
    except Exception as e:   # the short timeout ends the collective with an error
        out[rank] = type(e).__name__


def _free_port():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_timing_is_max_and_body_steps_sum():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    mp.start_processes(_combine_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    for r in (0, 1):
        ms_max, total, value = out[r]
        assert ms_max == 55.0 and total == 4.0e6
        assert value == pytest.approx(4.0e6 / 0.055)


def test_ranks_step_independent_scene_mixes():
    sys.path.insert(0, str(ROOT))
    import bench
    from shatterforge_b200 import scenes as S
    a = S.debris_mix(seed=bench.rank_seed(0), n_scenes=3, scale=0.02)
    b = S.debris_mix(seed=bench.rank_seed(1), n_scenes=3, scale=0.02)
    assert bench.rank_seed(0) != bench.rank_seed(1)
    assert not np.array_equal(a[0].body_pose[:10], b[0].body_pose[:10])


def test_a_rank_that_leaves_is_detected_by_timeout():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    ps = mp.start_processes(_dead_rank_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=False)
    for p in ps.processes:
        p.join(timeout=60)
    assert out.get(1) == "left"
    assert out.get(0) not in (None, "no error")
