"""The multi-GPU frame's host logic on CPU ranks (gloo, world size 2).

`bench.py --gpus N` gives rank r the sample range of bench.rank_sample_range
and sums the ranks' film sums with one all-reduce: the result must be the
film of all N ranges' samples. Here two gloo ranks render their ranges with
the CPU oracle and all-reduce the sums; rank 0 compares with one render of
every sample (the same per-sample values, summed in another order)."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]
W, H, SPP, BOUNCES = 24, 16, 3, 4


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out: str) -> None:
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch
    import torch.distributed as dist

    import bench
    import oracle
    from cenote_b200 import scenes

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        first, count = bench.rank_sample_range(rank, SPP)
        img = oracle.OracleScene(scenes.cornell(W, H, SPP, BOUNCES)).render_sum(W, H, first, count, BOUNCES, threads=1)
        sums = torch.from_numpy(np.ascontiguousarray(img, np.float32))
        dist.all_reduce(sums)
        if rank == 0:
            np.save(out, sums.numpy())
    finally:
        dist.destroy_process_group()


def test_two_ranks_sum_to_the_whole_frame(tmp_path):
    import oracle
    from cenote_b200 import scenes

    out = str(tmp_path / "frame.npy")
    mp.start_processes(_rank, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    frame = np.load(out)
    whole = oracle.OracleScene(scenes.cornell(W, H, SPP, BOUNCES)).render_sum(W, H, 0, 2 * SPP, BOUNCES, threads=1)
    assert np.allclose(frame, whole, rtol=1e-5, atol=1e-6)
    assert np.all(frame[..., 3] == 2 * SPP)  # every pixel took every sample exactly once


def test_rank_ranges_tile_the_samples():
    sys.path.insert(0, str(ROOT))
    import bench

    ranges = [bench.rank_sample_range(r, 16) for r in range(8)]
    covered = sorted(i for f, n in ranges for i in range(f, f + n))
    assert covered == list(range(8 * 16))
