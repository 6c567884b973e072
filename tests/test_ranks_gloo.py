"""The exchanges of the multi-GPU paths, on two CPU processes over gloo:
frames shared by bin-packing and their energies gathered back in frame
order, the parameter gradient summed in f64 in one all-reduce, the
slowest rank's time."""

import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        from mdir_b200.batch import shard
        from mdir_b200.ranks import gather_frame_values, max_over_ranks, sum_gradients
        rng = np.random.default_rng(4)
        atoms = 3 * rng.integers(333, 2667, size=40)
        mine = shard(atoms, world)[rank]
        # a stand-in per-frame energy: a function of the frame's number and size
        energies = np.array([[f * 10.0 + atoms[f], -float(f)] for f in mine])
        full = gather_frame_values(len(atoms), mine, energies)
        # a stand-in gradient: rank r holds r + 1 in every entry
        q = torch.full((7,), float(rank + 1), dtype=torch.float64)
        table = torch.full((2, 3, 3), 0.5 * (rank + 1), dtype=torch.float64)
        sum_gradients(q, table)
        slowest = max_over_ranks(1.0 + rank)
        out[rank] = (full.tolist(), q.tolist(), table.reshape(-1).tolist(), slowest, mine)
    finally:
        dist.destroy_process_group()


def test_frames_gradients_and_times_over_two_gloo_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    rng = np.random.default_rng(4)
    atoms = 3 * rng.integers(333, 2667, size=40)
    want = np.array([[f * 10.0 + atoms[f], -float(f)] for f in range(len(atoms))])
    covered = []
    for r in range(world):
        full, q, table, slowest, mine = out[r]
        assert np.array_equal(np.array(full), want)
        assert q == [3.0] * 7  # 1 + 2
        assert table == [1.5] * 18  # 0.5 + 1.0
        assert slowest == 2.0
        covered += mine
    assert sorted(covered) == list(range(len(atoms)))
