"""The exchanges of the multi-GPU paths, on two CPU processes over gloo:
frames shared by bin-packing and their energies gathered back in frame
order, the parameter gradient summed in f64 in one all-reduce, the
slowest rank's time.  The second test exchanges real per-frame results
(the FP64 oracle's energies of solvated frames, and its reciprocal-space
charge gradient dE/dq and forces of force-matching frames) and checks
that the frames split over two ranks give what one process gives."""

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


def _oracle_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=120))
    try:
        from oracle import oracle as O
        from mdir_b200 import systems
        from mdir_b200.batch import shard
        from mdir_b200.ranks import gather_frame_values, sum_gradients
        frames = systems.batch_frames(count=6, low=900, high=1500, seed=21)
        mine = shard([len(f["charges"]) for f in frames], world)[rank]
        e = np.array([[O.evaluate(frames[k], frames[k]["positions"])["energy"]] for k in mine])
        energies = gather_frame_values(len(frames), mine, e)
        s, X, _ = systems.force_matching(frames=4, waters=300)
        n = len(s["charges"])
        dq = torch.zeros(n, dtype=torch.float64)
        forces = torch.zeros((n, 3), dtype=torch.float64)
        for k in range(rank, len(X), world):
            ref = O.evaluate(s, X[k], want_potential=True)
            dq += torch.from_numpy(ref["potential"])
            forces += torch.from_numpy(ref["forces"])
        sum_gradients(dq, forces)
        out[rank] = (energies[:, 0].tolist(), dq.numpy().tolist(), forces.numpy().reshape(-1).tolist())
    finally:
        dist.destroy_process_group()


def test_real_frame_results_over_two_gloo_ranks():
    from oracle import oracle as O
    from mdir_b200 import systems
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    mp.start_processes(_oracle_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    frames = systems.batch_frames(count=6, low=900, high=1500, seed=21)
    want_e = [O.evaluate(f, f["positions"])["energy"] for f in frames]
    s, X, _ = systems.force_matching(frames=4, waters=300)
    refs = [O.evaluate(s, X[k], want_potential=True) for k in range(len(X))]
    want_dq = sum(r["potential"] for r in refs)
    want_f = sum(r["forces"] for r in refs)
    for r in range(world):
        e, dq, f = out[r]
        assert e == want_e  # each frame's value, in frame order, bit for bit
        np.testing.assert_allclose(dq, want_dq, rtol=1e-12, atol=1e-12 * np.abs(want_dq).max())
        np.testing.assert_allclose(np.reshape(f, (-1, 3)), want_f, rtol=1e-12, atol=1e-12 * np.abs(want_f).max())
