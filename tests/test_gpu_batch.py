"""The batching form: frames of uneven sizes, each with its own cell and PME
grid, evaluated by one launch of each kernel over all of them, against the
FP64 oracle frame by frame and against one context per frame."""

import numpy as np
import pytest
import torch

from oracle import oracle as O
from mdir_b200 import NonbondedTerm, systems
from mdir_b200 import _lib as L
from mdir_b200.batch import TERMS, BatchEvaluator

pytestmark = pytest.mark.gpu
# The solvated frames put solute atoms (sigma up to 0.40 nm) where water
# sites were, so some contacts are far inside the LJ wall (forces up to
# 3e6 kJ/mol/nm); the f32 pair arithmetic of the device path (one context
# or the batch alike: they agree to 1e-7) stays within 2e-5 RMS of FP64
# there, and within 1e-5 on the water box (test_gpu_forces.py).
FORCE_RMS_TOL = 2e-5
ENERGY_TOL = 1e-6


def rms_rel(a, b):
    return float(np.sqrt(np.mean((a - b) ** 2) / np.mean(b ** 2)))


@pytest.fixture(scope="module")
def frames():
    # the smallest frames of the batching workload (2.15 nm cells: images of
    # the own group) up to 4,500 atoms; one frame unwrapped by whole cells
    fr = systems.batch_frames(count=7, low=1000, high=4500, seed=41)
    fr[2] = dict(fr[2])
    fr[2]["positions"] = fr[2]["positions"] + np.array([3.0, -2.0, 1.0]) * fr[2]["box"]
    return fr


def test_batch_matches_the_oracle_frame_by_frame(cuda, frames):
    ev = BatchEvaluator(frames)
    F = ev.force(energy=True).cpu().numpy()
    E = ev.energies()
    for k, fr in enumerate(frames):
        ref = O.evaluate(fr, fr["positions"])
        assert rms_rel(ev.frame(k, F), ref["forces"]) < FORCE_RMS_TOL, k
        scale = sum(abs(v) for v in ref["terms"].values())
        for t in TERMS:
            assert abs(E[t][k] - ref["terms"][t]) <= ENERGY_TOL * scale, (k, t, E[t][k], ref["terms"][t])


def test_batch_equals_one_context_per_frame(cuda, frames):
    ev = BatchEvaluator(frames)
    F = ev.force(energy=True).cpu().numpy()
    E = ev.energies()
    for k, fr in enumerate(frames):
        n = len(fr["charges"])
        t = NonbondedTerm(n)
        t.set_particles(fr["charges"], fr["types"], fr["sigma"], fr["epsilon"])
        t.set_exclusions(pairs=fr["excluded_pairs"])
        t.set_interaction(fr["cutoff"], fr["reach"], fr["beta"])
        t.set_pme(fr["grid"], fr["order"])
        x = torch.tensor(fr["positions"], dtype=torch.float64, device="cuda")
        t.build(x, fr["box"])
        f1 = t.force(x, energy=True).cpu().numpy()
        e1 = t.energies()
        assert rms_rel(ev.frame(k, F), f1) < 1e-6, k
        # the same pairs and f32 pair terms: the sums agree to rounding
        for name in ("lj", "coulomb", "excluded"):
            assert abs(E[name][k] - e1[name]) <= 1e-9 * max(1.0, abs(e1[name])), (k, name)
        assert abs(E["reciprocal"][k] - e1["reciprocal"]) <= 1e-6 * max(1.0, abs(e1["reciprocal"])), k
        t.close()


def test_graph_replay_and_autotuned_shapes_give_the_same_forces(cuda, frames):
    ev = BatchEvaluator(frames)
    F0 = ev.force(energy=True).clone()
    E0 = ev.energies()["potential"]
    for _ in range(2):
        F1 = ev.force(energy=True, graph=True).clone()
    E1 = ev.energies()["potential"]
    assert rms_rel(F1.cpu().numpy(), F0.cpu().numpy()) < 1e-6
    # up to the order of the f32 atomics of PME spreading
    assert np.allclose(E1, E0, rtol=1e-7, atol=1e-6)
    choice = ev.autotune()
    assert choice["search_warps"] in (1, 4) and 1 <= choice["pair_blocks_per_sm"] <= 4
    assert choice["staging_depth"] in (1, 2)
    # every shape the autotuner chooses among gives the same forces
    for depth in (1, 2):
        for blocks in (4, 1):
            ev.set_tuning(pair_blocks_per_sm=blocks, staging_depth=depth)
            Fd = ev.force(energy=True).clone()
            assert rms_rel(Fd.cpu().numpy(), F0.cpu().numpy()) < 1e-6, (depth, blocks)
    ev.set_tuning(pair_blocks_per_sm=choice["pair_blocks_per_sm"], staging_depth=choice["staging_depth"])
    F2 = ev.force(energy=True).clone()
    assert rms_rel(F2.cpu().numpy(), F0.cpu().numpy()) < 1e-6
    # new positions: the graph reads them from the same buffer
    ev.set_positions([fr["positions"] + 0.003 for fr in frames])
    ev.build()
    F3 = ev.force(energy=True, graph=True).cpu().numpy()
    ref = O.evaluate(frames[1], frames[1]["positions"] + 0.003)
    assert rms_rel(ev.frame(1, F3), ref["forces"]) < FORCE_RMS_TOL


def test_exclusions_across_frames_are_refused(cuda, frames):
    ev = BatchEvaluator(frames[:2])
    n = ev.n
    bad = np.array([[0, n - 1]])  # atom 0 of frame 0 with the last atom of frame 1
    from mdir_b200.term import exclusion_rows, _hp, _host
    off, part = exclusion_rows(n, bad)
    s = L.lib().mdrtNbBatchSetExclusions(ev._h, _hp(_host(off, np.int32)), _hp(_host(part, np.int32)))
    assert s == L.INVALID_ARGUMENT
