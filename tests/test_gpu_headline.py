"""Parity on the shapes the benchmark measures: the 7,850-water TIP3P box
(23,550 atoms, 64^3 grid) at the autotuner's reaches (outer lists at
1.7 nm, pruned lists at 1.025 nm) in the default mixed mode; the public API
(compile -> Simulation.run) against the integrator it drives; and the
256-frame batch of 1,000-8,000-atom solvated frames, frame by frame.

The oracle: the FP64 evaluation of the same method (same beta, grid and
order), the f32 pair set of the build (MDIR's distance formula,
GroupsBuild.cpp:2592-2607), and the f32 restatement of the pruning
(MDExecToGPU.cpp:9588)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
import mdir_b200 as mdir
from mdir_b200 import NonbondedTerm, systems
from mdir_b200 import _lib as L
from mdir_b200.batch import TERMS, BatchEvaluator
from mdir_b200.md import Integrator

pytestmark = pytest.mark.gpu

FORCE_RMS_TOL = 1e-5      # the water box: RMS relative force error against FP64
FRAME_FORCE_RMS_TOL = 2e-5  # solvated frames (solute atoms deep in LJ walls), as test_gpu_batch.py
ENERGY_TOL = 1e-6         # each term within 1e-6 of the potential's scale
# Solvated frames whose solute atoms sit where water sites were have LJ
# energies of 1e6 to 6e6 kJ/mol from a few wall contacts near 0.12 nm
# (U ~ r^-12, so dU/U = 12 dr/r): the f32 rounding of those pairs'
# coordinates (~1e-7 nm in a 4 nm cell) alone moves the term by up to
# ~1e-5 of it (frames 44 and 55 of the 256: 3.4e-6 and 8.9e-6), so the
# frames' energies are held to 1e-5 of the scale.
FRAME_ENERGY_TOL = 1e-5
REACH, PRUNED = 1.7, 1.025


def rms_rel(f, ref):
    return np.sqrt(np.mean(np.sum((f - ref) ** 2, 1))) / np.sqrt(np.mean(np.sum(ref ** 2, 1)))


def canon(p):
    p = np.asarray(p, dtype=np.int64)
    return p[np.lexsort((p[:, 2], p[:, 1], p[:, 0]))]


@pytest.fixture(scope="module")
def box23550():
    s = systems.tip3p()
    assert len(s["charges"]) == 23550 and list(s["grid"]) == [64, 64, 64]
    # a second configuration: every atom moved by less than half the
    # pruned skin of the build at the initial positions
    rng = np.random.default_rng(12)
    d = rng.normal(size=s["positions"].shape)
    d *= (0.9 * 0.5 * (PRUNED - s["cutoff"])) / np.linalg.norm(d, axis=1, keepdims=True).max()
    return s, s["positions"] + d


def tuned_term(s, deterministic=False):
    t = NonbondedTerm(len(s["charges"]))
    t.set_particles(s["charges"], s["types"], s["sigma"], s["epsilon"])
    t.set_exclusions(pairs=s["excluded_pairs"])
    t.set_interaction(s["cutoff"], REACH, s["beta"])
    t.set_pruned_reach(PRUNED)
    t.set_pme(s["grid"], s["order"])
    t.set_deterministic(deterministic)
    return t


def test_outer_and_pruned_lists_at_the_tuned_reaches(cuda, box23550):
    s, x1 = box23550
    x0 = s["positions"]
    t = tuned_term(s)
    xd = torch.tensor(x0, device=cuda)
    sizes = t.build(xd, s["box"])
    # the outer lists: the oracle's set of (pair, image) at 1.7 nm, bit for bit
    got = t.pair_set(sizes)
    count, ref = O.pairset(x0, s["box"], REACH, O.rows_from_pairs(len(x0), s["excluded_pairs"]))
    assert len(got) == count > 20_000_000
    np.testing.assert_array_equal(canon(got), canon(ref))
    del got, ref
    # the pruned lists, entry for entry and in order, at the build's
    # positions and after the atoms moved
    G = int(sizes[L.SIZE_GROUPS])
    for x in (x0, x1):
        xd = torch.tensor(x, device=cuda)
        t.prune(xd, s["box"])
        torch.cuda.synchronize()
        cap = t.info()["list_capacity"]
        want = O.prune_lists(t.buffer(L.SLOT_ENTRIES, np.int32, 2)[: G * cap].reshape(G, cap, 2),
                             t.buffer(L.SLOT_COUNTS, np.int32)[:G], t.buffer(L.SLOT_PLACED, np.float32, 4),
                             t.buffer(L.SLOT_ORDER, np.int32), list(s["box"]), PRUNED)
        got_c = t.buffer(L.SLOT_INNER_COUNTS, np.int32)[:G]
        got_e = t.buffer(L.SLOT_INNER_ENTRIES, np.int32, 2)[: G * cap].reshape(G, cap, 2)
        assert sum(len(r) for r in want) > 0
        for g in range(G):
            assert got_c[g] == len(want[g]), g
            e = got_e[g, : got_c[g]].astype(np.int64)
            e[:, 1] &= 0xFFFFFFFF
            np.testing.assert_array_equal(e, want[g])
    t.close()


@pytest.mark.parametrize("deterministic", [False, True])
def test_forces_and_energies_at_the_tuned_reaches(cuda, box23550, deterministic):
    s, x1 = box23550
    t = tuned_term(s, deterministic)
    t.build(torch.tensor(s["positions"], device=cuda), s["box"])
    for x in (s["positions"], x1):  # the lists of the build serve both
        xd = torch.tensor(x, device=cuda)
        t.prune(xd, s["box"])
        f = t.force(xd, energy=True).cpu().numpy()
        e = t.energies()
        c = t.constants()
        ref = O.evaluate(s, x)
        assert rms_rel(f, ref["forces"]) < FORCE_RMS_TOL
        scale = sum(abs(v) for v in ref["terms"].values())
        for name in ("lj", "coulomb", "excluded", "reciprocal"):
            assert abs(e[name] - ref["terms"][name]) <= ENERGY_TOL * scale, (name, e[name], ref["terms"][name])
        assert c["self"] == pytest.approx(ref["terms"]["self"], rel=1e-12)
        W = e["virial_pair"] + e["virial_reciprocal"] + np.eye(3) * c["background"]
        np.testing.assert_allclose(W, ref["virial"], rtol=1e-5, atol=1e-5 * np.abs(ref["virial"]).max())
    t.close()


def _program(s, deterministic, tau):
    system = mdir.System.from_dict(s)
    system.pairlist_distance = REACH
    system.pruned_distance = PRUNED
    v = systems.maxwell_velocities(s, 300.0, seed=2)
    state = mdir.InitialState(s["positions"], v, s["box"])
    integ, ens, exe, sch = mdir.Integrator(), mdir.Ensemble(), mdir.Execution(), mdir.Schedule()
    ens.kind = mdir.EnsembleKind.NVT if tau else mdir.EnsembleKind.NVE
    ens.tau_t, ens.seed = tau or 0.1, 5
    exe.deterministic = deterministic
    exe.graph_steps = 10
    return mdir.compile(system, state, integ, ens, exe, sch), v


@pytest.mark.parametrize("tau", [0.0, 0.1])
def test_simulation_run_is_the_integrator_run_bitwise(cuda, tau):
    s = systems.tip3p(waters=1500, seed=31)
    program, v0 = _program(s, deterministic=True, tau=tau)
    sim = mdir.Simulation(program)
    sim.run(40)
    # the state read back and written again (a checkpoint-restart loop, as
    # the bench's e2e leg runs): the lists are kept and the run goes on as
    # one run would
    mid = sim.state()
    sim.set_state(mid.positions, mid.velocities)
    sim.run(35)
    got = sim.state()
    assert got.step == 75
    # the same run through the integrator directly
    t = tuned_term(s, deterministic=True)
    md = Integrator(t, s["masses"], s["waters"])
    md.thermostat(300.0, tau, 5)
    x = torch.tensor(s["positions"], device=cuda)
    v = torch.tensor(v0, device=cuda)
    md.build(x, s["box"])
    md.run(x, v, s["box"], 0.002, 40, unroll=10)
    md.run(x, v, s["box"], 0.002, 35, unroll=10)
    np.testing.assert_array_equal(got.positions, x.cpu().numpy())
    np.testing.assert_array_equal(got.velocities, v.cpu().numpy())
    # the energies of the public API are the term's and the constants'
    e = sim.energies()
    ref = O.evaluate(s, got.positions)
    scale = sum(abs(v) for v in ref["terms"].values())
    assert abs(e["potential"] - ref["energy"]) <= 4 * ENERGY_TOL * scale
    sim.set_state(s["positions"], v0)  # from host arrays; the lists are rebuilt
    sim.run(10)
    assert np.all(np.isfinite(sim.state().positions))


def test_simulation_reports_positions_that_are_not_numbers(cuda):
    s = systems.tip3p(waters=300, seed=32)
    program, v0 = _program(s, deterministic=False, tau=0.1)
    sim = mdir.Simulation(program)
    x = s["positions"].copy()
    x[5, 2] = np.nan
    sim.set_state(x, v0)
    with pytest.raises(mdir.SimulationError):
        sim.run(10)


def test_the_256_frame_batch_frame_by_frame(cuda):
    frames = systems.batch_frames(count=256)  # the benchmark's batch: 1.18 M atoms, 8 grid shapes
    sizes = [len(f["charges"]) for f in frames]
    assert min(sizes) >= 1000 and max(sizes) <= 8000 and len(set(map(tuple, (f["grid"] for f in frames)))) > 1
    ev = BatchEvaluator(frames)
    F = ev.force(energy=True).cpu().numpy()
    E = ev.energies()
    worst = 0.0
    for k, fr in enumerate(frames):
        ref = O.evaluate(fr, fr["positions"])
        err = rms_rel(ev.frame(k, F), ref["forces"])
        worst = max(worst, err)
        assert err < FRAME_FORCE_RMS_TOL, (k, sizes[k], err)
        scale = sum(abs(v) for v in ref["terms"].values())
        for name in TERMS:
            assert abs(E[name][k] - ref["terms"][name]) <= FRAME_ENERGY_TOL * scale, (k, name)
    # the graph replay of the autotuned shape gives the same forces
    ev.autotune()
    F2 = ev.force(energy=True, graph=True).cpu().numpy()
    assert rms_rel(F2, F) < 1e-6
    ev.close()


@pytest.mark.parametrize("x_kind", ["start", "moved"])
def test_tuned_reaches_leave_the_pairs_and_forces_unchanged(cuda, box23550, x_kind):
    """Every (outer reach, pruned reach) the step autotuner tries (Integrator.
    tune's candidates, MDIR's skins search D281) gives the same pairs within
    the cutoff, and forces and energies equal to the FP64 oracle's: the
    reaches change the work, never the result."""
    s, x1 = box23550
    x = s["positions"] if x_kind == "start" else x1
    ref = O.evaluate(s, x)
    scale = sum(abs(v) for v in ref["terms"].values())
    rc = s["cutoff"]
    within = None
    forces = []
    for R, Rin in ((1.3, 1.025), (1.5, 1.05), (1.7, 1.025), (1.7, 1.05), (1.0, 0.0)):
        t = NonbondedTerm(len(s["charges"]))
        t.set_particles(s["charges"], s["types"], s["sigma"], s["epsilon"])
        t.set_exclusions(pairs=s["excluded_pairs"])
        t.set_interaction(rc, R, s["beta"])
        t.set_pruned_reach(Rin)
        t.set_pme(s["grid"], s["order"])
        t.build(torch.tensor(s["positions"], device=cuda), s["box"])
        xd = torch.tensor(x, device=cuda)
        if Rin:
            t.prune(xd, s["box"])
        f = t.force(xd, energy=True).cpu().numpy()
        e = t.energies()
        assert rms_rel(f, ref["forces"]) < FORCE_RMS_TOL, (R, Rin)
        for name in ("lj", "coulomb"):
            assert abs(e[name] - ref["terms"][name]) <= ENERGY_TOL * scale, (R, Rin, name)
        forces.append(f)
        # the pairs of the build's lists within the cutoff (at the build's positions)
        if x_kind == "start":
            p = t.pair_set(t.build(torch.tensor(s["positions"], device=cuda), s["box"]))
            xs = s["positions"]
            d = xs[p[:, 1]] - xs[p[:, 0]]
            d -= s["box"] * np.round(d / s["box"])
            inside = canon(p[np.sum(d * d, 1) < rc * rc])
            if within is None:
                within = inside
            else:
                np.testing.assert_array_equal(inside, within)
        t.close()
    for f in forces[1:]:
        assert rms_rel(f, forces[0]) < 1e-6
