"""The MD step on the device: SETTLE, the CUDA-graph replay with
conditional rebuilds, energy conservation and the thermostat."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from mdir_b200 import NonbondedTerm, systems
from mdir_b200.md import Integrator

pytestmark = pytest.mark.gpu


def setup(s, deterministic=False, tau=0.0, seed=1):
    n = len(s["charges"])
    t = NonbondedTerm(n)
    t.set_particles(s["charges"], s["types"], s["sigma"], s["epsilon"])
    t.set_exclusions(pairs=s["excluded_pairs"])
    t.set_interaction(s["cutoff"], s["reach"], s["beta"])
    t.set_pme(s["grid"], s["order"])
    t.set_deterministic(deterministic)
    md = Integrator(t, s["masses"], s["waters"])
    md.thermostat(300.0, tau, seed)
    x = torch.tensor(s["positions"], dtype=torch.float64, device="cuda")
    v = torch.tensor(systems.maxwell_velocities(s, 300.0, seed=2), device="cuda")
    md.build(x, s["box"])
    return t, md, x, v


def water_geometry(x, waters):
    x = x.cpu().numpy()
    o, h1, h2 = x[waters[:, 0]], x[waters[:, 1]], x[waters[:, 2]]
    return (np.linalg.norm(h1 - o, axis=1), np.linalg.norm(h2 - o, axis=1), np.linalg.norm(h2 - h1, axis=1))


def test_settle_keeps_waters_rigid(cuda):
    s = systems.tip3p(waters=600, seed=21)
    t, md, x, v = setup(s)
    md.run(x, v, s["box"], 0.002, 50, unroll=10)
    d1, d2, d3 = water_geometry(x, s["waters"])
    dhh = 2 * 0.09572 * np.sin(np.radians(104.52) / 2)
    assert np.abs(d1 - 0.09572).max() < 1e-9
    assert np.abs(d2 - 0.09572).max() < 1e-9
    assert np.abs(d3 - dhh).max() < 1e-9


def test_graph_replay_equals_step_by_step_bitwise(cuda):
    s = systems.tip3p(waters=500, seed=22)
    t1, md1, x1, v1 = setup(s, deterministic=True, tau=0.1)
    md1.run(x1, v1, s["box"], 0.002, 60, unroll=10)
    t2, md2, x2, v2 = setup(s, deterministic=True, tau=0.1)
    md2.run(x2, v2, s["box"], 0.002, 60, unroll=0)
    assert md1.thermo()["builds"] == md2.thermo()["builds"]
    assert torch.equal(x1, x2) and torch.equal(v1, v2)


def test_lists_stay_valid_across_device_rebuilds(cuda):
    s = systems.tip3p(waters=700, seed=23)
    t, md, x, v = setup(s, tau=0.1)
    md.run(x, v, s["box"], 0.002, 400, unroll=20)
    th = md.thermo()
    assert th["builds"] >= 2  # the test of validity asked for rebuilds on the device
    assert t.status() == 0
    f = t.force(x, energy=True).cpu().numpy()
    ref = O.evaluate(s, x.cpu().numpy())
    err = np.sqrt(np.mean(np.sum((f - ref["forces"]) ** 2, 1)) / np.mean(np.sum(ref["forces"] ** 2, 1)))
    assert err < 1e-5


def test_nve_energy_is_conserved(cuda):
    """600 waters brought to 300 K by a strong thermostat, then NVE at 1 fs:
    the total energy (the potential and the kinetic energy at the same time)
    fluctuates by about 1e-4 of the kinetic energy and does not drift."""
    s = systems.tip3p(waters=600, seed=24)
    t, md, x, v = setup(s, tau=0.02)
    md.run(x, v, s["box"], 0.001, 2000, unroll=10)
    md.thermostat(300.0, 0.0, 1)
    samples = []
    for _ in range(20):
        md.run(x, v, s["box"], 0.001, 50, unroll=10)
        samples.append(md.total_energy(x, v, s["box"], 0.001))
    E = np.array(samples)
    kin = E[:, 2].mean()
    slope = np.polyfit(np.arange(len(E)) * 0.051, E[:, 0], 1)[0]  # kJ/mol/ps
    assert E[:, 0].std() < 3e-4 * kin, (E[:, 0].std(), kin)
    assert abs(slope * 1.0) < 3e-4 * kin, (slope, kin)


def test_dual_list_keeps_every_pair_within_the_cutoff(cuda):
    # outer lists at 1.2 nm rebuilt rarely, inner lists pruned to 1.0 nm on
    # the device whenever the positions moved half of the inner skin
    s = systems.tip3p(waters=700, seed=26)
    s["reach"] = 1.2
    t, md, x, v = setup(s, tau=0.1)
    t.set_pruned_reach(1.0)
    md.build(x, s["box"])
    md.run(x, v, s["box"], 0.002, 400, unroll=20)
    th = md.thermo()
    assert th["prunes"] > th["builds"] >= 1
    assert t.status() == 0
    ref = O.evaluate(s, x.cpu().numpy())
    f = md.forces()
    # the forces of the next evaluation at these positions, over the inner lists
    got = t.force(x, energy=True).cpu().numpy()
    err = np.sqrt(np.mean(np.sum((got - ref["forces"]) ** 2, 1)) / np.mean(np.sum(ref["forces"] ** 2, 1)))
    assert err < 1e-5
    e = t.energies()
    assert abs(e["coulomb"] - ref["terms"]["coulomb"]) < 1e-6 * sum(abs(v) for v in ref["terms"].values())
    del f


def test_dual_list_step_by_step_equals_graph(cuda):
    s = systems.tip3p(waters=500, seed=27)
    s["reach"] = 1.15
    runs = []
    for unroll in (10, 0):
        t, md, x, v = setup(s, deterministic=True, tau=0.1)
        t.set_pruned_reach(1.0)
        md.build(x, s["box"])
        md.run(x, v, s["box"], 0.002, 80, unroll=unroll)
        runs.append((x.clone(), md.thermo()))
    assert torch.equal(runs[0][0], runs[1][0])
    assert runs[0][1]["prunes"] == runs[1][1]["prunes"] > 0


def test_thermostat_holds_the_temperature(cuda):
    s = systems.tip3p(waters=500, seed=25)
    t, md, x, v = setup(s, tau=0.05)
    md.run(x, v, s["box"], 0.002, 1500, unroll=10)
    temps = []
    for _ in range(10):
        md.run(x, v, s["box"], 0.002, 50, unroll=10)
        temps.append(md.temperature())
    assert abs(np.mean(temps) - 300.0) < 15.0, temps


def test_lists_that_outgrow_their_capacity_inside_the_graphs_are_redone(cuda):
    """Argon as a dilute gas (5 nm^-3) with every atom moving toward the
    centre: the swarm compresses, the lists outgrow the capacity sized at
    the first build, and a rebuild inside the step graphs overflows.  The
    run goes back to its checkpoint with grown lists; the result is the
    step-by-step run's, bit for bit (deterministic mode)."""
    s = systems.argon(length=5.57, skin=0.4)  # a wide skin: no stops at stale lists
    L = s["box"][0]
    v0 = -1.5 * (s["positions"] - 0.5 * L)

    def run(unroll):
        n = len(s["charges"])
        t = NonbondedTerm(n)
        t.set_particles(s["charges"], s["types"], s["sigma"], s["epsilon"])
        t.set_interaction(s["cutoff"], s["reach"], 0.0)
        t.set_deterministic(True)
        md = Integrator(t, s["masses"], None)
        md.thermostat(120.0, 0.0, 1)
        md.lookahead(100.0)  # a rebuild at the end of every window: the growth comes inside the graphs
        x = torch.tensor(s["positions"], dtype=torch.float64, device="cuda")
        v = torch.tensor(v0, dtype=torch.float64, device="cuda")
        md.build(x, s["box"])
        cap0 = t.info()["list_capacity"]
        md.run(x, v, s["box"], 0.002, 150, unroll=unroll)
        return t, md, x, v, cap0

    t1, md1, x1, v1, cap0 = run(5)
    th = md1.thermo()
    assert th["regrows"] >= 1
    assert t1.info()["list_capacity"] > cap0
    assert t1.status() & 1 == 0  # no overflow left behind
    t2, md2, x2, v2, _ = run(-5)
    assert md2.thermo()["builds"] == th["builds"]
    assert torch.equal(x1, x2) and torch.equal(v1, v2)


def test_stops_at_a_stale_list_equal_the_host_rebuilding_at_once(cuda):
    """With no look-ahead (factor 0) the drift passes half the skin inside
    windows again and again: the graphs stop at that step and the host
    rebuilds there, which must give the step-by-step run (the host testing
    every step) bit for bit, a stale list never used."""
    s = systems.tip3p(waters=500, seed=28)
    s["reach"] = 1.0
    runs = []
    for unroll in (10, 0):
        t, md, x, v = setup(s, deterministic=True, tau=0.1)
        md.lookahead(0.0)
        md.build(x, s["box"])
        md.run(x, v, s["box"], 0.002, 200, unroll=unroll)
        runs.append((x.clone(), v.clone(), md.thermo()))
    (x1, v1, th1), (x2, v2, th2) = runs
    assert th1["redone"] > 0 and th1["redone"] == th2["redone"]
    assert th1["builds"] == th2["builds"]
    assert torch.equal(x1, x2) and torch.equal(v1, v2)


@pytest.mark.parametrize("deterministic", [False, True])
def test_forces_of_a_step_are_the_oracle_forces(cuda, deterministic):
    """The forces that a step of the graphs used (pairs over the pruned
    lists, the excluded correction inside the update, PME through the step's
    own chain and the update's gather), at the positions the step started
    from, against the FP64 oracle there."""
    import ctypes
    from mdir_b200.term import _cudart
    s = systems.tip3p(waters=700, seed=29)
    s["reach"] = 1.3
    t, md, x, v = setup(s, deterministic=deterministic, tau=0.1)
    t.set_pruned_reach(1.0)
    md.build(x, s["box"])
    md.run(x, v, s["box"], 0.002, 200, unroll=10)  # rebuilds and prunings inside the graphs
    x0 = x.cpu().numpy()
    md.run(x, v, s["box"], 0.002, 1, unroll=0)  # one step from x0
    n = len(s["charges"])
    f = np.empty((n, 3))
    torch.cuda.synchronize()
    res = _cudart().cudaMemcpy(ctypes.c_void_p(f.ctypes.data), ctypes.c_void_p(md.forces()),
                               ctypes.c_size_t(f.nbytes), 2)
    assert int(res) == 0
    ref = O.evaluate(s, x0)["forces"]
    err = np.sqrt(np.mean(np.sum((f - ref) ** 2, 1)) / np.mean(np.sum(ref ** 2, 1)))
    assert err < 1e-5, err
    assert md.thermo()["prunes"] > 0 and t.status() == 0


def test_velocity_verlet_argon_nve(cuda):
    """The liquid-argon workload (864 atoms, cutoff 1.0 nm, Maxwell
    velocities at 120 K) under velocity Verlet, NVE at 2 fs: the first 20
    steps follow an FP64 velocity-Verlet integration on the oracle's forces
    (positions and on-step velocities), and over 2,000 steps the total energy
    with on-step velocities (the dispersion correction is a constant) moves
    by a small part of its fluctuations."""
    s = systems.argon()
    n = len(s["charges"])
    t = NonbondedTerm(n)
    t.set_particles(s["charges"], s["types"], s["sigma"], s["epsilon"])
    t.set_interaction(s["cutoff"], s["reach"], 0.0)
    md = Integrator(t, s["masses"])
    md.method("velocity_verlet")
    md.thermostat(120.0, 0.0, 1)
    v0 = systems.maxwell_velocities(s, 120.0, seed=2)
    x = torch.tensor(s["positions"], dtype=torch.float64, device="cuda")
    v = torch.tensor(v0, device="cuda")
    md.build(x, s["box"])
    dt = 0.002
    md.run(x, v, s["box"], dt, 20, unroll=10)
    # the FP64 reference: velocity Verlet on the oracle's forces
    m = np.asarray(s["masses"])[:, None]
    xr, vr = s["positions"].copy(), v0.copy()
    f = O.evaluate(s, xr)["forces"]
    for _ in range(20):
        vr = vr + 0.5 * dt * f / m
        xr = xr + dt * vr
        f = O.evaluate(s, xr)["forces"]
        vr = vr + 0.5 * dt * f / m
    np.testing.assert_allclose(x.cpu().numpy(), xr, atol=1e-6)
    vd = v.cpu().numpy()
    assert np.sqrt(np.mean((vd - vr) ** 2)) < 1e-4 * np.sqrt(np.mean(vr ** 2))

    def total():
        xe = x.cpu().numpy()
        e = O.evaluate(s, xe)["energy"]
        return e + 0.5 * float(np.sum(m * v.cpu().numpy() ** 2))

    e0 = [total()]
    for _ in range(10):
        md.run(x, v, s["box"], dt, 198, unroll=-6)
        e0.append(total())
    e0 = np.array(e0)
    # the plain LJ cut makes the energy jump when pairs cross the cutoff:
    # a drift well inside a percent of the kinetic energy (about 1.3 kJ/mol
    # per atom at 120 K)
    kin = 0.5 * float(np.sum(m * v.cpu().numpy() ** 2))
    assert abs(e0[-1] - e0[0]) < 0.01 * kin
    # leap-frog from v_{-1/2} gives the same positions
    t2 = NonbondedTerm(n)
    t2.set_particles(s["charges"], s["types"], s["sigma"], s["epsilon"])
    t2.set_interaction(s["cutoff"], s["reach"], 0.0)
    md2 = Integrator(t2, s["masses"])
    md2.thermostat(120.0, 0.0, 1)
    x2 = torch.tensor(s["positions"], dtype=torch.float64, device="cuda")
    md2.build(x2, s["box"])
    f0 = O.evaluate(s, s["positions"])["forces"]
    v2 = torch.tensor(v0 - 0.5 * dt * f0 / m, device="cuda")
    md2.run(x2, v2, s["box"], dt, 20, unroll=10)
    np.testing.assert_allclose(x2.cpu().numpy(), xr, atol=1e-6)


def test_a_state_written_back_keeps_the_lists_and_the_trajectory(cuda):
    """Positions and velocities read back after a run and written again
    (a checkpoint-restart loop): mdrtMdRefresh keeps the lists, and the two
    runs give the trajectory of one run of their length bit for bit
    (deterministic mode); a state beyond half the skin builds."""
    s = systems.tip3p(waters=600, seed=51)
    t1, md1, x1, v1 = setup(s, deterministic=True, tau=0.1)
    md1.run(x1, v1, s["box"], 0.002, 200, unroll=10)
    t2, md2, x2, v2 = setup(s, deterministic=True, tau=0.1)
    md2.run(x2, v2, s["box"], 0.002, 100, unroll=10)
    hx, hv = x2.cpu(), v2.cpu()
    x2.zero_()
    v2.zero_()
    x2.copy_(hx)
    v2.copy_(hv)
    builds = md2.thermo()["builds"]
    assert md2.refresh(x2, s["box"]) is False
    assert md2.thermo()["builds"] == builds
    md2.run(x2, v2, s["box"], 0.002, 100, unroll=10)
    assert torch.equal(x1, x2) and torch.equal(v1, v2)
    assert md1.thermo()["builds"] == md2.thermo()["builds"]
    # an atom moved by more than half the skin: the lists are built again
    x2[5, 0] += 0.6 * (s["reach"] - s["cutoff"])
    assert md2.refresh(x2, s["box"]) is True
    md2.run(x2, v2, s["box"], 0.002, 20, unroll=10)
    assert t2.status() == 0
