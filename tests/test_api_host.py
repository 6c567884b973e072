"""The host side of the public API, without a GPU: the Ewald beta and the
PME grid the product plans with (mdir_b200.systems, used by compile())
equal the oracle's restatement of MDIR's (lib/Driver/TermNonbonded.cpp:
755-838, 1104-1130), and compile() refuses what MDIR's compile refuses
(python/Bindings.cpp:951; InputError / UnsupportedError)."""
import math

import numpy as np
import pytest

from oracle import oracle as O
import mdir_b200 as mdir
from mdir_b200 import systems


@pytest.mark.parametrize("rc,tol", [(0.9, 1e-5), (1.0, 1e-5), (0.8, 1e-6), (1.2, 5e-4), (0.9, 1e-8)])
def test_beta_is_the_oracles(rc, tol):
    beta = systems.ewald_beta(rc, tol)
    assert beta == O.ewald_beta(rc, tol)
    assert math.erfc(beta * rc) == pytest.approx(tol, rel=1e-9)


def test_grids_of_every_workload_are_the_oracles():
    # the water box, the large box, the 256 batch frames' cells, and
    # edges just above and below a smooth size
    edges = [(7850 / 33.4) ** (1 / 3), 22.008, 6.4, 6.4000001, 6.3999999, 1.3, 3.47]
    edges += [(a / 100.2) ** (1 / 3) for a in range(1002, 8001, 333)]
    for L in edges:
        for order in (4, 5, 6, 8):
            for spacing in (0.1, 0.12):
                assert systems.pme_grid([L] * 3, spacing, order) == O.pme_grid([L] * 3, spacing, order), (L, order)
    assert systems.pme_grid([(7850 / 33.4) ** (1 / 3)] * 3) == [64, 64, 64]
    assert systems.pme_grid([22.008] * 3) == [224, 224, 224]


def _program_inputs(waters=300, **over):
    s = systems.tip3p(waters=waters, seed=2)
    s = dict(s, **over)
    system = mdir.System.from_dict(s)
    state = mdir.InitialState(s["positions"], None, s["box"])
    return s, system, state, mdir.Integrator(), mdir.Ensemble(), mdir.Execution(), mdir.Schedule()


def test_compile_plans_the_oracles_beta_and_grid():
    s, system, state, integ, ens, exe, sch = _program_inputs(waters=7850)
    system.pme_alpha = 0.0  # from the tolerance
    system.pme_grid = (0, 0, 0)  # from the spacing
    p = mdir.compile(system, state, integ, ens, exe, sch).plan
    assert p["beta"] == O.ewald_beta(s["cutoff"], 1e-5)
    assert p["pme_grid"] == O.pme_grid(s["box"], 0.1, 4) == [64, 64, 64]
    # a given grid below 2 * order is raised to it, as MDIR does
    system.pme_grid = (4, 64, 64)
    assert mdir.compile(system, state, integ, ens, exe, sch).plan["pme_grid"] == [8, 64, 64]


def test_compile_refuses_bad_inputs():
    s, system, state, integ, ens, exe, sch = _program_inputs()
    n = system.particle_count
    bad = mdir.InitialState(s["positions"][:-1], None, s["box"])
    with pytest.raises(mdir.InputError):
        mdir.compile(system, bad, integ, ens, exe, sch)
    x = s["positions"].copy()
    x[3, 1] = np.nan
    with pytest.raises(mdir.InputError):
        mdir.compile(system, mdir.InitialState(x, None, s["box"]), integ, ens, exe, sch)
    with pytest.raises(mdir.InputError):
        mdir.compile(system, mdir.InitialState(s["positions"], np.zeros((n - 1, 3)), s["box"]), integ, ens,
                     exe, sch)
    # a reach at 0.999 of the least edge or more, and a cutoff above half of it
    system.pairlist_distance = 0.999 * s["box"][0]
    with pytest.raises(mdir.InputError):
        mdir.compile(system, state, integ, ens, exe, sch)
    system.pairlist_distance = s["reach"]
    system.cutoff = 2 * s["reach"]
    with pytest.raises(mdir.InputError):
        mdir.compile(system, state, integ, ens, exe, sch)
    system.cutoff = s["cutoff"]
    system.pruned_distance = 0.5 * s["cutoff"]
    with pytest.raises(mdir.InputError):
        mdir.compile(system, state, integ, ens, exe, sch)
    system.pruned_distance = 0.0
    integ.timestep = 0.0
    with pytest.raises(mdir.InputError):
        mdir.compile(system, state, integ, ens, exe, sch)
    integ.timestep = 0.002
    system.types = system.types.copy()
    system.types[0] = system.sigma.shape[0]
    with pytest.raises(mdir.InputError):
        mdir.compile(system, state, integ, ens, exe, sch)
    system.types[0] = 0
    # the PME transforms: the library's own kernels or cuFFT
    exe.pme_fft = "vkfft"
    with pytest.raises(mdir.InputError):
        mdir.compile(system, state, integ, ens, exe, sch)
    exe.pme_fft = "cufft"
    mdir.compile(system, state, integ, ens, exe, sch)
    # the program is fine again once the inputs are
    exe.pme_fft = "own"
    mdir.compile(system, state, integ, ens, exe, sch)


def test_compile_refuses_what_the_library_does_not_offer():
    s, system, state, integ, ens, exe, sch = _program_inputs()
    tric = mdir.InitialState(s["positions"], None, np.r_[s["box"], 0.1, 0.0, 0.0])
    with pytest.raises(mdir.UnsupportedError):
        mdir.compile(system, tric, integ, ens, exe, sch)
    exe.target = mdir.Target.CPU
    with pytest.raises(mdir.UnsupportedError):
        mdir.compile(system, state, integ, ens, exe, sch)
    exe.target = mdir.Target.GPU
    exe.precision = mdir.Precision.DOUBLE
    with pytest.raises(mdir.UnsupportedError):
        mdir.compile(system, state, integ, ens, exe, sch)
    exe.precision = mdir.Precision.MIXED
    system.pme_order = 7
    with pytest.raises(mdir.UnsupportedError):
        mdir.compile(system, state, integ, ens, exe, sch)
    system.pme_order = 4
    ens.kind = "NPT"
    with pytest.raises(mdir.UnsupportedError):
        mdir.compile(system, state, integ, ens, exe, sch)


def test_compile_takes_the_integrators_mdir_names():
    s, system, state, integ, ens, exe, sch = _program_inputs()
    integ.method = "VELOCITY_VERLET"  # rigid waters need velocity constraints
    with pytest.raises(mdir.UnsupportedError):
        mdir.compile(system, state, integ, ens, exe, sch)
    integ.method = "BROWNIAN"
    with pytest.raises(mdir.UnsupportedError):
        mdir.compile(system, state, integ, ens, exe, sch)
    a = systems.argon()
    argon = mdir.System.from_dict(a)
    integ.method = "VELOCITY_VERLET"
    p = mdir.compile(argon, mdir.InitialState(a["positions"], None, a["box"]), integ, ens, exe, sch)
    assert p.plan["waters"] == 0
