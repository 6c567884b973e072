"""MDIR's Python interface for the nonbonded + PME path, over the device
library: `compile(system, state, integrator, ensemble, execution, schedule)`
returns a `Program`, `Simulation(program)` runs it, and
`FrameEvaluator(program).evaluate(frames)` gives energies and gradients of
stored frames.

Names, argument meaning and errors follow MDIR (python/Bindings.cpp:951
compile, 1625 Simulation, 2230 run; python/mdir/_frames.py:458, 715;
docs/python-compile.md): snake-case properties on plain objects, typed
enums, InputError / UnsupportedError / CompileError / SimulationError.  The
supported subset is the one this library implements: orthorhombic cells,
Lennard-Jones from a type table (optionally with the r^2 switch), Ewald
direct + PME or no electrostatics, rigid three-site waters, NVE or NVT
(Bussi), mixed precision with an optional deterministic mode.  Units: nm,
ps, kJ/mol, e, K."""

import enum

import numpy as np
import torch

from . import _lib as L
from .md import Integrator as _Integrator
from .systems import ewald_beta, pme_grid
from .term import COULOMB, NonbondedTerm, _dp, _hp


class InputError(ValueError):
    """Invalid inputs (MDIR: mdir.InputError)."""


class UnsupportedError(RuntimeError):
    """A request outside the supported subset (MDIR: mdir.UnsupportedError)."""


class CompileError(RuntimeError):
    """A program that cannot be set up (MDIR: mdir.CompileError)."""


class SimulationError(RuntimeError):
    """A run that stopped (MDIR: mdir.SimulationError, from stopWith)."""


class Target(enum.Enum):
    CPU = "CPU"
    GPU = "GPU"


class Precision(enum.Enum):
    MIXED = "MIXED"
    DOUBLE = "DOUBLE"


class EnsembleKind(enum.Enum):
    NVE = "NVE"
    NVT = "NVT"


class Electrostatics(enum.Enum):
    NONE = "NONE"
    PME = "PME"


class Truncation(enum.Enum):
    NONE = "NONE"
    SWITCH = "SWITCH"  # the cubic switch of the LJ potential in r^2 from switch_distance
    POTENTIAL_SWITCH = "POTENTIAL_SWITCH"  # the quintic switch in r of MDIR's md dialect


_SWITCH_FORM = {Truncation.NONE: 0, Truncation.SWITCH: 1, Truncation.POTENTIAL_SWITCH: 2}


class System:
    """The model: topology tables and the nonbonded settings.

    `from_dict` takes a dict of mdir_b200.systems (charges, types, sigma,
    epsilon tables, excluded_pairs, masses, waters, box)."""

    def __init__(self, charges, types, sigma, epsilon, masses, excluded_pairs=(), waters=None):
        self.charges = np.asarray(charges, dtype=np.float64)
        self.types = np.asarray(types, dtype=np.int32)
        self.sigma = np.asarray(sigma, dtype=np.float64)
        self.epsilon = np.asarray(epsilon, dtype=np.float64)
        self.masses = np.asarray(masses, dtype=np.float64)
        self.excluded_pairs = np.asarray(excluded_pairs, dtype=np.int64).reshape(-1, 2)
        self.water_residues = None if waters is None else np.asarray(waters, dtype=np.int32).reshape(-1, 3)
        self.periodic = True
        self.cutoff = 1.0
        self.pairlist_distance = 1.1
        self.pruned_distance = 0.0  # the dual list's inner reach (D114); 0: one list
        self.switch_distance = 0.0
        self.truncation = Truncation.NONE
        self.electrostatics = Electrostatics.PME
        self.dispersion = False
        self.pme_alpha = 0.0  # beta in nm^-1; 0: from pme_tolerance
        self.pme_tolerance = 1e-5
        self.pme_spacing = 0.1
        self.pme_grid = (0, 0, 0)
        self.pme_order = 4
        self.rigid_water = waters is not None

    @property
    def particle_count(self):
        return len(self.charges)

    @classmethod
    def from_dict(cls, d):
        s = cls(d["charges"], d["types"], d["sigma"], d["epsilon"], d["masses"], d["excluded_pairs"],
                d.get("waters"))
        s.cutoff = d["cutoff"]
        s.pairlist_distance = d["reach"]
        s.electrostatics = Electrostatics.PME if d["pme"] else Electrostatics.NONE
        s.dispersion = bool(d.get("dispersion", False))
        if d["pme"]:
            s.pme_alpha = d["beta"]
            s.pme_grid = tuple(d["grid"])
            s.pme_order = d["order"]
        if d.get("lj_switch"):
            s.truncation = Truncation.POTENTIAL_SWITCH if d["lj_switch"] == 2 else Truncation.SWITCH
            s.switch_distance = d["switch"]
        return s


class InitialState:
    def __init__(self, positions, velocities=None, cell=None):
        self.positions = np.asarray(positions, dtype=np.float64)
        self.velocities = (np.zeros((0, 3)) if velocities is None else np.asarray(velocities, dtype=np.float64))
        self.cell = None if cell is None else np.asarray(cell, dtype=np.float64)


class Integrator:
    """method: "LEAP_FROG" or "VELOCITY_VERLET" (MDIR's integrators,
    docs/dynamics.md); velocity Verlet keeps the velocities on the step and
    takes no rigid waters."""

    def __init__(self):
        self.method = "LEAP_FROG"
        self.timestep = 0.002


class Ensemble:
    def __init__(self):
        self.kind = EnsembleKind.NVE
        self.temperature = 300.0
        self.thermostat = "BUSSI"
        self.tau_t = 0.1
        self.seed = 1


class Execution:
    def __init__(self):
        self.target = Target.GPU
        self.precision = Precision.MIXED
        self.device = 0
        self.deterministic = False
        self.step_graph = True
        self.graph_steps = 10
        self.pair_sms = 0  # SMs the pair kernel spans (0: all); the others are left to PME
        self.pair_blocks_per_sm = 0  # blocks of the pair kernel an SM (0: the library's default, 4)
        self.fused_prune = 0  # the pruning inside the pair kernel: 0 by group count, 1 always, 2 never
        self.staging_depth = 1  # the pair kernel's staging depth (1 or 2)
        self.pme_fft = "own"  # the PME transforms: "own" (three kernels where the grid allows) or "cufft"


class Schedule:
    def __init__(self):
        self.steps = 0
        self.energy_period = 0


class Program:
    """A validated, immutable plan (MDIR: mdir.Program with `plan`)."""

    def __init__(self, system, state, integrator, ensemble, execution, schedule, plan):
        self.system, self.state, self.integrator = system, state, integrator
        self.ensemble, self.execution, self.schedule = ensemble, execution, schedule
        self.plan = dict(plan)


def compile(system, state, integrator, ensemble, execution, schedule):
    """Validates the inputs and fixes the plan of the run (MDIR
    python/Bindings.cpp:951): beta by bisection of erfc(beta r_c) = tol, the
    PME grid as the smallest even 2,3,5,7-smooth size per edge
    (lib/Driver/TermNonbonded.cpp:755-838, 1104-1130)."""
    n = system.particle_count
    x = state.positions
    if x.shape != (n, 3):
        raise InputError(f"positions: expected shape ({n}, 3); found {x.shape}")
    if not np.all(np.isfinite(x)):
        raise InputError("positions: not finite")
    if state.velocities.shape not in ((0, 3), (n, 3)):
        raise InputError(f"velocities: expected shape ({n}, 3) or (0, 3)")
    if state.cell is None or np.shape(state.cell) != (3,):
        raise UnsupportedError("an orthorhombic cell of three edges is required (triclinic cells are not supported)")
    box = np.asarray(state.cell, dtype=np.float64)
    if execution.target != Target.GPU:
        raise UnsupportedError("this library runs the GPU target only")
    if execution.precision != Precision.MIXED:
        raise UnsupportedError("precision: MIXED (f32 pairs, f64 sums; deterministic=True for fixed point)")
    if system.sigma.shape != system.epsilon.shape or system.sigma.ndim != 2:
        raise InputError("sigma and epsilon are type x type tables")
    if system.types.min(initial=0) < 0 or system.types.max(initial=0) >= system.sigma.shape[0]:
        raise InputError("a type out of the range of the tables")
    rc, R = float(system.cutoff), float(system.pairlist_distance)
    if not (0 < rc <= R):
        raise InputError("cutoff must be positive and at most pairlist_distance")
    if R >= 0.999 * box.min() or 2 * rc > box.min():
        raise InputError("pairlist_distance must be below 0.999 of the least edge and the cutoff at most half of it")
    if np.any(np.abs(system.charges) >= 100.0):
        raise InputError("particle mesh Ewald holds charges of less than 100 e")
    Rin = float(system.pruned_distance or 0.0)
    if Rin and not (rc <= Rin <= R):
        raise InputError("pruned_distance must lie between the cutoff and pairlist_distance")
    plan = {"particles": n, "cutoff": rc, "reach": R, "pruned_reach": Rin, "box": box.tolist(),
            "device": execution.device}
    if system.electrostatics == Electrostatics.PME:
        beta = system.pme_alpha or ewald_beta(rc, system.pme_tolerance)
        auto = pme_grid(box, system.pme_spacing, system.pme_order)
        grid = [max(int(g), 2 * system.pme_order) if g else a for g, a in zip(system.pme_grid, auto)]
        if system.pme_order not in (4, 5, 6, 8):
            raise UnsupportedError("pme_order: 4, 5, 6 or 8")
        plan.update({"beta": beta, "pme_grid": grid, "pme_order": system.pme_order})
    else:
        plan.update({"beta": 0.0, "pme_grid": None})
    if ensemble.kind not in (EnsembleKind.NVE, EnsembleKind.NVT):
        raise UnsupportedError("ensembles: NVE and NVT")
    if not integrator.timestep > 0:
        raise InputError("timestep must be positive")
    method = str(integrator.method).upper()
    if method not in ("LEAP_FROG", "VELOCITY_VERLET"):
        raise UnsupportedError("integrators: LEAP_FROG and VELOCITY_VERLET")
    if method == "VELOCITY_VERLET" and system.rigid_water and system.water_residues is not None:
        raise UnsupportedError("VELOCITY_VERLET with rigid waters needs velocity constraints; use LEAP_FROG")
    if getattr(execution, "pme_fft", "own") not in ("own", "cufft"):
        raise InputError("pme_fft: \"own\" or \"cufft\"")
    plan["waters"] = 0 if system.water_residues is None else len(system.water_residues)
    return Program(system, state, integrator, ensemble, execution, schedule, plan)


class State:
    def __init__(self, positions, velocities, step):
        self.positions, self.velocities, self.step = positions, velocities, step


def _make_term(program):
    s, p = program.system, program.plan
    t = NonbondedTerm(s.particle_count, device=program.execution.device)
    t.set_particles(s.charges, s.types, s.sigma, s.epsilon)
    t.set_exclusions(pairs=s.excluded_pairs)
    t.set_interaction(p["cutoff"], p["reach"], p["beta"], coulomb=COULOMB,
                      lj_switch=_SWITCH_FORM[s.truncation], switch_distance=s.switch_distance)
    if p["pme_grid"]:
        t.set_pme(p["pme_grid"], p["pme_order"])
    t.set_deterministic(program.execution.deterministic)
    if p["pruned_reach"]:
        t.set_pruned_reach(p["pruned_reach"])
    if program.execution.pair_sms:
        t.set_tuning(pair_sms=program.execution.pair_sms)
    if program.execution.pair_blocks_per_sm:
        t.set_tuning(pair_blocks_per_sm=program.execution.pair_blocks_per_sm)
    if getattr(program.execution, "fused_prune", 0):
        t.set_tuning(fused_prune=program.execution.fused_prune)
    if getattr(program.execution, "staging_depth", 1) != 1:
        t.set_tuning(staging_depth=program.execution.staging_depth)
    if getattr(program.execution, "pme_fft", "own") != "own":
        t.set_tuning(pme_fft=program.execution.pme_fft)
    return t


class Simulation:
    """A persistent run of a program on its device (MDIR:
    python/Bindings.cpp:1625 and lib/Compiler/Simulation.cpp:1679)."""

    def __init__(self, program):
        self.program = program
        s, p = program.system, program.plan
        self.device = torch.device("cuda", program.execution.device)
        self.term = _make_term(program)
        self.box = np.asarray(p["box"])
        self.md = _Integrator(self.term, s.masses, s.water_residues if s.rigid_water else None)
        e = program.ensemble
        self.md.thermostat(e.temperature, e.tau_t if e.kind == EnsembleKind.NVT else 0.0, e.seed)
        self.md.method(str(program.integrator.method))
        st = program.state
        self.x = torch.tensor(st.positions, dtype=torch.float64, device=self.device)
        v = st.velocities if len(st.velocities) else np.zeros_like(st.positions)
        self.v = torch.tensor(v, dtype=torch.float64, device=self.device)
        self.step = 0
        self._build()

    def _build(self):
        try:
            self.md.build(self.x, self.box)
        except L.NativeError as e:
            if e.status == L.NAN_POSITION:
                raise SimulationError("positions that are not numbers or are far outside the cell") from e
            raise

    def tune(self, **kw):
        """Times short runs over outer and pruned reaches and spans of the
        pair grid and keeps the fastest (Integrator.tune; MDIR's skins
        search, D281); the state is put back.  Returns the choice."""
        return self.md.tune(self.x, self.v, self.box, self.program.integrator.timestep, **kw)

    def set_state(self, positions, velocities=None, non_blocking=False):
        """New positions (and velocities) from host or device arrays.  The
        next run keeps the lists when the new positions lie within half the
        skin of their build, and builds otherwise (mdrtMdRefresh)."""
        self.x.copy_(torch.as_tensor(positions), non_blocking=non_blocking)
        if velocities is not None:
            self.v.copy_(torch.as_tensor(velocities), non_blocking=non_blocking)
        self._stale = True

    def run(self, steps):
        if steps < 0:
            raise InputError("steps must be nonnegative")
        if getattr(self, "_stale", False):
            try:
                self.md.refresh(self.x, self.box)
            except L.NativeError as e:
                if e.status == L.NAN_POSITION:
                    raise SimulationError("positions that are not numbers or are far outside the cell") from e
                raise
            self._stale = False
        ex = self.program.execution
        unroll = ex.graph_steps if ex.step_graph else 0
        self.md.run(self.x, self.v, self.box, self.program.integrator.timestep, steps, unroll=unroll)
        self.step += steps
        status = self.term.status(clear=True)
        if status & 1:
            raise SimulationError("the lists overflowed their room during the run; rebuild with more room")
        if status & 4:
            raise SimulationError("positions that are not numbers or are far outside the cell")

    def state(self):
        return State(self.x.cpu().numpy(), self.v.cpu().numpy(), self.step)

    def energies(self):
        """The potential energy terms (kJ/mol) at the current positions and
        the kinetic energy of leap-frog, the mean of the last two half steps
        (centred one step behind the positions; `Integrator.total_energy`
        pairs them at the same time, by one more step)."""
        f = self.term.force(self.x, self.box, energy=True)
        e = self.term.energies()
        c = self.term.constants(self.box, dispersion=self.program.system.dispersion)
        terms = {"lj": e["lj"], "coulomb": e["coulomb"], "excluded": e["excluded"],
                 "reciprocal": e["reciprocal"], "self": c["self"], "background": c["background"],
                 "dispersion": c["dispersion"]}
        terms["potential"] = sum(terms.values())
        t = self.md.thermo()
        terms["kinetic"] = t["kinetic"]
        del f
        return terms
