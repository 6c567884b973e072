"""The MD step over the C ABI: leap-frog with SETTLE for rigid waters and the
Bussi thermostat, replayed as a CUDA graph whose list rebuilds are decided
on the device (mdrtMd* of include/mdrt_nb.h)."""

import ctypes

import numpy as np
import torch

from . import _lib as L
from .term import NonbondedTerm, _dp, _host, _hp, _stream

KB = 0.0083144626181532  # kJ/mol/K


class Integrator:
    """Leap-frog MD of one system on the device: `x` and `v` are device f64
    tensors (n, 3) that the integrator updates in place."""

    def __init__(self, term: NonbondedTerm, masses, waters=None, d_oh=0.09572, d_hh=None):
        self.term = term
        m = _host(masses, np.float64)
        w = np.zeros((0, 3), dtype=np.int32) if waters is None else _host(waters, np.int32).reshape(-1, 3)
        if d_hh is None:
            d_hh = 2.0 * d_oh * np.sin(np.radians(104.52) / 2.0)
        h = ctypes.c_void_p()
        L.check(L.lib().mdrtMdCreate(ctypes.byref(h), term._h, _hp(m), len(w), _hp(w) if len(w) else None,
                                     d_oh, d_hh), "mdrtMdCreate")
        self._h = h
        self.masses = m
        self.nwaters = len(w)

    def close(self):
        if getattr(self, "_h", None):
            L.lib().mdrtMdDestroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def thermostat(self, temperature, tau, seed=1):
        L.check(L.lib().mdrtMdSetThermostat(self._h, temperature, tau, seed), "mdrtMdSetThermostat")

    def method(self, name):
        """The integrator: "leap_frog" (velocities half a step behind the
        positions) or "velocity_verlet" (velocities on the step at the start
        and the end of each run; the same positions; no rigid waters)."""
        code = {"leap_frog": L.LEAP_FROG, "velocity_verlet": L.VELOCITY_VERLET}[name.lower()]
        L.check(L.lib().mdrtMdSetIntegrator(self._h, code), "mdrtMdSetIntegrator")

    def lookahead(self, factor):
        """The rebuild decision's extrapolation of the drift (default 1.5)."""
        L.check(L.lib().mdrtMdSetLookahead(self._h, float(factor)), "mdrtMdSetLookahead")

    def build(self, x, box, stream=None):
        b = _host(box, np.float64)
        self.term.box = b
        L.check(L.lib().mdrtMdBuild(self._h, _dp(x), _hp(b), _stream(stream)), "mdrtMdBuild")

    def refresh(self, x, box, stream=None):
        """Positions x written anew: keeps the lists when x lies within half
        the skin of their build (the test of every step), else builds.
        Returns True when it built."""
        b = _host(box, np.float64)
        self.term.box = b
        built = ctypes.c_int32()
        L.check(L.lib().mdrtMdRefresh(self._h, _dp(x), _hp(b), _stream(stream), ctypes.byref(built)),
                "mdrtMdRefresh")
        return bool(built.value)

    def run(self, x, v, box, dt, steps, unroll=10, stream=None):
        b = _host(box, np.float64)
        L.check(L.lib().mdrtMdRun(self._h, _dp(x), _dp(v), _hp(b), dt, int(steps), int(unroll), _stream(stream)),
                "mdrtMdRun")

    def thermo(self, stream=None):
        out = np.zeros(9)
        L.check(L.lib().mdrtMdThermo(self._h, _stream(stream), _hp(out)), "mdrtMdThermo")
        return {"lambda": out[0], "kinetic_half": out[1], "kinetic_half_before": out[2],
                "steps": int(out[3]), "builds": int(out[4]), "ndof": int(out[5]), "prunes": int(out[6]),
                "regrows": int(out[7]), "redone": int(out[8]),
                "kinetic": 0.5 * (out[1] + out[2])}

    def forces(self):
        p = ctypes.c_void_p()
        L.check(L.lib().mdrtMdForces(self._h, ctypes.byref(p)), "mdrtMdForces")
        return p.value

    def tune(self, x, v, box, dt, reaches=(1.3, 1.4, 1.5, 1.6, 1.7), pruned=(0.975, 1.0, 1.025, 1.05),
             pair_sms=(0, 112, 120, 128, 136), pair_blocks=(4, 3), depths=(1, 2), fused=(2, 1), steps=400, reps=3,
             stream=None):
        """The autotuner of the step, in four stages: the outer and pruned
        reaches first (the launch shapes as set), then the span of the pair
        grid (SMs; the others are left to the PME kernels beside it), its
        blocks per SM and its staging depth at the reaches kept, then the
        three leading pairs of reaches at each of the two leading shapes
        again, in runs twice as long and more of them (the leaders differ by
        about the noise of the short runs, and the best reaches depend on
        the shape), then the
        pruning inside the pair kernel (MDIR D284) or in a launch of its
        own.  Each choice is timed as `reps` runs of `steps` steps after a
        build and half as many untimed steps; the fastest is kept and built
        for.  x and v are put back; the step
        counter and the thermostat's noise move on.  MDIR searches its
        reaches the same way (the skins search, D281,
        lib/Compiler/Skins.cpp).  Returns the choice with its time per step
        (µs)."""
        t = self.term
        cutoff = t.interaction["cutoff"]
        least = float(np.min(np.asarray(box, dtype=np.float64)))
        keep_x, keep_v = x.clone(), v.clone()
        st = stream if stream is not None else torch.cuda.current_stream(x.device)

        def trial(R, Rin, sms, blocks, depth=None, steps=steps, reps=reps):
            t.set_reach(R)
            t.set_pruned_reach(Rin)
            t.set_tuning(pair_sms=sms, pair_blocks_per_sm=blocks, staging_depth=depth)
            x.copy_(keep_x)
            v.copy_(keep_v)
            self.build(x, box, stream=st)
            self.run(x, v, box, dt, steps // 2, unroll=10, stream=st)
            ms = []
            for _ in range(reps):
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(st)
                self.run(x, v, box, dt, steps, unroll=10, stream=st)
                b.record(st)
                b.synchronize()
                ms.append(a.elapsed_time(b) / steps)
            return float(np.median(ms)) * 1e3

        sms0 = getattr(t, "pair_sms", 0)
        blocks0 = getattr(t, "pair_blocks_per_sm", 4)
        fused0 = getattr(t, "fused_prune", 0)
        depth0 = getattr(t, "staging_depth", 1)
        trials = []
        for R in reaches:
            if not R < 0.999 * least:
                continue
            for Rin in pruned:
                if cutoff <= Rin < R:
                    trials.append((trial(R, Rin, sms0, blocks0, depth0), R, Rin, sms0, blocks0, depth0))
        _, R, Rin, _, _, _ = min(trials)
        for sms in pair_sms:
            for blocks in pair_blocks:
                for depth in depths:
                    if (sms, blocks, depth) != (sms0, blocks0, depth0):
                        trials.append((trial(R, Rin, sms, blocks, depth), R, Rin, sms, blocks, depth))
        us, R, Rin, sms, blocks, depth = min(t_ for t_ in trials if t_[1] == R and t_[2] == Rin)
        first = sorted((t_[0], t_[1], t_[2]) for t_ in trials if t_[3:] == (sms0, blocks0, depth0))
        leaders = []
        for _, R_, Rin_ in first:
            if (R_, Rin_) not in leaders:
                leaders.append((R_, Rin_))
        # the two leading shapes at the reaches kept, each with the three
        # leading reaches, in the longer runs
        shapes = []
        for t_ in sorted(t_ for t_ in trials if t_[1] == R and t_[2] == Rin):
            if t_[3:] not in shapes:
                shapes.append(t_[3:])
        final = [(trial(R_, Rin_, sh[0], sh[1], sh[2], steps=2 * steps, reps=reps + 2), R_, Rin_) + sh
                 for sh in shapes[:2] for R_, Rin_ in leaders[:3]]
        us, R, Rin, sms, blocks, depth = min(final)
        t.set_tuning(staging_depth=depth)
        # the pruning in the pair kernel (MDIR D284) or in a launch of its
        # own, at the shape kept
        fused_trials = []
        for f in fused:
            t.set_tuning(fused_prune=f)
            fused_trials.append((trial(R, Rin, sms, blocks), f))
        fus, fchoice = min(fused_trials)
        if fus < us:
            us = fus
        else:
            fchoice = fused0
        t.set_tuning(fused_prune=fchoice)
        t.set_reach(R)
        t.set_pruned_reach(Rin)
        t.set_tuning(pair_sms=sms, pair_blocks_per_sm=blocks)
        x.copy_(keep_x)
        v.copy_(keep_v)
        self.build(x, box, stream=st)
        return {"reach": R, "pruned_reach": Rin, "pair_sms": sms, "pair_blocks_per_sm": blocks,
                "staging_depth": depth, "fused_prune": fchoice, "us_per_step": round(us, 2),
                "trials": len(trials) + len(final) + len(fused_trials)}

    def temperature(self, stream=None):
        t = self.thermo(stream)
        return 2.0 * t["kinetic"] / (t["ndof"] * KB)

    def total_energy(self, x, v, box, dt, dispersion=False, stream=None):
        """The total energy at the current positions x_N, for energy
        conservation: the potential at x_N and the kinetic energy centred at
        N, the mean of the half steps N - 1/2 and N + 1/2 of leap-frog.  The
        half step N + 1/2 is one more MD step, so this advances the state by
        one step.  (The kinetic energy of `thermo` is centred one step behind
        the positions; paired with the potential at x_N it is off by O(dt).)
        Returns (total, potential, kinetic)."""
        t = self.term
        t.force(x, box, energy=True, stream=stream)
        e = t.energies(stream)
        c = t.constants(box, dispersion=dispersion)
        pot = e["lj"] + e["coulomb"] + e["excluded"] + e["reciprocal"] + c["self"] + c["background"] + \
            c["dispersion"]
        self.run(x, v, box, dt, 1, unroll=0, stream=stream)
        kin = self.thermo(stream)["kinetic"]
        return pot + kin, pot, kin
