"""Frames of one system on the device: energies, forces, and the gradients
in the parameters (per-type LJ sigma / epsilon and per-atom charges).

Mirrors MDIR's frame evaluator (python/mdir/_frames.py:467-715,
docs/python-frames.md): `FrameEvaluator(system).evaluate(positions,
gradients=("tunables", "positions"))` returns `FrameEnergies` with
`.energy`, `.gradients` and `.vjp(cotangent, positions=)`, the product of
force matching (D381), whose cotangent is on dU/dx = -F.  The tunables are
named "sigma", "epsilon" (one per LJ type, mixed by Lorentz-Berthelot) and
"charges" (one per atom).  MDIR refuses the product in per-atom charges
with PME (D379); here it is given by the adjoint of the reciprocal sum.

Frames of a batch share one neighbor build while they stay within half
the skin of the positions it was made at (one displacement test per batch
on the device, `mdrtNbDisplacement`); a frame that moved further is
evaluated after a new build.  Every evaluation goes through libmdrt_nb.so."""

import numpy as np
import torch

from .api import UnsupportedError
from .term import NonbondedTerm

TUNABLES = ("sigma", "epsilon", "charges")


def lorentz_berthelot(sigma, epsilon):
    """The (ntypes, ntypes) tables sigma_ab = (sigma_a + sigma_b)/2 and
    epsilon_ab = sqrt(epsilon_a epsilon_b)."""
    s = np.asarray(sigma, dtype=np.float64)
    e = np.asarray(epsilon, dtype=np.float64)
    return 0.5 * (s[:, None] + s[None, :]), np.sqrt(e[:, None] * e[None, :])


def lorentz_berthelot_chain(dtable, sigma, epsilon):
    """The gradient in the per-type values from the gradient in the tables
    (dtable[0]: d/dsigma_ab, dtable[1]: d/depsilon_ab, each pair counted
    once in each order).  A type with epsilon 0 has no LJ term and gets no
    epsilon gradient (sqrt is not differentiable there)."""
    T = np.asarray(dtable, dtype=np.float64)
    S = T + np.swapaxes(T, 1, 2)
    s_grad = 0.5 * S[0].sum(axis=1)
    e = np.asarray(epsilon, dtype=np.float64)
    eab = np.sqrt(e[:, None] * e[None, :])
    with np.errstate(divide="ignore", invalid="ignore"):
        w = np.where(e[:, None] > 0, eab / (2.0 * e[:, None]), 0.0)
    e_grad = (S[1] * w).sum(axis=1)
    return s_grad, e_grad


def diagonal_types(system):
    """Per-type sigma and epsilon of a system whose tables are the
    Lorentz-Berthelot mixtures of their diagonals; raises otherwise."""
    sg = np.asarray(system["sigma"], dtype=np.float64)
    ep = np.asarray(system["epsilon"], dtype=np.float64)
    s, e = np.diag(sg).copy(), np.diag(ep).copy()
    ms, me = lorentz_berthelot(s, e)
    if not (np.allclose(ms, sg, rtol=1e-12, atol=0) and np.allclose(me, ep, rtol=1e-12, atol=1e-300)):
        raise UnsupportedError("the LJ tables are not Lorentz-Berthelot mixtures of per-type values")
    return s, e


def dispersion_table_gradient(system, sigma_table, epsilon_table, box):
    """d E_disp / d(sigma_ab, epsilon_ab) of the long-range dispersion
    correction E_disp = -(2 pi / 3V) N^2 <C6> / rc^3, <C6> over the distinct
    non-excluded pairs (MDIR TermNonbonded.cpp:601-637), C6_ab = 4 eps sig^6."""
    types = np.asarray(system["types"])
    nt = sigma_table.shape[0]
    n = len(types)
    cnt = np.bincount(types, minlength=nt).astype(np.float64)
    M = cnt[:, None] * cnt[None, :] - np.diag(cnt)
    pairs = np.asarray(system["excluded_pairs"]).reshape(-1, 2)
    # an excluded pair (i < j) leaves the sum as 2 C6[type_i, type_j], the
    # form of the library's constant (mdrtNbConstants)
    np.subtract.at(M, (types[pairs[:, 0]], types[pairs[:, 1]]), 2.0)
    npair = n * (n - 1.0) - 2.0 * len(pairs)
    V = float(np.prod(box))
    rc = system["cutoff"]
    dE_dc6 = -2.0 * np.pi / (3.0 * V) * n * n / (npair * rc ** 3) * M
    out = np.zeros((2, nt, nt))
    out[0] = dE_dc6 * 24.0 * epsilon_table * sigma_table ** 5
    out[1] = dE_dc6 * 4.0 * sigma_table ** 6
    return out


class FrameEnergies:
    """The result of `FrameEvaluator.evaluate` (MDIR _frames.py:281)."""

    def __init__(self, evaluator, positions, energy, gradients):
        self._evaluator = evaluator
        self._positions = positions
        self._version = evaluator.version
        self.energy = energy
        self.gradients = gradients

    def vjp(self, cotangent=None, *, positions=None):
        """sum_n [g_n dU_n/dtheta + sum_i Gbar_ni . d^2 U_n / dx_i dtheta]
        with g = cotangent (K,) and Gbar = positions (K, n, 3), a cotangent on
        dU/dx = -F (MDIR FrameEnergies.vjp, docs/python-frames.md:203-260);
        returns {"sigma", "epsilon", "charges"} (numpy f64)."""
        ev = self._evaluator
        if ev.version != self._version:
            raise RuntimeError("the parameters changed since this evaluation")
        X = self._positions
        K = X.shape[0]
        dq = torch.zeros(ev.n, dtype=torch.float64, device=ev.device)
        dt = torch.zeros((2, ev.ntypes, ev.ntypes), dtype=torch.float64, device=ev.device)
        if positions is not None:
            Gbar = torch.as_tensor(positions, dtype=torch.float64, device=ev.device).reshape(K, ev.n, 3)
            ev.product(X, -Gbar, dq=dq, dtable=dt)
        if cotangent is not None:
            g = np.broadcast_to(np.asarray(cotangent, dtype=np.float64), (K,))
            for k in ev.schedule(X):
                if g[k] != 0.0:
                    q1, t1 = ev.term.parameter_gradient(X[k])
                    dq += g[k] * q1
                    dt += g[k] * t1
                    if ev.system.get("dispersion", False):
                        dt += g[k] * torch.as_tensor(ev.dispersion_gradient(), device=ev.device)
        return ev.per_type(dq, dt)


class FrameEvaluator:
    """Energies, forces and parameter gradients of frames of one system.

    `lanes` contexts evaluate the frames of one call side by side, frame i
    of the call on lane i mod lanes: lane 0 on the caller's current stream,
    the others on streams of their own, each with its own lists (built at
    the positions of the build in force when it first gets a frame after
    that build) and scratch.  The kernels of one 23,550-atom frame leave
    most of the GPU idle between its two pair launches (FFTs of a 64^3 grid,
    spreading, gathers, short reductions), which the other lanes fill.
    Each lane holds the device memory of one context (lists, frames, PME
    grids); `lanes=1` keeps one.
    Gradient sums are kept per lane and added in lane order at the end of a
    call, so a result does not depend on how the lanes' work interleaves.
    The caller's stream waits for the side lanes before a call returns, so
    the tensors of a call may be freed or reused on that stream at once
    (torch's allocator hands a block back only to the stream it was made on).

    With `frame_graphs` (the default) the library keeps the launches of each
    lane's frames as a CUDA graph and replays it when a call repeats the
    same buffers (mdrtNbForceFrames): a lane then takes all its frames of a
    run in one native call."""

    def __init__(self, system, device=0, sigma=None, epsilon=None, charges=None, lanes=4, keep_potentials=True,
                 frame_graphs=True):
        self.system = system
        self.n = len(system["charges"])
        self.device = torch.device("cuda", device)
        self.box = np.asarray(system["box"], dtype=np.float64)
        self.types = np.asarray(system["types"], dtype=np.int32)
        s0, e0 = (sigma, epsilon) if sigma is not None else diagonal_types(system)
        self.sigma = np.asarray(s0, dtype=np.float64).copy()
        self.epsilon = np.asarray(e0, dtype=np.float64).copy()
        self.charges = np.asarray(system["charges"] if charges is None else charges, dtype=np.float64).copy()
        self.ntypes = len(self.sigma)
        self.cutoff = float(system["cutoff"])
        self.reach = float(system["reach"])
        if int(lanes) < 1:
            raise ValueError("lanes >= 1")
        self.lanes = int(lanes)
        # the forces of the differentiable op keep each frame's reciprocal
        # potential grid (4 bytes a grid point a frame) for the adjoint
        self.grid = list(system["grid"]) if system.get("pme", True) else None
        self.keep_potentials = bool(keep_potentials) and self.grid is not None
        self.frame_graphs = bool(frame_graphs)
        self.term = self._new_term()
        self.version = 0
        self._uploaded = -1
        self._built = False
        self.builds = 0
        # lanes 1.. (created at the first call of several frames)
        self._lane_terms = [self.term]
        self._lane_streams = [None]
        self._lane_built = [0]
        self._lane_uploaded = [-1]
        # the side lanes' gradient sums: charges (lanes - 1, n) and tables
        # (lanes - 1, 2, nt, nt), made at the first product over several lanes
        self._side_sums = None
        self._build_id = 0
        self._build_x = None
        # (build, frames) of the last forces() call when one run served all
        # its frames: the autograd op hands it to its product
        self.last_run = None

    def _new_term(self):
        system = self.system
        term = NonbondedTerm(self.n, self.device.index)
        term.set_exclusions(system["excluded_pairs"])
        pme = system.get("pme", True)
        term.set_interaction(self.cutoff, self.reach, system["beta"] if pme else 0.0,
                             coulomb_shift=system.get("coulomb_shift", False),
                             lj_switch=system.get("lj_switch", False), switch_distance=system.get("switch", 0.0))
        if pme:
            term.set_pme(system["grid"], system["order"])
        if not self.frame_graphs:
            term.set_tuning(frame_graphs=False)
        return term

    # -- parameters ------------------------------------------------------------
    def set_parameters(self, sigma=None, epsilon=None, charges=None):
        """New values of the tunables (host arrays); the next evaluation uses them."""
        changed = False
        for name, value in (("sigma", sigma), ("epsilon", epsilon), ("charges", charges)):
            if value is None:
                continue
            v = np.asarray(value, dtype=np.float64).reshape(getattr(self, name).shape)
            if not np.array_equal(v, getattr(self, name)):
                setattr(self, name, v.copy())
                changed = True
        if changed:
            self.version += 1

    def tables(self):
        return lorentz_berthelot(self.sigma, self.epsilon)

    def _upload(self):
        if self._uploaded != self.version:
            if len(self._lane_terms) > 1:
                # the uploads replace buffers that the lanes' kernels may still read
                torch.cuda.synchronize(self.device)
            sg, ep = self.tables()
            self.term.set_particles(self.charges, self.types, sg, ep)
            self._uploaded = self.version
            self._lane_uploaded[0] = self.version

    def lorentz_berthelot_chain_device(self, dtable):
        """lorentz_berthelot_chain of a device table gradient (2, nt, nt), on
        the device: the sigma and epsilon gradients (nt,) each, f64.  The
        epsilon weights eps_ab / (2 eps_a) are uploaded once per set of
        parameters."""
        key = (self.version, self.device)
        if getattr(self, "_lb_weights", (None,))[0] != key:
            e = np.asarray(self.epsilon, dtype=np.float64)
            eab = np.sqrt(e[:, None] * e[None, :])
            with np.errstate(divide="ignore", invalid="ignore"):
                w = np.where(e[:, None] > 0, eab / (2.0 * e[:, None]), 0.0)
            self._lb_weights = (key, torch.as_tensor(w, dtype=torch.float64, device=self.device))
        w = self._lb_weights[1]
        S = dtable + dtable.transpose(1, 2)
        return 0.5 * S[0].sum(dim=1), (S[1] * w).sum(dim=1)

    def per_type(self, dq, dtable):
        """{"sigma", "epsilon", "charges"} from the table gradient."""
        ds, de = lorentz_berthelot_chain(dtable.cpu().numpy(), self.sigma, self.epsilon)
        return {"sigma": ds, "epsilon": de, "charges": dq.cpu().numpy()}

    def dispersion_gradient(self):
        sg, ep = self.tables()
        return dispersion_table_gradient(self.system, sg, ep, self.box)

    # -- frames ----------------------------------------------------------------
    def frames(self, positions):
        """(K, n, 3) contiguous f64 device frames from a tensor or an array."""
        X = torch.as_tensor(positions, dtype=torch.float64, device=self.device)
        if X.dim() == 2:
            X = X.unsqueeze(0)
        if X.dim() != 3 or X.shape[1:] != (self.n, 3):
            raise ValueError(f"positions: (K, {self.n}, 3)")
        return X.contiguous()

    def runs(self, X, reuse=None):
        """Yields runs (k0, k1) of consecutive frames that one build serves,
        in order, building before a run where needed: the frames ahead are
        tested against the positions of the current build in one launch,
        and a frame that moved more than half the skin gets a new build
        first.  `reuse`: the last_run of a forces() call on these same
        frames, taken as it is (no displacement test) while its build is
        still the one in force."""
        self._upload()
        K = X.shape[0]
        if reuse is not None and reuse == (self._build_id, K) and self._built:
            yield 0, K
            return
        half_skin = 0.5 * (self.reach - self.cutoff)
        k = 0
        while k < K:
            if not self._built:
                self._build(X[k])
            d = self.term.displacement(X[k:])
            bad = np.nonzero(~(d < half_skin))[0]
            run = int(bad[0]) if len(bad) else K - k
            if run == 0:
                self._build(X[k])
                continue
            yield k, k + run
            k += run

    def schedule(self, X):
        """Yields the frame numbers in order, each with a build whose lists
        serve it (the frames of runs())."""
        for k0, k1 in self.runs(X):
            yield from range(k0, k1)

    # frames a lane takes in one native call before the next lane's turn
    # when the launches are not kept as graphs: every lane gets work early,
    # and the host still makes few calls
    LANE_CHUNK = 2

    def _lanes_of_run(self, k0, k1, count):
        """(term, stream, first frame, end) of the native calls of the run
        [k0, k1): frame k goes to lane k mod count, as schedule() hands them
        out, LANE_CHUNK frames of a lane a call, the lanes in turn; with
        frame graphs a lane's frames of the run in one call (one graph
        launch once its buffers repeat)."""
        chunk = -(-(k1 - k0) // count) if self.frame_graphs else self.LANE_CHUNK
        span = count * chunk
        for c0 in range(k0, k1, span):
            c1 = min(k1, c0 + span)
            for l in range(count):
                first = c0 + (l - c0) % count
                if first < c1:
                    term, st, _ = self._lane(first, count)
                    yield term, st, first, c1

    def _build(self, x):
        self.term.build(x, self.box, self.reach)
        self._built = True
        self.builds += 1
        self._build_id += 1
        self._lane_built[0] = self._build_id
        if self.lanes > 1:
            self._build_x = x.clone()  # where the other lanes build when they next get a frame

    # -- lanes -----------------------------------------------------------------
    def _open_lanes(self, frames, sums=False):
        """The lanes of a call of `frames` frames (with `sums`, the side lanes'
        gradient sums zeroed); the side lanes' streams wait for the work
        queued so far on the current stream."""
        count = max(1, min(self.lanes, frames))
        while len(self._lane_terms) < count:
            self._lane_terms.append(self._new_term())
            self._lane_streams.append(torch.cuda.Stream(device=self.device))
            self._lane_built.append(0)
            self._lane_uploaded.append(-1)
        if sums and count > 1:
            self._zero_sums(count)
        if count > 1:
            self._fork(range(1, count))
        return count

    def _fork(self, lanes):
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream(self.device))
        for l in lanes:
            self._lane_streams[l].wait_event(ev)

    def _lane(self, i, count):
        """(term, stream, lane) for frame i of a call over `count` lanes."""
        l = i % count
        if l == 0:
            return self.term, None, 0
        term, st = self._lane_terms[l], self._lane_streams[l]
        if self._lane_uploaded[l] != self.version:
            torch.cuda.synchronize(self.device)
            sg, ep = self.tables()
            term.set_particles(self.charges, self.types, sg, ep)
            self._lane_uploaded[l] = self.version
        if self._lane_built[l] != self._build_id:
            self._fork([l])  # the build's positions were made on the current stream
            term.build(self._build_x, self.box, self.reach, stream=st)
            self._lane_built[l] = self._build_id
        return term, st, l

    def _join(self, count):
        cur = torch.cuda.current_stream(self.device)
        for l in range(1, count):
            ev = torch.cuda.Event()
            ev.record(self._lane_streams[l])
            cur.wait_event(ev)

    def _zero_sums(self, count):
        """The side lanes' gradient sums of a call over `count` lanes, set to
        zero on the current stream (two launches)."""
        if self._side_sums is None or self._side_sums[0].shape[0] < count - 1:
            self._side_sums = (torch.zeros((self.lanes - 1, self.n), dtype=torch.float64, device=self.device),
                               torch.zeros((self.lanes - 1, 2, self.ntypes, self.ntypes), dtype=torch.float64,
                                           device=self.device))
        else:
            self._side_sums[0][:count - 1].zero_()
            self._side_sums[1][:count - 1].zero_()

    def potential_buffers(self, frames):
        """A device f32 (frames, K1, K2, K3) buffer for the potential grids of
        `frames` frames (forces(potentials=...)), or None without PME."""
        if self.grid is None:
            return None
        return torch.empty((frames, *self.grid), dtype=torch.float32, device=self.device)

    def forces(self, positions, energy=False, out=None, potentials=None):
        """Forces (K, n, 3) of every frame (and, with `energy`, the
        potential energies (K,) as a host array).  With `potentials` (from
        potential_buffers), each frame's reciprocal potential grid is kept
        there for product(..., potentials=)."""
        X = self.frames(positions)
        F = torch.empty_like(X) if out is None else out
        E = np.zeros(X.shape[0]) if energy else None
        count = self._open_lanes(X.shape[0])
        self.last_run = None
        if not energy:
            # each lane's frames of a run in one native call (the host's
            # launch rate, not the GPU, bounds a call of many small frames)
            K = X.shape[0]

            def launch(k0, k1):
                for term, st, first, end in self._lanes_of_run(k0, k1, count):
                    term.force_frames(X[:end], first, count, F[:end],
                                      potentials=None if potentials is None else potentials[:end], stream=st)

            done = []
            try:
                start = 0
                if self._built:
                    # the frames go on the build in force while their test
                    # runs ahead of them on the device; its result, read
                    # after they are queued, sends the frames from the first
                    # that moved past half the skin round again after a build
                    self._upload()
                    pending = self.term.displacement_start(X)
                    launch(0, K)
                    d = self.term.displacement_result(pending)
                    bad = np.nonzero(~(d < 0.5 * (self.reach - self.cutoff)))[0]
                    start = int(bad[0]) if len(bad) else K
                    if start == K:
                        done.append((0, K))
                    else:
                        # the lanes' frames read the old lists: they finish
                        # before a build writes new ones
                        self._join(count)
                        self._fork(range(1, count))
                if start < K:
                    for k0, k1 in self.runs(X[start:]):
                        done.append((start + k0, start + k1))
                        launch(start + k0, start + k1)
            finally:
                self._join(count)
            if done == [(0, K)]:
                self.last_run = (self._build_id, K)
            return F
        pending = {}  # lane -> the frame whose energies it holds
        try:
            for i, k in enumerate(self.schedule(X)):
                term, st, l = self._lane(i, count)
                if l in pending:
                    E[pending.pop(l)] = self._energy(term, st)
                term.force(X[k], energy=energy, forces=F[k], stream=st)
                if potentials is not None:
                    term.potential_grid(out=potentials[k], stream=st)
                if energy:
                    pending[l] = k
            for l, k in pending.items():
                E[k] = self._energy(self._lane_terms[l], self._lane_streams[l])
        finally:
            self._join(count)
        return (F, E) if energy else F

    def _energy(self, term=None, stream=None):
        term = self.term if term is None else term
        e = term.energies(stream=stream)
        c = term.constants(dispersion=self.system.get("dispersion", False))
        return (e["lj"] + e["coulomb"] + e["excluded"] + e["reciprocal"] + c["self"] + c["background"]
                + c["dispersion"])

    def product(self, positions, cotangent, dq=None, dtable=None, potentials=None, run=None):
        """sum over frames of sum_i g_ni . dF_ni/dtheta for a cotangent g
        (K, n, 3) on the forces: the charge gradient (n,) and the table
        gradient (2, ntypes, ntypes), device f64, accumulated into dq and
        dtable when given.  `potentials`: the grids that forces() kept for
        these frames at these parameters (the reciprocal forward is then
        not run again); `run`: that call's last_run (the frames' test
        against the build is then not made again)."""
        X = self.frames(positions)
        G = torch.as_tensor(cotangent, dtype=torch.float64, device=self.device).reshape(X.shape).contiguous()
        if dq is None:
            dq = torch.zeros(self.n, dtype=torch.float64, device=self.device)
        if dtable is None:
            dtable = torch.zeros((2, self.ntypes, self.ntypes), dtype=torch.float64, device=self.device)
        count = self._open_lanes(X.shape[0], sums=True)
        side = self._side_sums
        sums = [None] + [(side[0][l - 1], side[1][l - 1]) for l in range(1, count)]
        try:
            for k0, k1 in self.runs(X, reuse=run):
                for term, st, first, end in self._lanes_of_run(k0, k1, count):
                    l = first % count
                    q, t = (dq, dtable) if l == 0 else sums[l]
                    term.parameter_gradient_frames(X[:end], first, count, G[:end], q, t,
                                                   potentials=None if potentials is None else potentials[:end],
                                                   stream=st)
        finally:
            self._join(count)
        if count > 1:
            # the lanes' sums in a fixed order (one reduction each)
            dq += side[0][:count - 1].sum(dim=0)
            dtable += side[1][:count - 1].sum(dim=0)
        return dq, dtable

    def energy_gradient(self, positions):
        """dU_n/dtheta per frame: charges (K, n) and tables (K, 2, nt, nt)."""
        X = self.frames(positions)
        K = X.shape[0]
        dq = torch.zeros((K, self.n), dtype=torch.float64, device=self.device)
        dt = torch.zeros((K, 2, self.ntypes, self.ntypes), dtype=torch.float64, device=self.device)
        disp = None
        if self.system.get("dispersion", False):
            disp = torch.as_tensor(self.dispersion_gradient(), device=self.device)
        count = self._open_lanes(K)
        try:
            for i, k in enumerate(self.schedule(X)):
                term, st, _ = self._lane(i, count)
                term.parameter_gradient(X[k], dq=dq[k], dtable=dt[k], stream=st)
        finally:
            self._join(count)
        if disp is not None:
            dt += disp
        return dq, dt

    def evaluate(self, positions, cells=None, tilts=None, *, gradients=("tunables",)):
        """Energies of the frames and the gradients asked for: "positions"
        (dU/dx, (K, n, 3)) and "tunables" (per frame: sigma (K, nt),
        epsilon (K, nt), charges (K, n)).  MDIR: FrameEvaluator.evaluate,
        python/mdir/_frames.py:715.  The cell is the system's edges; `tilts`
        (bx, cx, cy), one cell for every frame, makes it triclinic (the
        lists are built for each frame; the tunables' gradient runs in
        orthorhombic cells only).  Another cell is refused."""
        for g in gradients:
            if g not in ("tunables", "positions"):
                raise ValueError(f"unknown gradient {g!r}")
        if cells is not None and not np.allclose(np.asarray(cells, dtype=np.float64).reshape(-1, 3), self.box):
            raise UnsupportedError("frames in another cell than the system's")
        X = self.frames(positions)
        if tilts is not None:
            t = np.asarray(tilts, dtype=np.float64).reshape(-1, 3)
            if not np.allclose(t, t[0]):
                raise UnsupportedError("frames in different triclinic cells")
            if "tunables" in gradients:
                raise UnsupportedError("parameter gradients in triclinic cells are not implemented")
            cell = np.concatenate([self.box, t[0]])
            self._upload()
            F = torch.empty_like(X)
            E = np.zeros(X.shape[0])
            for k in range(X.shape[0]):
                self.term.build(X[k], cell, self.reach)
                self.builds += 1
                self.term.force(X[k], cell, energy=True, forces=F[k])
                E[k] = self._energy()
            self._built = False  # the lists are the triclinic build's
            out = {"positions": -F} if "positions" in gradients else {}
            return FrameEnergies(self, X, E, out)
        F, E = self.forces(X, energy=True)
        out = {}
        if "positions" in gradients:
            out["positions"] = -F
        if "tunables" in gradients:
            dq, dt = self.energy_gradient(X)
            tab = dt.cpu().numpy()
            per = [lorentz_berthelot_chain(tab[k], self.sigma, self.epsilon) for k in range(X.shape[0])]
            out["tunables"] = {"sigma": np.stack([p[0] for p in per]), "epsilon": np.stack([p[1] for p in per]),
                               "charges": dq.cpu().numpy()}
        return FrameEnergies(self, X, E, out)
