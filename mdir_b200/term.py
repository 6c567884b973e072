"""The nonbonded + PME term over the C ABI (include/mdrt_nb.h).

`NonbondedTerm` owns one native context: the neighbor structure, the
particle tables and the PME plans of one system on one device.  Device
arrays are torch CUDA tensors (torch is the allocator and the stream
source, nothing more); every call goes through libmdrt_nb.so."""

import ctypes

import numpy as np
import torch

from . import _lib as L

COULOMB = float.fromhex("0x1.15def44ac2182p+7")  # kJ mol^-1 nm e^-2 (MDIR COULOMB_NATIVE)


def _stream(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _host(a, dtype):
    return np.ascontiguousarray(np.asarray(a, dtype=dtype))


def _hp(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _dp(t):
    return ctypes.c_void_p(t.data_ptr())


def exclusion_rows(n, pairs):
    """Ragged rows (offsets[n+1], partners) of excluded pairs, both ways."""
    pairs = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    if len(pairs) == 0:
        return np.zeros(n + 1, dtype=np.int32), np.zeros(0, dtype=np.int32)
    both = np.concatenate([pairs, pairs[:, ::-1]])
    both = both[np.lexsort((both[:, 1], both[:, 0]))]
    counts = np.bincount(both[:, 0], minlength=n)
    off = np.zeros(n + 1, dtype=np.int32)
    off[1:] = np.cumsum(counts)
    return off, both[:, 1].astype(np.int32)


class NonbondedTerm:
    """One system's short-range nonbonded + PME term on one CUDA device."""

    def __init__(self, particles, device=0):
        self.n = int(particles)
        self.device = torch.device("cuda", device)
        torch.cuda.set_device(self.device)
        handle = ctypes.c_void_p()
        L.check(L.lib().mdrtNbCreate(ctypes.byref(handle), device, self.n), "mdrtNbCreate")
        self._h = handle
        self.box = None
        self.ntypes = 1
        self.interaction = None
        self.pruned = 0.0
        self.pair_sms = 0
        self.pair_blocks_per_sm = 4
        self.fused_prune = 0
        self.staging_depth = 1
        self.frame_graphs = True

    def close(self):
        if getattr(self, "_h", None):
            L.lib().mdrtNbDestroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- configuration -----------------------------------------------------
    def set_particles(self, charges, types, sigma, epsilon):
        q = _host(charges, np.float64)
        t = _host(types, np.int32)
        sg = _host(sigma, np.float64)
        ep = _host(epsilon, np.float64)
        nt = sg.shape[0]
        L.check(L.lib().mdrtNbSetParticles(self._h, _hp(q), _hp(t), nt, _hp(sg), _hp(ep)),
                "mdrtNbSetParticles")
        self.ntypes = nt

    def set_exclusions(self, pairs=None, rows=None):
        off, part = rows if rows is not None else exclusion_rows(self.n, pairs if pairs is not None else [])
        off = _host(off, np.int32)
        part = _host(part, np.int32)
        L.check(L.lib().mdrtNbSetExclusions(self._h, _hp(off), _hp(part) if len(part) else None),
                "mdrtNbSetExclusions")

    def set_interaction(self, cutoff, reach, beta, coulomb=COULOMB, coulomb_shift=False,
                        lj_switch=False, switch_distance=0.0):
        L.check(L.lib().mdrtNbSetInteraction(self._h, cutoff, reach, beta, coulomb, int(coulomb_shift),
                                             int(lj_switch), switch_distance), "mdrtNbSetInteraction")
        self.interaction = {"cutoff": cutoff, "reach": reach, "beta": beta, "coulomb": coulomb,
                            "coulomb_shift": coulomb_shift, "lj_switch": lj_switch,
                            "switch_distance": switch_distance}

    def set_reach(self, reach):
        """A new reach of the lists (the next build uses it)."""
        kw = dict(self.interaction)
        kw["reach"] = reach
        self.set_interaction(**kw)

    def set_pme(self, grid, order=4):
        k = [0, 0, 0] if grid is None else [int(v) for v in grid]
        L.check(L.lib().mdrtPmeSetup(self._h, k[0], k[1], k[2], int(order)), "mdrtPmeSetup")
        self.pme_grid = k

    def set_pruned_reach(self, pruned_distance):
        """The dual list: prune the lists to this reach (0: one list)."""
        L.check(L.lib().mdrtNbSetPrunedReach(self._h, float(pruned_distance)), "mdrtNbSetPrunedReach")
        self.pruned = float(pruned_distance)

    def prune(self, x, box=None, stream=None):
        b = _host(self.box if box is None else box, np.float64)
        L.check(L.lib().mdrtNbPrune(self._h, _dp(x), _hp(b), _stream(stream)), "mdrtNbPrune")

    def set_tuning(self, pair_blocks_per_sm=None, pair_sms=None, fused_prune=None, staging_depth=None,
                   pme_fft=None, pme_spread=None, frame_graphs=None):
        """Launch shapes, the MD step's pruning in the pair kernel (0 by
        group count, 1 always, 2 never) and the PME transforms ("own", the
        library's three-kernel convolution where every grid dimension is 32,
        64 or 128; "cufft"): the autotuner's knobs; results do not depend on
        them beyond the order of f32 sums.  pme_spread: "auto" (global
        atomics, measured faster on the B200), "global" or "tiles"
        (shared-memory tiles, the mixed mode).  frame_graphs: whether
        force_frames and parameter_gradient_frames keep their launches as
        CUDA graphs (True, the default)."""
        if pair_blocks_per_sm is not None:
            L.check(L.lib().mdrtNbSetTuning(self._h, L.TUNE_PAIR_BLOCKS_PER_SM, int(pair_blocks_per_sm)),
                    "mdrtNbSetTuning")
            self.pair_blocks_per_sm = int(pair_blocks_per_sm)
        if pair_sms is not None:
            L.check(L.lib().mdrtNbSetTuning(self._h, L.TUNE_PAIR_SMS, int(pair_sms)), "mdrtNbSetTuning")
            self.pair_sms = int(pair_sms)
        if staging_depth is not None:
            L.check(L.lib().mdrtNbSetTuning(self._h, L.TUNE_STAGING_DEPTH, int(staging_depth)), "mdrtNbSetTuning")
            self.staging_depth = int(staging_depth)
        if fused_prune is not None:
            L.check(L.lib().mdrtNbSetTuning(self._h, L.TUNE_FUSED_PRUNE, int(fused_prune)), "mdrtNbSetTuning")
            self.fused_prune = int(fused_prune)
        if pme_fft is not None:
            code = {"own": 0, "cufft": 1}[pme_fft]
            L.check(L.lib().mdrtNbSetTuning(self._h, L.TUNE_PME_FFT, code), "mdrtNbSetTuning")
            self.pme_fft = pme_fft
        if pme_spread is not None:
            code = {"auto": 0, "global": 1, "tiles": 2}[pme_spread]
            L.check(L.lib().mdrtNbSetTuning(self._h, L.TUNE_PME_SPREAD, code), "mdrtNbSetTuning")
            self.pme_spread = pme_spread
        if frame_graphs is not None:
            L.check(L.lib().mdrtNbSetTuning(self._h, L.TUNE_FRAME_GRAPHS, int(bool(frame_graphs))),
                    "mdrtNbSetTuning")
            self.frame_graphs = bool(frame_graphs)

    def frame_graph_info(self):
        """(captures, replays) of the frames entries' graphs so far."""
        a, b = ctypes.c_int64(0), ctypes.c_int64(0)
        L.check(L.lib().mdrtNbFrameGraphInfo(self._h, ctypes.byref(a), ctypes.byref(b)), "mdrtNbFrameGraphInfo")
        return a.value, b.value

    def set_deterministic(self, on=True):
        L.check(L.lib().mdrtNbSetDeterministic(self._h, int(bool(on))), "mdrtNbSetDeterministic")

    # -- the path ------------------------------------------------------------
    def _check_x(self, x):
        if not (x.is_cuda and x.dtype == torch.float64 and x.shape == (self.n, 3) and x.is_contiguous()):
            raise ValueError("positions: a contiguous CUDA float64 tensor of shape (n, 3)")

    def build(self, x, box, reach=0.0, stream=None, allow_nan=False):
        """The neighbor build at device positions x; returns the sizes.  `box`
        is the three edges of an orthorhombic cell or the six numbers
        (ax, by, cz, bx, cx, cy) of a triclinic one."""
        self._check_x(x)
        b = _host(box, np.float64)
        sizes = np.zeros(L.SIZE_COUNT, dtype=np.int32)
        entry = L.lib().mdrtNbBuildTriclinic if len(b) == 6 else L.lib().mdrtNbBuild
        s = entry(self._h, _dp(x), self.n, _hp(b), reach, _stream(stream), _hp(sizes))
        if not (s == L.NAN_POSITION and allow_nan):
            L.check(s, "mdrtNbBuild")
        self.box = b
        return sizes

    def force(self, x, box=None, energy=False, potential=False, forces=None, accumulate=False,
              pairs=True, pme=True, excluded=True, prune=False, stream=None):
        """Forces (device f64 (n, 3)) of the term at x; `prune` prunes the
        dual list at x first (in the pair kernel itself for forces alone)."""
        self._check_x(x)
        b = _host(self.box if box is None else box, np.float64)
        if forces is None:
            forces = torch.empty((self.n, 3), dtype=torch.float64, device=x.device)
        flags = (L.ENERGY if energy else 0) | (L.POTENTIAL if potential else 0) | \
            (L.ACCUMULATE if accumulate else 0) | (0 if pairs else L.NO_PAIRS) | \
            (0 if pme else L.NO_PME) | (0 if excluded else L.NO_EXCLUDED) | (L.PRUNE if prune else 0)
        entry = L.lib().mdrtNbForceTriclinic if len(b) == 6 else L.lib().mdrtNbForce
        L.check(entry(self._h, _dp(x), _hp(b), flags, _dp(forces), _stream(stream)), "mdrtNbForce")
        return forces

    def force_frames(self, X, first, step, F, potentials=None, box=None, stream=None):
        """Forces of the frames first, first + step, ... of X (device f64
        (K, n, 3)) into the same frames of F, one native call
        (mdrtNbForceFrames); with `potentials` (device f32 (K, K1, K2, K3))
        each frame's reciprocal potential grid is kept there."""
        K = X.shape[0]
        count = len(range(first, K, step))
        if count == 0:
            return
        b = _host(self.box if box is None else box, np.float64)
        frame = 3 * self.n
        phi, pstride = None, 0
        if potentials is not None:
            pstride = step * potentials[0].numel()
            phi = ctypes.c_void_p(potentials.data_ptr() + 4 * first * potentials[0].numel())
        L.check(L.lib().mdrtNbForceFrames(self._h, ctypes.c_void_p(X.data_ptr() + 8 * first * frame), step * frame,
                                          count, _hp(b), 0, ctypes.c_void_p(F.data_ptr() + 8 * first * frame),
                                          step * frame, phi, pstride, _stream(stream)), "mdrtNbForceFrames")

    def parameter_gradient_frames(self, X, first, step, G, dq, dtable, potentials=None, box=None, stream=None):
        """parameter_gradient over the frames first, first + step, ... of X
        with their cotangents in G (device f64 (K, n, 3)) and, when given,
        their kept potential grids; one native call
        (mdrtNbParameterGradientFrames), accumulating into dq and dtable."""
        K = X.shape[0]
        count = len(range(first, K, step))
        if count == 0:
            return
        b = _host(self.box if box is None else box, np.float64)
        frame = 3 * self.n
        phi, pstride = None, 0
        if potentials is not None:
            pstride = step * potentials[0].numel()
            phi = ctypes.c_void_p(potentials.data_ptr() + 4 * first * potentials[0].numel())
        L.check(L.lib().mdrtNbParameterGradientFrames(
            self._h, ctypes.c_void_p(X.data_ptr() + 8 * first * frame), step * frame, count, _hp(b),
            ctypes.c_void_p(G.data_ptr() + 8 * first * frame), step * frame, L.GRAD_PRODUCT, phi, pstride,
            _dp(dq), _dp(dtable), _stream(stream)), "mdrtNbParameterGradientFrames")

    def energies(self, stream=None):
        out = np.zeros(L.E_COUNT)
        L.check(L.lib().mdrtNbEnergies(self._h, _stream(stream), _hp(out)), "mdrtNbEnergies")
        return {"lj": out[L.E_LJ], "coulomb": out[L.E_COULOMB], "excluded": out[L.E_EXCLUDED],
                "reciprocal": out[L.E_RECIPROCAL],
                "virial_pair": _sym(out[L.W_PAIR:L.W_PAIR + 6]),
                "virial_reciprocal": _sym(out[L.W_RECIPROCAL:L.W_RECIPROCAL + 6])}

    def constants(self, box=None, dispersion=False):
        b = _host(self.box if box is None else box, np.float64)
        out = np.zeros(4)
        L.check(L.lib().mdrtNbConstants(self._h, _hp(b), int(dispersion), _hp(out)), "mdrtNbConstants")
        return {"self": out[0], "background": out[1], "dispersion": out[2], "dispersion_virial": out[3]}

    def potential(self, stream=None):
        out = torch.empty(self.n, dtype=torch.float64, device=self.device)
        L.check(L.lib().mdrtPmePotential(self._h, _dp(out), _stream(stream)), "mdrtPmePotential")
        return out

    def displacement(self, frames, box=None, stream=None):
        """The largest displacement of each frame (device f64 (K, n, 3))
        from the positions of the last build (host f64 (K,))."""
        if not (frames.is_cuda and frames.dtype == torch.float64 and frames.is_contiguous()
                and frames.shape[-2:] == (self.n, 3)):
            raise ValueError("frames: a contiguous CUDA float64 tensor of shape (K, n, 3)")
        count = frames.numel() // (3 * self.n)
        b = _host(self.box if box is None else box, np.float64)
        out = np.zeros(count)
        L.check(L.lib().mdrtNbDisplacement(self._h, _dp(frames), count, _hp(b), _hp(out), _stream(stream)),
                "mdrtNbDisplacement")
        return out

    def displacement_start(self, frames, box=None, stream=None):
        """Queues the test of displacement() without waiting; returns the
        frame count for displacement_result()."""
        if not (frames.is_cuda and frames.dtype == torch.float64 and frames.is_contiguous()
                and frames.shape[-2:] == (self.n, 3)):
            raise ValueError("frames: a contiguous CUDA float64 tensor of shape (K, n, 3)")
        count = frames.numel() // (3 * self.n)
        b = _host(self.box if box is None else box, np.float64)
        L.check(L.lib().mdrtNbDisplacementStart(self._h, _dp(frames), count, _hp(b), _stream(stream)),
                "mdrtNbDisplacementStart")
        return count

    def displacement_result(self, count):
        """The result of the test displacement_start() queued (host f64
        (count,)); waits for that test only."""
        out = np.zeros(count)
        L.check(L.lib().mdrtNbDisplacementResult(self._h, _hp(out)), "mdrtNbDisplacementResult")
        return out

    def potential_grid(self, out=None, stream=None):
        """The reciprocal potential grid of the last force evaluation (device
        f32 of the grid's shape), into `out` when given."""
        if out is None:
            out = torch.empty(tuple(self.pme_grid), dtype=torch.float32, device=self.device)
        if not (out.is_cuda and out.dtype == torch.float32 and out.is_contiguous()
                and out.numel() == int(np.prod(self.pme_grid))):
            raise ValueError("out: a contiguous CUDA float32 tensor of the grid's size")
        L.check(L.lib().mdrtPmePotentialGrid(self._h, ctypes.c_void_p(out.data_ptr()), _stream(stream)),
                "mdrtPmePotentialGrid")
        return out

    def parameter_gradient(self, x, cotangent=None, box=None, dq=None, dtable=None, ntypes=None,
                           stream=None, potential=None):
        """The gradient in the charges and the sigma / epsilon table at x:
        with a cotangent g (device f64 (n, 3)) on the forces, the product
        sum_k g_k . dF_k/dtheta, else dE/dtheta (without the dispersion
        correction).  Adds into dq (device f64 (n,)) and dtable (device f64
        (2, ntypes, ntypes)), created as zeros when not given; returns both.
        `potential`: the potential grid that potential_grid() kept from the
        force evaluation at the same x and charges, so that the reciprocal
        forward is not run again."""
        self._check_x(x)
        b = _host(self.box if box is None else box, np.float64)
        if dq is None:
            dq = torch.zeros(self.n, dtype=torch.float64, device=x.device)
        if dtable is None:
            nt = self.ntypes if ntypes is None else ntypes
            dtable = torch.zeros((2, nt, nt), dtype=torch.float64, device=x.device)
        mode = L.GRAD_ENERGY
        g = None
        if cotangent is not None:
            self._check_x(cotangent)
            mode = L.GRAD_PRODUCT
            g = _dp(cotangent)
        phi = None
        if potential is not None:
            if not (potential.is_cuda and potential.dtype == torch.float32 and potential.is_contiguous()
                    and potential.numel() == int(np.prod(self.pme_grid))):
                raise ValueError("potential: a contiguous CUDA float32 tensor of the grid's size")
            phi = ctypes.c_void_p(potential.data_ptr())
        L.check(L.lib().mdrtNbParameterGradientPotential(self._h, _dp(x), _hp(b), g, mode, phi, _dp(dq),
                                                         _dp(dtable), _stream(stream)),
                "mdrtNbParameterGradientPotential")
        return dq, dtable

    def status(self, clear=False, stream=None):
        v = ctypes.c_int32()
        L.check(L.lib().mdrtNbStatus(self._h, _stream(stream), int(clear), ctypes.byref(v)), "mdrtNbStatus")
        return v.value

    def info(self):
        cap, builds, grows = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        L.check(L.lib().mdrtNbGroupsInfo(self._h, ctypes.byref(cap), ctypes.byref(builds),
                                         ctypes.byref(grows)), "mdrtNbGroupsInfo")
        return {"list_capacity": cap.value, "builds": builds.value, "grows": grows.value}

    def buffer(self, slot, dtype, width=1):
        """A host copy of a buffer of the neighbor structure."""
        p, k = ctypes.c_void_p(), ctypes.c_int64()
        L.check(L.lib().mdrtNbGroupsBuffer(self._h, slot, ctypes.byref(p), ctypes.byref(k)),
                "mdrtNbGroupsBuffer")
        itemsize = np.dtype(dtype).itemsize * width
        out = np.empty(k.value * width, dtype=dtype)
        torch.cuda.synchronize(self.device)
        res = _cudart().cudaMemcpy(ctypes.c_void_p(out.ctypes.data), p, ctypes.c_size_t(k.value * itemsize), 2)
        if int(res) != 0:
            raise RuntimeError(f"cudaMemcpy failed: {res}")
        return out.reshape(-1, width) if width > 1 else out

    def pair_set(self, sizes):
        """The (i, j, image code) of every bit of the lists, i < j by atom
        number, code = 9(sz+1)+3(sy+1)+(sx+1) of j relative to i."""
        order = self.buffer(L.SLOT_ORDER, np.int32)
        counts = self.buffer(L.SLOT_COUNTS, np.int32)
        cap = self.info()["list_capacity"]
        entries = self.buffer(L.SLOT_ENTRIES, np.int32, 2)
        G = int(sizes[L.SIZE_GROUPS])
        counts = counts[:G]
        E = entries[: G * cap].reshape(G, cap, 2)
        valid = np.arange(cap)[None, :] < counts[:, None]
        g_idx, e_idx = np.nonzero(valid)
        q = E[g_idx, e_idx, 0]
        bits = E[g_idx, e_idx, 1].astype(np.uint32)
        mask = bits & 0xFFFF
        code = (bits >> 16) & 0x7FFF  # a lattice vector, five bits a component
        m_bits = (mask[:, None] >> np.arange(16)[None, :]) & 1
        k_idx, m_idx = np.nonzero(m_bits)
        a = order[16 * g_idx[k_idx] + m_idx]
        b = order[q[k_idx]]
        c = code[k_idx].astype(np.int64)
        sx, sy, sz = (c & 31) - 16, ((c >> 5) & 31) - 16, ((c >> 10) & 31) - 16
        swap = b < a
        sx = np.where(swap, -sx, sx)
        sy = np.where(swap, -sy, sy)
        sz = np.where(swap, -sz, sz)
        i = np.minimum(a, b)
        j = np.maximum(a, b)
        out = np.stack([i, j, 9 * (sz + 1) + 3 * (sy + 1) + (sx + 1)], axis=1).astype(np.int32)
        return out

    def pair_images(self, sizes):
        """The (i, j, na, nb, nc) of every bit of the lists, i < j by atom
        number: the lattice vector of j's image relative to i in the raw
        positions (the entry's image plus the places' shifts), for either
        cell."""
        order = self.buffer(L.SLOT_ORDER, np.int32)
        counts = self.buffer(L.SLOT_COUNTS, np.int32)
        shifts = self.buffer(L.SLOT_SHIFTS, np.int8, 4).astype(np.int64)
        cap = self.info()["list_capacity"]
        entries = self.buffer(L.SLOT_ENTRIES, np.int32, 2)
        G = int(sizes[L.SIZE_GROUPS])
        counts = counts[:G]
        E = entries[: G * cap].reshape(G, cap, 2)
        valid = np.arange(cap)[None, :] < counts[:, None]
        g_idx, e_idx = np.nonzero(valid)
        q = E[g_idx, e_idx, 0]
        bits = E[g_idx, e_idx, 1].astype(np.uint32)
        mask = bits & 0xFFFF
        code = ((bits >> 16) & 0x7FFF).astype(np.int64)
        m_bits = (mask[:, None] >> np.arange(16)[None, :]) & 1
        k_idx, m_idx = np.nonzero(m_bits)
        pa = 16 * g_idx[k_idx] + m_idx
        pb = q[k_idx]
        a, b = order[pa], order[pb]
        c = code[k_idx]
        n = np.stack([(c & 31) - 16, ((c >> 5) & 31) - 16, ((c >> 10) & 31) - 16], 1)
        n = n + shifts[pb, :3] - shifts[pa, :3]
        swap = (b < a)[:, None]
        n = np.where(swap, -n, n)
        return np.concatenate([np.minimum(a, b)[:, None], np.maximum(a, b)[:, None], n], 1).astype(np.int32)


_CUDART = None


def _cudart():
    # the CUDA runtime that libmdrt_nb.so loaded (by its soname)
    global _CUDART
    if _CUDART is None:
        L.lib()
        _CUDART = ctypes.CDLL("libcudart.so.12")
        _CUDART.cudaMemcpy.restype = ctypes.c_int
        _CUDART.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    return _CUDART


def _sym(v):
    xx, yy, zz, xy, xz, yz = v
    return np.array([[xx, xy, xz], [xy, yy, yz], [xz, yz, zz]])
