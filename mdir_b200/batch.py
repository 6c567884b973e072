"""Batches of independent frames on the device (the batching form).

`BatchEvaluator(frames)` takes a list of system dicts (`systems.batch_frames`:
solvated boxes of uneven sizes, each with its own cell and PME grid, one LJ
type table) and evaluates the forces and energies of all of them with one
launch of each kernel over all frames (`mdrtNbBatch*` of libmdrt_nb.so):
the build, the persistent pair kernel, the excluded pairs, PME (one batched
cuFFT plan pair per grid shape), and the per-frame energy sums.  With
`graph=True` the evaluation is replayed as a CUDA graph.

MDIR evaluates frames one after another (D251); its device batch (D386)
loops over frames of one program (python/mdir/_frames.py:769)."""

import ctypes

import numpy as np
import torch

from . import _lib as L
from .term import _dp, _host, _hp, _stream, exclusion_rows

TERMS = ("lj", "coulomb", "excluded", "reciprocal", "self", "background")


def pack(frames):
    """The batch's arrays from a list of frames: atoms per frame, charges,
    types, exclusion rows and positions in the batch's numbering, boxes
    (frames, 3) and grids (frames, 3); checks that the frames share what a
    batch shares."""
    f0 = frames[0]
    for f in frames[1:]:
        for key in ("cutoff", "reach", "beta", "order"):
            if f[key] != f0[key]:
                raise ValueError(f"frames differ in {key!r}; a batch shares it")
        if not (np.array_equal(f["sigma"], f0["sigma"]) and np.array_equal(f["epsilon"], f0["epsilon"])):
            raise ValueError("frames differ in the LJ type table; a batch shares one")
    atoms = np.array([len(f["charges"]) for f in frames], dtype=np.int64)
    start = np.concatenate([[0], np.cumsum(atoms)])
    pairs = [np.asarray(f["excluded_pairs"], dtype=np.int64).reshape(-1, 2) + start[k]
             for k, f in enumerate(frames)]
    pairs = np.concatenate(pairs) if pairs else np.zeros((0, 2), dtype=np.int64)
    return {
        "atoms": atoms, "start": start,
        "charges": np.concatenate([f["charges"] for f in frames]).astype(np.float64),
        "types": np.concatenate([f["types"] for f in frames]).astype(np.int32),
        "excluded_pairs": pairs,
        "positions": np.concatenate([f["positions"] for f in frames]).astype(np.float64),
        "boxes": np.stack([np.asarray(f["box"], dtype=np.float64) for f in frames]),
        "grids": np.stack([np.asarray(f["grid"], dtype=np.int32) for f in frames]),
    }


class BatchEvaluator:
    """Forces and energies of a batch of frames on one device."""

    def __init__(self, frames, device=0):
        self.frames = frames
        self.device = torch.device("cuda", device)
        torch.cuda.set_device(self.device)
        p = pack(frames)
        self.packed = p
        self.count = len(frames)
        self.n = int(p["start"][-1])
        self.start = p["start"]
        self.boxes = np.ascontiguousarray(p["boxes"])
        h = ctypes.c_void_p()
        atoms = _host(p["atoms"], np.int64)
        L.check(L.lib().mdrtNbBatchCreate(ctypes.byref(h), device, self.count, _hp(atoms)), "mdrtNbBatchCreate")
        self._h = h
        f0 = frames[0]
        sg = _host(f0["sigma"], np.float64)
        ep = _host(f0["epsilon"], np.float64)
        L.check(L.lib().mdrtNbBatchSetParticles(h, _hp(_host(p["charges"], np.float64)),
                                                _hp(_host(p["types"], np.int32)), sg.shape[0], _hp(sg), _hp(ep)),
                "mdrtNbBatchSetParticles")
        off, part = exclusion_rows(self.n, p["excluded_pairs"])
        off = _host(off, np.int32)
        part = _host(part, np.int32)
        L.check(L.lib().mdrtNbBatchSetExclusions(h, _hp(off), _hp(part) if len(part) else None),
                "mdrtNbBatchSetExclusions")
        pme = f0.get("pme", True)
        L.check(L.lib().mdrtNbBatchSetInteraction(h, f0["cutoff"], f0["reach"], f0["beta"] if pme else 0.0,
                                                  float.fromhex("0x1.15def44ac2182p+7")),
                "mdrtNbBatchSetInteraction")
        if pme:
            grids = _host(p["grids"], np.int32)
            L.check(L.lib().mdrtNbBatchPmeSetup(h, _hp(grids), int(f0["order"])), "mdrtNbBatchPmeSetup")
        self.x = torch.tensor(p["positions"], dtype=torch.float64, device=self.device)
        self.forces_out = torch.zeros((self.n, 3), dtype=torch.float64, device=self.device)
        self.built = False

    def close(self):
        if getattr(self, "_h", None):
            L.lib().mdrtNbBatchDestroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def frame(self, k, array):
        """Frame k's rows of a (n, ...) array of the batch."""
        return array[self.start[k]:self.start[k + 1]]

    def set_positions(self, positions):
        """Positions of all frames: an (n, 3) array or tensor in the batch's
        numbering, or a list of per-frame (n_f, 3) arrays."""
        if isinstance(positions, (list, tuple)):
            positions = np.concatenate([np.asarray(x, dtype=np.float64) for x in positions])
        self.x.copy_(torch.as_tensor(positions, dtype=torch.float64), non_blocking=True)

    def build(self, stream=None):
        sizes = np.zeros(L.SIZE_COUNT, dtype=np.int32)
        L.check(L.lib().mdrtNbBatchBuild(self._h, _dp(self.x), _hp(self.boxes), _stream(stream), _hp(sizes)),
                "mdrtNbBatchBuild")
        self.built = True
        return sizes

    def set_tuning(self, pair_blocks_per_sm=None, search_warps=None, staging_depth=None):
        if staging_depth is not None:
            L.check(L.lib().mdrtNbBatchSetTuning(self._h, L.TUNE_STAGING_DEPTH, int(staging_depth)),
                    "mdrtNbBatchSetTuning")
        if pair_blocks_per_sm is not None:
            L.check(L.lib().mdrtNbBatchSetTuning(self._h, L.TUNE_PAIR_BLOCKS_PER_SM, int(pair_blocks_per_sm)),
                    "mdrtNbBatchSetTuning")
        if search_warps is not None:
            L.check(L.lib().mdrtNbBatchSetTuning(self._h, L.TUNE_SEARCH_WARPS, int(search_warps)),
                    "mdrtNbBatchSetTuning")

    def autotune(self, stream=None):
        """Times every launch shape of the build and the pair kernel on this
        batch (search warps a group, pair blocks an SM, staging depth) and
        keeps the fastest; returns the choice, with the group's members and
        the threads its accumulators rotate over, which the layout fixes."""
        if not self.built:
            self.build(stream)
        choice = np.zeros(3, dtype=np.int32)
        L.check(L.lib().mdrtNbBatchAutotune(self._h, _dp(self.x), _dp(self.forces_out), _stream(stream),
                                            _hp(choice)), "mdrtNbBatchAutotune")
        return {"search_warps": int(choice[0]), "pair_blocks_per_sm": int(choice[1]),
                "staging_depth": int(choice[2]), "members_per_group": 16, "threads_per_group": 16}

    def force(self, energy=True, graph=False, stream=None):
        """The forces of all frames (device f64 (n, 3), the evaluator's
        buffer) at the current positions; with `energy`, the energies are
        summed per frame on the device (read them with `energies()`)."""
        if not self.built:
            self.build(stream)
        flags = (L.ENERGY if energy else 0) | (L.GRAPH if graph else 0)
        L.check(L.lib().mdrtNbBatchForce(self._h, _dp(self.x), flags, _dp(self.forces_out), _stream(stream)),
                "mdrtNbBatchForce")
        return self.forces_out

    def energies(self, stream=None):
        """Per-frame energy terms (kJ/mol) of the last evaluation with
        energies: a dict of (frames,) arrays, with "potential" their sum."""
        out = np.zeros((self.count, L.E_COUNT))
        L.check(L.lib().mdrtNbBatchEnergies(self._h, _stream(stream), _hp(out)), "mdrtNbBatchEnergies")
        const = np.zeros((self.count, 2))
        L.check(L.lib().mdrtNbBatchConstants(self._h, _hp(const)), "mdrtNbBatchConstants")
        terms = {"lj": out[:, L.E_LJ], "coulomb": out[:, L.E_COULOMB], "excluded": out[:, L.E_EXCLUDED],
                 "reciprocal": out[:, L.E_RECIPROCAL], "self": const[:, 0], "background": const[:, 1]}
        terms["potential"] = sum(terms[k] for k in TERMS)
        terms["virial_pair"] = out[:, L.W_PAIR:L.W_PAIR + 6]
        terms["virial_reciprocal"] = out[:, L.W_RECIPROCAL:L.W_RECIPROCAL + 6]
        return terms


def shard(atoms, ranks):
    """Frames assigned to ranks by greedy bin-packing on their atom counts
    (largest first, each to the least loaded rank): a list of frame-number
    lists, each in increasing order."""
    load = [0] * ranks
    out = [[] for _ in range(ranks)]
    for f in sorted(range(len(atoms)), key=lambda k: (-int(atoms[k]), k)):
        r = min(range(ranks), key=lambda q: (load[q], q))
        out[r].append(f)
        load[r] += int(atoms[f])
    return [sorted(o) for o in out]
