"""Driver of the OpenMP CPU port (cpu_port.c): the CPU baseline that
bench.py times beside the device path, and its reference arm.  Baseline /
test infrastructure only; the product never imports it.

One force evaluation: the neighbor matrix (cell list, f32 test against the
widened reach), the f32 row loop of LJ + Ewald direct with each pair for
both particles, the excluded-pair correction, and SPME with i64 fixed-point
spreading at 2^40, numpy's FFT (pocketfft) and the f64 gather, following
MDIR's host path (lib/Conversion/MDExecToLoops/HostPMESpread.cpp,
HostPMEConvolve.cpp, HostPMEGather.cpp; lib/Runtime/Templates/
NeighborsMatrix.mlir)."""

import ctypes
import os
import time
from pathlib import Path

import numpy as np

from . import oracle as O

HERE = Path(__file__).resolve().parent
_port = None


def port():
    global _port
    if _port is None:
        path = HERE / "libcpu_port.so"
        if not path.exists():
            O.build()
        _port = ctypes.CDLL(str(path))
        p, i64, i32, d = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_double
        _port.cpu_neighbor_matrix.restype = i32
        _port.cpu_neighbor_matrix.argtypes = [i64, p, p, d, p, p, i32, p, p, p]
        _port.cpu_pairs.argtypes = [i64, p, p, p, i32, p, p, p, d, d, d, i32, p, p, p, p]
        _port.cpu_pme_spread.argtypes = [i64, p, p, p, p, i32, p, p]
        _port.cpu_pme_gather.argtypes = [i64, p, p, p, p, i32, p, p]
        _port.cpu_threads.restype = i32
        _port.cpu_set_threads.argtypes = [i32]
    return _port


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class CpuPort:
    """The CPU path for one system dict (mdir_b200.systems)."""

    def __init__(self, system, threads=None):
        self.s = system
        self.n = len(system["charges"])
        if threads:
            port().cpu_set_threads(int(threads))
        self.threads = port().cpu_threads()
        self.box = np.ascontiguousarray(system["box"], dtype=np.float64)
        self.q = np.ascontiguousarray(system["charges"], dtype=np.float64)
        self.qf = self.q.astype(np.float32)
        self.types = np.ascontiguousarray(system["types"], dtype=np.int32)
        sig, eps = np.asarray(system["sigma"]), np.asarray(system["epsilon"])
        self.c6 = np.ascontiguousarray(4 * eps * sig ** 6, dtype=np.float32)
        self.c12 = np.ascontiguousarray(4 * eps * sig ** 12, dtype=np.float32)
        pairs = np.asarray(system["excluded_pairs"]).reshape(-1, 2)
        self.pairs = pairs
        self.rows = O.rows_from_pairs(self.n, pairs) if len(pairs) else (None, None)
        self.width = 512
        self.xw = np.zeros((self.n, 4), dtype=np.float32)
        self.counts = np.zeros(self.n, dtype=np.int32)
        self.nbr = np.zeros(self.n * self.width, dtype=np.int32)
        if system["pme"]:
            self.K = np.asarray(system["grid"], dtype=np.int64)
            self.fixed = np.zeros(int(np.prod(self.K)), dtype=np.int64)
            self.grid = np.zeros(tuple(self.K))
            self.bc, _ = O.influence(self.box, list(self.K), system["order"], system["beta"])

    def build(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        off, ex = self.rows
        while True:
            longest = port().cpu_neighbor_matrix(self.n, _p(x), _p(self.box), self.s["reach"],
                                                 None if off is None else _p(off),
                                                 None if ex is None else _p(ex), self.width,
                                                 _p(self.xw), _p(self.counts), _p(self.nbr))
            if longest <= self.width:
                return
            self.width = int(longest * 1.25) + 8
            self.nbr = np.zeros(self.n * self.width, dtype=np.int32)

    def force(self, x):
        """Forces (n, 3) and the energy terms at x (lists from the last build)."""
        s = self.s
        x = np.ascontiguousarray(x, dtype=np.float64)
        f = np.zeros((self.n, 3))
        e = np.zeros(2)
        port().cpu_pairs(self.n, _p(self.xw), _p(self.qf), _p(self.types), self.c6.shape[0], _p(self.c6),
                         _p(self.c12), _p(self.box), s["cutoff"], s["beta"], O.COULOMB, self.width,
                         _p(self.counts), _p(self.nbr), _p(f), _p(e))
        terms = {"lj": e[0], "coulomb": e[1]}
        if s["pme"]:
            e_ex, f_ex, _ = O.excluded(x, self.q, self.pairs, self.box, s["beta"])
            f += f_ex
            terms["excluded"] = e_ex
            port().cpu_pme_spread(self.n, _p(x), _p(self.q), _p(self.box), _p(self.K), s["order"],
                                  _p(self.fixed), _p(self.grid))
            S = np.fft.rfftn(self.grid)
            w = np.full(self.bc.shape[2], 2.0)
            w[0] = 1.0
            if self.K[2] % 2 == 0:
                w[-1] = 1.0
            terms["reciprocal"] = float(0.5 * (self.bc * (S.real ** 2 + S.imag ** 2) * w).sum())
            phi = np.ascontiguousarray(np.fft.irfftn(self.bc * S, s=tuple(self.K), axes=(0, 1, 2))
                                       * float(np.prod(self.K)))
            port().cpu_pme_gather(self.n, _p(x), _p(self.q), _p(self.box), _p(self.K), s["order"],
                                  _p(phi), _p(f))
        return f, terms


def time_md_steps(system, x, steps, rebuild_every=10, threads=None):
    """Wall seconds per MD step of the CPU path: a force evaluation each step
    and a rebuild of the matrix every `rebuild_every` steps (the half-skin
    test rebuilds a 0.1 nm skin about this often for water at 300 K)."""
    cp = CpuPort(system, threads)
    cp.build(x)
    cp.force(x)  # warm
    t0 = time.perf_counter()
    cp.build(x)
    tb = time.perf_counter() - t0
    t0 = time.perf_counter()
    for _ in range(steps):
        cp.force(x)
    tf = (time.perf_counter() - t0) / steps
    return tf + tb / rebuild_every, cp.threads, tb, tf
