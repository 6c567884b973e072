"""Driver of the OpenMP CPU port (cpu_port.c): the CPU baseline that
bench.py times beside the device path, and its reference arm.  Baseline /
test infrastructure only; the product never imports it.

One force evaluation: the f32 positions in the frame of the last build,
the f32 row loop of LJ + Ewald direct with each pair for both particles,
the f64 excluded-pair correction, and SPME with i64 fixed-point spreading
at 2^40, MDIR's own host FFT (runtime/mdrt_fft.c over pocketfft, built
into oracle/_ref/ from the reference's sources; numpy's pocketfft when that
library is absent), the product with the influence function, and the f64
gather, following MDIR's host path (lib/Conversion/MDExecToLoops/
HostPMESpread.cpp, HostPMEConvolve.cpp, HostPMEGather.cpp; D271;
lib/Runtime/Templates/NeighborsMatrix.mlir)."""

import ctypes
import time
from pathlib import Path

import numpy as np

from . import oracle as O

HERE = Path(__file__).resolve().parent
REF_FFT = HERE / "_ref" / "libmdrt_fft.so"
_port = None
_fft = None


def port():
    global _port, _fft
    if _port is None:
        path = HERE / "libcpu_port.so"
        if not path.exists():
            O.build()
        _port = ctypes.CDLL(str(path))
        p, i64, i32, d = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_double
        _port.cpu_neighbor_matrix.restype = i32
        _port.cpu_neighbor_matrix.argtypes = [i64, p, p, d, p, p, i32, p, p, p, p]
        _port.cpu_frames.argtypes = [i64, p, p, p, p]
        _port.cpu_pairs.argtypes = [i64, p, p, p, i32, p, p, p, d, d, d, i32, p, p, p, p]
        _port.cpu_excluded.argtypes = [i64, p, p, p, p, p, d, d, p, p]
        _port.cpu_pme_spread.argtypes = [i64, p, p, p, p, i32, p, p]
        _port.cpu_pme_gather.argtypes = [i64, p, p, p, p, i32, p, p]
        _port.cpu_pme_reciprocal.restype = d
        _port.cpu_pme_reciprocal.argtypes = [p, p, p, p, p]
        _port.cpu_fft_load.restype = i32
        _port.cpu_fft_load.argtypes = [ctypes.c_char_p]
        _port.cpu_threads.restype = i32
        _port.cpu_set_threads.argtypes = [i32]
        _fft = REF_FFT.exists() and _port.cpu_fft_load(str(REF_FFT).encode()) == 0
    return _port


def reference_fft():
    """True when the port transforms with MDIR's own mdrt_fft.c."""
    port()
    return bool(_fft)


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
        self.shift = np.zeros((self.n, 3), dtype=np.int32)
        self.counts = np.zeros(self.n, dtype=np.int32)
        self.nbr = np.zeros(self.n * self.width, dtype=np.int32)
        if system["pme"]:
            self.K = np.asarray(system["grid"], dtype=np.int64)
            self.fixed = np.zeros(int(np.prod(self.K)), dtype=np.int64)
            self.grid = np.zeros(tuple(self.K))
            self.bc = np.ascontiguousarray(O.influence(self.box, list(self.K), system["order"],
                                                      system["beta"])[0])
            self.spec = np.zeros(2 * int(self.K[0] * self.K[1] * (self.K[2] // 2 + 1)))
            self.rowsum = np.zeros(int(self.K[0] * self.K[1]))

    def build(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        off, ex = self.rows
        while True:
            longest = port().cpu_neighbor_matrix(self.n, _p(x), _p(self.box), self.s["reach"],
                                                 None if off is None else _p(off),
                                                 None if ex is None else _p(ex), self.width,
                                                 _p(self.xw), _p(self.shift), _p(self.counts), _p(self.nbr))
            if longest <= self.width:
                return
            self.width = int(longest * 1.25) + 8
            self.nbr = np.zeros(self.n * self.width, dtype=np.int32)

    def force(self, x):
        """Forces (n, 3) and the energy terms at x, with the matrix of the
        last build (valid while no particle has moved half the skin)."""
        s = self.s
        x = np.ascontiguousarray(x, dtype=np.float64)
        port().cpu_frames(self.n, _p(x), _p(self.box), _p(self.shift), _p(self.xw))
        f = np.zeros((self.n, 3))
        e = np.zeros(3)
        port().cpu_pairs(self.n, _p(self.xw), _p(self.qf), _p(self.types), self.c6.shape[0], _p(self.c6),
                         _p(self.c12), _p(self.box), s["cutoff"], s["beta"], O.COULOMB, self.width,
                         _p(self.counts), _p(self.nbr), _p(f), _p(e))
        terms = {"lj": e[0], "coulomb": e[1]}
        if s["pme"]:
            off, ex = self.rows
            if off is not None:
                port().cpu_excluded(self.n, _p(x), _p(self.q), _p(self.box), _p(off), _p(ex), s["beta"],
                                    O.COULOMB, _p(f), _p(e))
            terms["excluded"] = e[2]
            port().cpu_pme_spread(self.n, _p(x), _p(self.q), _p(self.box), _p(self.K), s["order"],
                                  _p(self.fixed), _p(self.grid))
            if reference_fft():
                terms["reciprocal"] = port().cpu_pme_reciprocal(_p(self.K), _p(self.grid), _p(self.spec),
                                                                _p(self.bc), _p(self.rowsum))
                phi = self.grid
            else:
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
    test rebuilds a 0.15 nm skin about this often for water at 300 K)."""
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
