"""The entry point that allocates nothing, mdrtNbExcludedNoAlloc, against the
allocating path (mdrtNbForce with the pairs and PME switched off), called
through the C ABI twice in a row.

It is for callers that cannot allocate device memory (programs that own
all device memory through a fixed pool, loops that must not synchronize on
cudaFree): its scratch is a
fixed device array of the library, shared by every call.  This file sorts
last so that a run stopping at its first failure has run every other test."""
import ctypes

import numpy as np
import pytest
import torch

from mdir_b200 import COULOMB, NonbondedTerm, _lib, systems

pytestmark = pytest.mark.gpu

FORCE_RMS_TOL = 1e-5  # the tolerance of the force tests
ENERGY_TOL = 1e-6


def test_excluded_no_alloc_matches_the_allocating_path(cuda):
    s = systems.tip3p(waters=500, seed=41)
    n = len(s["charges"])
    t = NonbondedTerm(n)
    t.set_particles(s["charges"], s["types"], s["sigma"], s["epsilon"])
    t.set_exclusions(pairs=s["excluded_pairs"])
    t.set_interaction(s["cutoff"], s["reach"], s["beta"])
    x = torch.tensor(s["positions"], dtype=torch.float64, device="cuda")
    t.build(x, s["box"])
    f_ref = t.force(x, energy=True, pairs=False, pme=False).cpu().numpy()
    e = t.energies()
    w_ref = e["virial_pair"]

    pairs = torch.tensor(np.asarray(s["excluded_pairs"], dtype=np.int32), device="cuda")
    q = torch.tensor(s["charges"], dtype=torch.float64, device="cuda")
    box = np.ascontiguousarray(s["box"], dtype=np.float64)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    lib = _lib.lib()
    for call in range(2):  # the scratch keeps the last call's contents
        f = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
        ev = torch.full((7,), float("nan"), dtype=torch.float64, device="cuda")
        status = lib.mdrtNbExcludedNoAlloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(q.data_ptr()),
                                           ctypes.c_void_p(pairs.data_ptr()), len(pairs),
                                           box.ctypes.data_as(ctypes.c_void_p), s["beta"], COULOMB,
                                           ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(ev.data_ptr()), stream)
        assert status == _lib.OK, call
        got = f.cpu().numpy()
        rms = np.sqrt(np.mean(np.sum((got - f_ref) ** 2, 1)) / np.mean(np.sum(f_ref ** 2, 1)))
        assert rms < FORCE_RMS_TOL, (call, rms)
        ev = ev.cpu().numpy()
        assert abs(ev[0] - e["excluded"]) <= ENERGY_TOL * abs(e["excluded"]), (call, ev[0], e["excluded"])
        w = np.array([[ev[1], ev[4], ev[5]], [ev[4], ev[2], ev[6]], [ev[5], ev[6], ev[3]]])
        np.testing.assert_allclose(w, w_ref, rtol=1e-5, atol=1e-6 * np.abs(w_ref).max())


def test_excluded_no_alloc_refuses_more_pairs_than_its_scratch(cuda):
    lib = _lib.lib()
    x = torch.zeros((4, 3), dtype=torch.float64, device="cuda")
    q = torch.zeros(4, dtype=torch.float64, device="cuda")
    pairs = torch.zeros((1, 2), dtype=torch.int32, device="cuda")
    f = torch.zeros((4, 3), dtype=torch.float64, device="cuda")
    ev = torch.zeros(7, dtype=torch.float64, device="cuda")
    box = np.array([3.0, 3.0, 3.0])
    too_many = (1 << 20) + 1  # MDRT_NB_NOALLOC_MAX_PAIRS + 1: refused on the host, nothing launched
    status = lib.mdrtNbExcludedNoAlloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(q.data_ptr()),
                                       ctypes.c_void_p(pairs.data_ptr()), too_many,
                                       box.ctypes.data_as(ctypes.c_void_p), 3.0, COULOMB,
                                       ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(ev.data_ptr()), None)
    assert status == _lib.INVALID_ARGUMENT
