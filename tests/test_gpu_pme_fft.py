"""The library's own PME convolution (three kernels on grids whose every
dimension is 32, 64 or 128) against cuFFT's chain on the same inputs and
against the FP64 oracle; bitwise reproducibility in the deterministic mode;
the MD step's chain on both.

MDIR's reciprocal path: the spreading, cuFFT R2C, the influence multiply as
a cuFFT load callback, C2R and the gathering (runtime/mdrt_cuda.c:2942-2990,
runtime/pme_callback.cu:5-21)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from mdir_b200 import NonbondedTerm, systems
from mdir_b200.md import Integrator

pytestmark = pytest.mark.gpu

# own transforms against cuFFT's (both f32): relative RMS force difference,
# reciprocal energy and virial
AGREE_TOL = 1e-6
FORCE_RMS_TOL = 1e-5  # against FP64, as the other force tests
ENERGY_TOL = 1e-6


def rms_rel(f, ref):
    return np.sqrt(np.mean(np.sum((f - ref) ** 2, 1))) / np.sqrt(np.mean(np.sum(ref ** 2, 1)))


def term(s, fft, deterministic=False):
    t = NonbondedTerm(len(s["charges"]))
    t.set_particles(s["charges"], s["types"], s["sigma"], s["epsilon"])
    t.set_exclusions(pairs=s["excluded_pairs"])
    t.set_interaction(s["cutoff"], s["reach"], s["beta"])
    t.set_pme(s["grid"], s["order"])
    t.set_deterministic(deterministic)
    t.set_tuning(pme_fft=fft)
    return t


def evaluate(s, fft, deterministic=False, calls=1):
    t = term(s, fft, deterministic)
    x = torch.tensor(s["positions"], device="cuda")
    t.build(x, s["box"])
    out = []
    for _ in range(calls):
        f = t.force(x, energy=True).cpu().numpy()
        out.append((f, t.energies()))
    t.close()
    return out


GRIDS = [(64, 64, 64), (32, 64, 128), (128, 32, 64)]


@pytest.mark.parametrize("grid", GRIDS)
@pytest.mark.parametrize("deterministic", [False, True])
def test_own_transforms_agree_with_cufft(cuda, grid, deterministic):
    s = systems.tip3p(waters=900, seed=31)
    s["grid"] = list(grid)
    (fo, eo), = evaluate(s, "own", deterministic)
    (fc, ec), = evaluate(s, "cufft", deterministic)
    assert rms_rel(fo, fc) < AGREE_TOL
    assert abs(eo["reciprocal"] - ec["reciprocal"]) <= AGREE_TOL * abs(ec["reciprocal"])
    w = np.abs(ec["virial_reciprocal"]).max()
    np.testing.assert_allclose(eo["virial_reciprocal"], ec["virial_reciprocal"], rtol=0, atol=AGREE_TOL * w)
    for name in ("lj", "coulomb", "excluded"):
        if deterministic:
            assert eo[name] == ec[name], name
        else:
            assert eo[name] == pytest.approx(ec[name], rel=1e-6), name


@pytest.mark.parametrize("grid", [(32, 64, 128), (64, 32, 32)])
def test_own_transforms_match_fp64_oracle(cuda, grid):
    s = systems.tip3p(waters=900, seed=32)
    s["grid"] = list(grid)
    ref = O.evaluate(s, s["positions"])
    (f, e), = evaluate(s, "own")
    assert rms_rel(f, ref["forces"]) < FORCE_RMS_TOL
    scale = sum(abs(v) for v in ref["terms"].values())
    assert abs(e["reciprocal"] - ref["terms"]["reciprocal"]) <= ENERGY_TOL * scale


def test_deterministic_own_transforms_are_bitwise_and_empty_their_grid(cuda):
    """Two calls on one context (the second spreads into the grid the first
    one's forward plane kernel emptied) and a second context: all equal
    bit for bit."""
    s = systems.tip3p(waters=900, seed=33)
    s["grid"] = [64, 64, 64]
    runs = evaluate(s, "own", deterministic=True, calls=2) + evaluate(s, "own", deterministic=True)
    f0, e0 = runs[0]
    for f, e in runs[1:]:
        assert np.array_equal(f, f0)
        assert e["reciprocal"] == e0["reciprocal"]
        assert np.array_equal(e["virial_reciprocal"], e0["virial_reciprocal"])


def test_mixed_mode_calls_empty_their_grid(cuda):
    s = systems.tip3p(waters=900, seed=34)
    s["grid"] = [64, 64, 64]
    (f1, e1), (f2, e2) = evaluate(s, "own", calls=2)
    assert rms_rel(f2, f1) < 1e-6
    assert e2["reciprocal"] == pytest.approx(e1["reciprocal"], rel=1e-6)


def step_forces(md, n):
    import ctypes
    from mdir_b200.term import _cudart
    f = np.empty((n, 3))
    torch.cuda.synchronize()
    res = _cudart().cudaMemcpy(ctypes.c_void_p(f.ctypes.data), ctypes.c_void_p(md.forces()),
                               ctypes.c_size_t(f.nbytes), 2)
    assert int(res) == 0
    return f


@pytest.mark.parametrize("grid", [(32, 32, 32), (64, 64, 64)])
def test_md_chain_own_equals_cufft(cuda, grid):
    """The MD step's chain (spread, the three kernels, the update's gather)
    against the cuFFT chain, deterministic mode: the forces of a first step
    from the same state agree to the f32 roundings of the transforms, and
    after 40 more steps in graphs the trajectories are still that close.
    They separate as MD trajectories do: the f32 roundings of the two
    transforms (about 1e-7 of the reciprocal forces) grew to 2.2e-6 nm in the
    40 steps of a first run, so positions are held to 2e-5 nm."""
    s = systems.tip3p(waters=700, seed=35)
    s["grid"] = list(grid)
    n = len(s["charges"])
    out = []
    for fft in ("own", "cufft"):
        t = term(s, fft, deterministic=True)
        md = Integrator(t, s["masses"], s["waters"])
        md.thermostat(300.0, 0.1, 3)
        x = torch.tensor(s["positions"], device="cuda")
        v = torch.tensor(systems.maxwell_velocities(s, 300.0, seed=4), device="cuda")
        md.build(x, s["box"])
        md.run(x, v, s["box"], 0.002, 1, unroll=0)
        f = step_forces(md, n)
        md.run(x, v, s["box"], 0.002, 40, unroll=10)
        out.append((f, x.cpu().numpy(), md.thermo()["steps"]))
        md.close()
        t.close()
    (fo, xo, no), (fc, xc, nc) = out
    assert no == nc == 41
    assert rms_rel(fo, fc) < AGREE_TOL
    assert np.abs(xo - xc).max() < 2e-5
