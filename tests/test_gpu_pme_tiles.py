"""The tiled PME spreading (bins of 8^3 grid points spread into tiles of
shared memory, then added to the grid; MDIR D282:
lib/Dialect/MDExec/DevicePolicy.cpp:105-124,
lib/Conversion/MDExecToGPU/PMESpreadTile.cpp; here a tuning choice in the
mixed mode) against the spreading by global atomics on the same inputs,
against the FP64 oracle, in a triclinic cell, at orders 4 to 8, and inside
the MD step."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from mdir_b200 import NonbondedTerm, systems
from mdir_b200.md import Integrator
from tests.test_gpu_triclinic import CELLS, charged_lattice

pytestmark = pytest.mark.gpu

# tiles against global atomics, both f32 sums in their own orders: the
# relative RMS force difference, the reciprocal energy and virial
AGREE_TOL = 1e-6
FORCE_RMS_TOL = 1e-5
ENERGY_TOL = 1e-6


def rms_rel(f, ref):
    return np.sqrt(np.mean(np.sum((f - ref) ** 2, 1))) / np.sqrt(np.mean(np.sum(ref ** 2, 1)))


def evaluate(s, spread, box=None, deterministic=False):
    t = NonbondedTerm(len(s["charges"]))
    t.set_particles(s["charges"], s["types"], s["sigma"], s["epsilon"])
    t.set_exclusions(pairs=s["excluded_pairs"])
    t.set_interaction(s["cutoff"], s["reach"], s["beta"])
    t.set_pme(s["grid"], s["order"])
    t.set_deterministic(deterministic)
    t.set_tuning(pme_spread=spread)
    b = list(s["box"]) if box is None else list(box)
    x = torch.tensor(s["positions"], device="cuda")
    t.build(x, b)
    f = t.force(x, b, energy=True).cpu().numpy()
    e = t.energies()
    t.close()
    return f, e


def agree(a, b):
    (fa, ea), (fb, eb) = a, b
    assert rms_rel(fa, fb) < AGREE_TOL
    assert abs(ea["reciprocal"] - eb["reciprocal"]) <= AGREE_TOL * abs(eb["reciprocal"])
    w = np.abs(eb["virial_reciprocal"]).max()
    np.testing.assert_allclose(ea["virial_reciprocal"], eb["virial_reciprocal"], rtol=0, atol=AGREE_TOL * w)


@pytest.mark.parametrize("order", [4, 5, 6, 8])
def test_tiles_agree_with_global_atomics(cuda, order):
    s = systems.tip3p(waters=900, seed=41)
    s["grid"], s["order"] = [40, 48, 36], order
    agree(evaluate(s, "tiles"), evaluate(s, "global"))


def test_tiles_on_a_large_grid_match_fp64(cuda):
    """A grid of 512,000 points, the size from which MDIR tiles."""
    s = systems.tip3p(waters=900, seed=42)
    s["grid"] = [80, 80, 80]
    tiles = evaluate(s, "tiles")
    agree(tiles, evaluate(s, "auto"))
    f, e = tiles
    ref = O.evaluate(s, s["positions"])
    assert rms_rel(f, ref["forces"]) < FORCE_RMS_TOL
    scale = sum(abs(v) for v in ref["terms"].values())
    assert abs(e["reciprocal"] - ref["terms"]["reciprocal"]) <= ENERGY_TOL * scale


@pytest.mark.parametrize("cell", CELLS)
def test_tiles_in_a_triclinic_cell(cuda, cell):
    s = charged_lattice(cell)
    s["grid"], s["order"] = (36, 36, 32), 4
    s["box"] = list(cell)
    tiles = evaluate(s, "tiles")
    agree(tiles, evaluate(s, "global"))
    ref = O.evaluate_triclinic(s, s["positions"], cell)
    assert rms_rel(tiles[0], ref["forces"]) < FORCE_RMS_TOL


def test_the_deterministic_mode_keeps_its_fixed_point_spreading(cuda):
    s = systems.tip3p(waters=900, seed=43)
    s["grid"] = [80, 80, 80]
    (f1, e1), (f2, e2) = evaluate(s, "tiles", deterministic=True), evaluate(s, "global", deterministic=True)
    assert np.array_equal(f1, f2) and e1["reciprocal"] == e2["reciprocal"]


def test_md_step_with_tiles(cuda):
    """The MD step's chain spreading through tiles: the forces of a first
    step against those of global atomics from the same state, and the lists
    and waters intact after 100 steps in graphs."""
    s = systems.tip3p(waters=700, seed=44)
    s["grid"] = [40, 40, 40]
    n = len(s["charges"])
    out = []
    for spread in ("tiles", "global"):
        t = NonbondedTerm(n)
        t.set_particles(s["charges"], s["types"], s["sigma"], s["epsilon"])
        t.set_exclusions(pairs=s["excluded_pairs"])
        t.set_interaction(s["cutoff"], s["reach"], s["beta"])
        t.set_pme(s["grid"], s["order"])
        t.set_tuning(pme_spread=spread)
        md = Integrator(t, s["masses"], s["waters"])
        md.thermostat(300.0, 0.1, 3)
        x = torch.tensor(s["positions"], device="cuda")
        v = torch.tensor(systems.maxwell_velocities(s, 300.0, seed=4), device="cuda")
        md.build(x, s["box"])
        md.run(x, v, s["box"], 0.002, 1, unroll=0)
        from tests.test_gpu_pme_fft import step_forces
        f = step_forces(md, n)
        md.run(x, v, s["box"], 0.002, 100, unroll=10)
        out.append((f, md.thermo()["steps"], t.status()))
        md.close()
        t.close()
    (ft, nt, st), (fg, ng, sg) = out
    assert nt == ng == 101 and st == sg == 0
    assert rms_rel(ft, fg) < AGREE_TOL
