"""Triclinic cells: the device build against the oracle's canonical f32
pair test and MDIR's bit counts (test/Runtime/neighbors-groups-triclinic-
gpu.mlir), and the pair and excluded-pair forces against FP64."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.test_oracle import TRICLINIC_KAT, triclinic_case

pytestmark = pytest.mark.gpu


def canon(rows):
    rows = np.asarray(rows, dtype=np.int64)
    return rows[np.lexsort(tuple(rows[:, k] for k in range(rows.shape[1] - 1, -1, -1)))]


@pytest.mark.parametrize("cell,R,deg,poison,n,bits,several", TRICLINIC_KAT)
def test_triclinic_lists_are_the_oracle_set(cuda, cell, R, deg, poison, n, bits, several):
    from mdir_b200 import NonbondedTerm
    x, ex = triclinic_case(cell, R, deg, poison, n)
    t = NonbondedTerm(n)
    least = min(cell[:3])
    t.set_interaction(cutoff=min(R, 0.49 * least), reach=R, beta=0.0)
    if ex is not None:
        t.set_exclusions(rows=ex)
    xd = torch.tensor(x, dtype=torch.float64, device="cuda")
    sizes = t.build(xd, list(cell), allow_nan=poison)
    got = t.pair_images(sizes)
    assert len(got) == bits
    count, ref = O.pairset_triclinic_f32(x, cell, R, ex)
    assert count == bits
    np.testing.assert_array_equal(canon(got), canon(ref))
    assert sizes[4] == (1 if poison else 0)
    t.close()


def charged_lattice(cell, n_side=8, seed=3):
    """n_side^3 LJ sites on a jittered lattice of fractional coordinates in
    the cell, charges +-0.4 (neutral), the pairs (2k, 2k+1) excluded."""
    rng = np.random.default_rng(seed)
    g = (np.arange(n_side) + 0.5) / n_side
    f = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    f += rng.uniform(-0.02, 0.02, size=f.shape)
    H = O.cell_matrix(cell)
    x = f @ H + rng.integers(-2, 3, size=f.shape) @ H  # unwrapped by whole lattice vectors
    n = len(x)
    q = np.where(np.arange(n) % 2 == 0, 0.4, -0.4)
    return {"charges": q, "types": np.zeros(n, dtype=np.int32), "sigma": np.array([[0.30]]),
            "epsilon": np.array([[0.6]]), "excluded_pairs": np.stack([np.arange(0, n, 2), np.arange(1, n, 2)], 1),
            "cutoff": 0.9, "reach": 1.1, "beta": 3.12, "positions": x}


CELLS = [
    (3.6, 3.4, 3.1, -1.2, -1.5, -1.7),   # an octahedron-like cell, tilts of one sign
    (3.5, 3.5, 2.8, 0.0, 1.75, 1.75),    # a dodecahedron-like cell, tilts on the bounds
    (3.3, 3.0, 3.2, 1.1, -1.4, 0.9),     # tilts of both signs
]


@pytest.mark.parametrize("cell", CELLS)
@pytest.mark.parametrize("pruned", [0.0, 1.0])
def test_triclinic_pair_forces_match_fp64(cuda, cell, pruned):
    from mdir_b200 import NonbondedTerm
    s = charged_lattice(cell)
    n = len(s["charges"])
    t = NonbondedTerm(n)
    t.set_particles(s["charges"], s["types"], s["sigma"], s["epsilon"])
    t.set_exclusions(pairs=s["excluded_pairs"])
    t.set_interaction(s["cutoff"], s["reach"], s["beta"])
    if pruned:
        t.set_pruned_reach(pruned)
    xd = torch.tensor(s["positions"], dtype=torch.float64, device="cuda")
    t.build(xd, list(cell))
    if pruned:
        t.prune(xd, list(cell)[:3])
    f = t.force(xd, list(cell), energy=True).cpu().numpy()
    e = t.energies()
    ref = O.direct_triclinic(s, s["positions"], cell)
    err = np.sqrt(np.mean(np.sum((f - ref["forces"]) ** 2, 1)) / np.mean(np.sum(ref["forces"] ** 2, 1)))
    assert err < 1e-5, err
    scale = abs(ref["lj"]) + abs(ref["coulomb"]) + abs(ref["excluded"])
    for name in ("lj", "coulomb", "excluded"):
        assert abs(e[name] - ref[name]) <= 1e-6 * scale, (name, e[name], ref[name])
    t.close()


def test_triclinic_refusals(cuda):
    from mdir_b200 import NonbondedTerm, _lib
    s = charged_lattice(CELLS[0], n_side=4)
    n = len(s["charges"])
    t = NonbondedTerm(n)
    t.set_particles(s["charges"], s["types"], s["sigma"], s["epsilon"])
    t.set_interaction(0.8, 1.0, 3.0)
    xd = torch.tensor(s["positions"], dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.NativeError) as e:  # a tilt beyond the reduced form
        t.build(xd, [3.6, 3.4, 3.1, 2.0, 0.0, 0.0])
    assert e.value.status == _lib.INVALID_BOX
    t.build(xd, list(CELLS[0]))
    with pytest.raises(_lib.NativeError) as e:  # forces of a triclinic build in its own cell only
        t.force(xd, list(CELLS[0])[:3])
    assert e.value.status == _lib.INVALID_BOX
    g = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.NativeError) as e:  # the adjoint runs in orthorhombic cells
        t.parameter_gradient(xd, g, box=list(CELLS[0])[:3])
    assert e.value.status == _lib.UNSUPPORTED
    t.close()


@pytest.mark.parametrize("cell", CELLS)
def test_triclinic_pme_forces_and_energies_match_fp64(cuda, cell):
    """The whole term with SPME in a triclinic cell (fractional spreading
    and gathering, wave vectors H^-1 k) against the FP64 oracle."""
    from mdir_b200 import NonbondedTerm
    s = charged_lattice(cell)
    s["grid"], s["order"] = (36, 36, 32), 4
    n = len(s["charges"])
    t = NonbondedTerm(n)
    t.set_particles(s["charges"], s["types"], s["sigma"], s["epsilon"])
    t.set_exclusions(pairs=s["excluded_pairs"])
    t.set_interaction(s["cutoff"], s["reach"], s["beta"])
    t.set_pme(s["grid"], s["order"])
    xd = torch.tensor(s["positions"], dtype=torch.float64, device="cuda")
    t.build(xd, list(cell))
    f = t.force(xd, list(cell), energy=True).cpu().numpy()
    e = t.energies()
    ref = O.evaluate_triclinic(s, s["positions"], cell)
    err = np.sqrt(np.mean(np.sum((f - ref["forces"]) ** 2, 1)) / np.mean(np.sum(ref["forces"] ** 2, 1)))
    assert err < 1e-5, err
    scale = sum(abs(v) for v in ref["terms"].values())
    for name in ("lj", "coulomb", "excluded", "reciprocal"):
        assert abs(e[name] - ref["terms"][name]) <= 1e-6 * scale, (name, e[name], ref["terms"][name])
    c = t.constants(list(cell)[:3])
    assert abs(c["self"] - ref["terms"]["self"]) <= 1e-9 * abs(ref["terms"]["self"])
    t.close()


def test_frame_evaluator_in_a_triclinic_cell(cuda):
    """FrameEvaluator.evaluate(positions, tilts=...) gives the FP64 energies
    and forces of each frame in the triclinic cell."""
    from mdir_b200 import FrameEvaluator
    cell = CELLS[1]
    s = charged_lattice(cell)
    s["grid"], s["order"] = (36, 36, 32), 4
    s["box"] = np.array(cell[:3])
    rng = np.random.default_rng(5)
    frames = np.stack([s["positions"] + rng.normal(0, 0.002, s["positions"].shape) for _ in range(2)])
    ev = FrameEvaluator(s)
    res = ev.evaluate(frames, tilts=cell[3:], gradients=("positions",))
    for k in range(2):
        ref = O.evaluate_triclinic(s, frames[k], cell)
        assert abs(res.energy[k] - ref["energy"]) <= 1e-6 * sum(abs(v) for v in ref["terms"].values())
        f = -res.gradients["positions"][k].cpu().numpy()
        err = np.sqrt(np.mean(np.sum((f - ref["forces"]) ** 2, 1)) / np.mean(np.sum(ref["forces"] ** 2, 1)))
        assert err < 1e-5, err
    from mdir_b200.api import UnsupportedError
    with pytest.raises(UnsupportedError):
        ev.evaluate(frames, tilts=cell[3:])  # the tunables' gradient: orthorhombic cells only
