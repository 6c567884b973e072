"""Forces, energies and virials of the device path against the FP64
oracle, and the pme.test known answer (MDIR test/Driver/pme.test:21-29)."""
import json
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import oracle as O
from mdir_b200 import NonbondedTerm, systems

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
# Tolerances of the mixed-precision path (f32 positions, pair arithmetic
# and grid) against FP64: the RMS relative force error, and each energy term
# within ENERGY_TOL of the scale of the potential (the sum of the absolute
# values of its terms): f32 positions alone move a term by about 1e-7 of it.
FORCE_RMS_TOL = 1e-5
ENERGY_TOL = 1e-6


def scale(terms):
    return sum(abs(v) for v in terms.values())


def make_term(s, deterministic=False):
    n = len(s["charges"])
    t = NonbondedTerm(n)
    t.set_particles(s["charges"], s["types"], s["sigma"], s["epsilon"])
    t.set_exclusions(pairs=s["excluded_pairs"])
    t.set_interaction(s["cutoff"], s["reach"], s["beta"], lj_switch=s.get("lj_switch", 0),
                      switch_distance=s.get("switch", 0.0))
    if s["pme"]:
        t.set_pme(s["grid"], s["order"])
    t.set_deterministic(deterministic)
    return t


def run(s, deterministic=False, potential=False):
    t = make_term(s, deterministic)
    x = torch.tensor(s["positions"], dtype=torch.float64, device="cuda")
    t.build(x, s["box"])
    f = t.force(x, energy=True, potential=potential)
    e = t.energies()
    out = {"forces": f.cpu().numpy(), "e": e, "const": t.constants(dispersion=s["dispersion"])}
    if potential:
        out["potential"] = t.potential().cpu().numpy()
    t.close()
    return out


def rms_rel(f, ref):
    return np.sqrt(np.mean(np.sum((f - ref) ** 2, 1))) / np.sqrt(np.mean(np.sum(ref ** 2, 1)))


def test_water_box_matches_fp64_oracle(cuda):
    s = systems.tip3p(waters=900)
    ref = O.evaluate(s, s["positions"])
    got = run(s)
    assert rms_rel(got["forces"], ref["forces"]) < FORCE_RMS_TOL
    e, c = got["e"], got["const"]
    for name, val in [("lj", e["lj"]), ("coulomb", e["coulomb"]), ("excluded", e["excluded"]),
                      ("reciprocal", e["reciprocal"])]:
        assert abs(val - ref["terms"][name]) <= ENERGY_TOL * scale(ref["terms"]), name
    assert c["self"] == pytest.approx(ref["terms"]["self"], rel=1e-12)
    W = e["virial_pair"] + e["virial_reciprocal"] + np.eye(3) * c["background"]
    np.testing.assert_allclose(W, ref["virial"], rtol=1e-5, atol=1e-3 * np.abs(ref["virial"]).max())


def test_argon_matches_fp64_oracle(cuda):
    s = systems.argon()
    ref = O.evaluate(s, s["positions"])
    got = run(s)
    assert rms_rel(got["forces"], ref["forces"]) < FORCE_RMS_TOL
    assert abs(got["e"]["lj"] - ref["terms"]["lj"]) <= ENERGY_TOL * scale(ref["terms"])
    assert got["const"]["dispersion"] == pytest.approx(ref["terms"]["dispersion"], rel=1e-12)


def test_opc_three_waters_pme_kat(cuda):
    fx = json.loads((GOLDEN / "opc_three.json").read_text())
    n = len(fx["charges_e"])
    res = np.array(fx["residue"])
    pairs = [(i, j) for i in range(n) for j in range(i + 1, n) if res[i] == res[j]]
    s = {"positions": np.array(fx["positions_nm"]), "box": np.array(fx["box_nm"]),
         "charges": np.array(fx["charges_e"]), "types": np.zeros(n, dtype=np.int32),
         "sigma": np.full((1, 1), 0.3), "epsilon": np.zeros((1, 1)), "cutoff": fx["cutoff_nm"],
         "reach": 1.0, "pme": True, "beta": fx["beta_per_nm"], "grid": fx["pme_grid"],
         "order": fx["pme_order"], "excluded_pairs": np.array(pairs), "dispersion": False}
    got = run(s)
    kcal = O.KJ_PER_KCAL
    exp = fx["pme_test_printed_kcal"]  # the digits pme.test checks
    # mixed precision: each term within ENERGY_TOL of the potential's scale
    # (f32 pair terms of about 860 kJ/mol cancel to -14 kcal/mol here)
    tol = ENERGY_TOL * scale(exp)
    assert got["e"]["coulomb"] / kcal == pytest.approx(exp["direct"], abs=tol)
    assert got["e"]["excluded"] / kcal == pytest.approx(exp["excluded"], abs=tol)
    assert got["e"]["reciprocal"] / kcal == pytest.approx(exp["reciprocal"], abs=tol)
    c = got["const"]
    # the host constants are FP64: every printed digit
    assert (c["self"] + c["background"]) / kcal == pytest.approx(exp["self"], abs=1e-6)


def test_deterministic_mode_is_bitwise_and_accurate(cuda):
    s = systems.tip3p(waters=600, seed=11)
    a = run(s, deterministic=True)
    b = run(s, deterministic=True)
    np.testing.assert_array_equal(a["forces"], b["forces"])
    for k in ("lj", "coulomb", "excluded", "reciprocal"):
        assert a["e"][k] == b["e"][k]
    ref = O.evaluate(s, s["positions"])
    assert rms_rel(a["forces"], ref["forces"]) < FORCE_RMS_TOL


def test_pme_potential_is_dE_dq(cuda):
    s = systems.tip3p(waters=400, seed=5)
    ref = O.evaluate(s, s["positions"], want_potential=True)
    got = run(s, potential=True)
    np.testing.assert_allclose(got["potential"], ref["potential"], rtol=1e-4,
                               atol=1e-5 * np.abs(ref["potential"]).max())


def test_argon_test_potential_on_the_device(cuda):
    """MDIR's test/Driver/argon.test:9-14 through the device path: the
    864-atom lattice of examples/argon with LJ switched from 0.75 to
    0.85 nm by the md dialect's quintic potential switch (lj_switch 2)
    gives the step-0 potential -1304.88... kcal/mol; forces against the
    FP64 oracle, also on positions moved into the switching region."""
    fx = json.loads((GOLDEN / "argon_lattice.json").read_text())
    x = np.array(fx["positions_nm"])
    n = len(x)
    s = {"positions": x, "charges": np.zeros(n), "types": np.zeros(n, dtype=np.int32),
         "sigma": np.array([[fx["sigma_nm"]]]), "epsilon": np.array([[fx["epsilon_kj_mol"]]]),
         "box": np.array(fx["box_nm"]), "cutoff": fx["cutoff_nm"], "reach": fx["cutoff_nm"] + 0.1,
         "pme": False, "beta": 0.0, "grid": None, "order": 4, "excluded_pairs": np.zeros((0, 2), dtype=np.int64),
         "dispersion": False, "lj_switch": 2, "switch": fx["switch_nm"]}
    got = run(s)
    kcal = got["e"]["lj"] / O.KJ_PER_KCAL
    assert f"{kcal:.6f}".startswith(fx["potential_kcal_mol_prefix"]), kcal
    ref = O.evaluate(s, x)
    assert abs(got["e"]["lj"] - ref["terms"]["lj"]) <= ENERGY_TOL * abs(ref["terms"]["lj"])
    # on the lattice the forces cancel to ~0.01 kJ/mol/nm by symmetry, so
    # they are compared where the atoms have moved off it
    rng = np.random.default_rng(2)
    s["positions"] = x + rng.uniform(-0.03, 0.03, size=x.shape)
    got = run(s)
    ref = O.evaluate(s, s["positions"])
    assert rms_rel(got["forces"], ref["forces"]) < FORCE_RMS_TOL
    assert abs(got["e"]["lj"] - ref["terms"]["lj"]) <= ENERGY_TOL * abs(ref["terms"]["lj"])
    # the two switches are different functions of r: the quintic is not the cubic in r^2
    s["lj_switch"] = 1
    cubic = run(s)["e"]["lj"]
    assert abs(cubic - got["e"]["lj"]) > 1e-3
