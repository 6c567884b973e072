"""The oracle against MDIR's own known answers (CPU only)."""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"

# test/Runtime/neighbors-groups-gpu.mlir:508-630: (edge, reach, exclusion
# degree, poisoned particle 7, particles) -> bits of the lists.
GROUPS_KAT = [
    (12.0, 1.5, 0, False, 2000, 16352),
    (12.0, 1.5, 1, False, 2000, 16337),
    (12.0, 1.5, 9, False, 2000, 16200),
    (12.0, 1.5, 0, True, 2000, 16337),
    (7.0, 1.0, 0, False, 2000, 24389),
    (5.8, 0.8, 0, False, 2000, 21979),
    (4.0, 1.9, 0, False, 2000, 896816),
    (5.8, 3.19, 0, False, 2000, 1392935),
    (4.0, 2.4, 0, False, 320, 46145),
    (4.0, 3.0, 0, False, 320, 90433),
    (4.0, 3.6, 1, False, 320, 154718),
    (4.0, 3.9, 0, False, 320, 198183),
]


# test/Runtime/neighbors-groups-triclinic-gpu.mlir:636-812: the cell
# (ax, by, cz, bx, cx, cy), reach, exclusion degree, a position that is not
# a number, particles, the bits of the lists, the pairs with several images
# within the reach (the last line of each case, printed for the 320-particle
# cases)
_OCT = (12.0, 11.313708498984761, 9.797958971132712, -4.0, -4.0, -5.656854249492381)
_DODEC = (12.0, 12.0, 8.485281374238571, 0.0, 6.0, 6.0)
_SMALL = (4.2, 4.0, 3.9, 1.0, -1.5, 1.2)
_HEXA = (12.0, 10.392304845413264, 9.0, -6.0, 0.0, 0.0)
_NDODEC = (4.242640687119286, 4.242640687119286, 3.0, 0.0, 2.121320343559643, 2.121320343559643)
_NOCT = (3.6742346141747673, 3.4641016151377544, 3.0, -1.224744871391589, -1.224744871391589, -1.7320508075688772)
_NHEXA = (3.4641016151377544, 3.0, 3.2, -1.7320508075688772, 0.0, 0.0)
_NBOUNDS = (3.0, 3.0, 3.0, 1.5, -1.5, 1.5)
TRICLINIC_KAT = [
    (_OCT, 1.5, 0, False, 2000, 21149, None), (_OCT, 1.5, 1, False, 2000, 21125, None),
    (_OCT, 1.5, 9, False, 2000, 20953, None), (_OCT, 1.5, 0, True, 2000, 21132, None),
    (_DODEC, 1.5, 0, False, 2000, 23156, None), (_DODEC, 2.65, 0, False, 2000, 127147, None),
    (_SMALL, 1.9, 0, False, 2000, 875982, None), (_HEXA, 1.5, 0, False, 2000, 25088, None),
    (_NDODEC, 1.8, 0, False, 320, 22998, 0), (_NDODEC, 2.55, 1, False, 320, 65313, 15162),
    (_NDODEC, 2.925, 0, False, 320, 99408, 35791), (_NOCT, 1.8, 0, False, 320, 32533, 0),
    (_NOCT, 2.55, 1, False, 320, 92527, 33437), (_NOCT, 2.925, 0, False, 320, 140360, 46186),
    (_NHEXA, 1.8, 0, False, 320, 37351, 889), (_NHEXA, 2.55, 1, False, 320, 105866, 42846),
    (_NHEXA, 2.925, 0, False, 320, 161158, 50026), (_NBOUNDS, 1.8, 0, False, 320, 46107, 2703),
    (_NBOUNDS, 2.55, 1, False, 320, 130675, 45014), (_NBOUNDS, 2.925, 0, False, 320, 197964, 50644),
]


def triclinic_case(cell, R, deg, poison, n):
    x = O.lcg_positions_triclinic(n, cell)
    if poison:
        x[7, 0] = np.nan
    ex = O.chain_exclusions(n, deg) if deg else None
    return x, ex


@pytest.mark.parametrize("cell,R,deg,poison,n,bits,several", TRICLINIC_KAT)
def test_triclinic_pairset_matches_groups_kat(cell, R, deg, poison, n, bits, several):
    """The canonical f32 test of a triclinic build gives MDIR's bit counts;
    the f64 images within the reach give its counts of pairs with several."""
    x, ex = triclinic_case(cell, R, deg, poison, n)
    count, _ = O.pairset_triclinic_f32(x, cell, R, ex, want_list=False)
    assert count == bits
    if several is not None:
        _, _, multi = O.pairset_triclinic(x, cell, R, ex, want_list=False)
        assert multi == several


def lcg_case(L, R, deg, poison, n):
    x = O.lcg_positions(n, L)
    if poison:
        x[7, 0] = np.nan
    ex = O.chain_exclusions(n, deg) if deg else None
    return x, ex


@pytest.mark.parametrize("L,R,deg,poison,n,bits", GROUPS_KAT)
def test_pairset_matches_groups_kat(L, R, deg, poison, n, bits):
    x, ex = lcg_case(L, R, deg, poison, n)
    count, _ = O.pairset(x, [L, L, L], R, ex, want_list=False)
    assert count == bits


def test_pairset_covers_f64_reach():
    # every image within R in f64 has a bit; the extra bits are within R'
    L, R, n = 12.0, 1.5, 2000
    x = O.lcg_positions(n, L)
    count, pairs = O.pairset(x, [L, L, L], R)
    xw = x - np.floor(x / L) * L
    d = xw[pairs[:, 1]] - xw[pairs[:, 0]]
    code = pairs[:, 2]
    s = np.stack([code % 3 - 1, (code // 3) % 3 - 1, code // 9 - 1], 1)
    r = np.linalg.norm(d + s * L, axis=1)
    assert r.max() <= O.lib().orc_widened_reach(R, np.array([L, L, L]).ctypes.data) + 1e-6
    assert (r <= R).sum() == 16349  # neighbors-groups-gpu.mlir:37 (in f64)


def test_opc_three_waters_pme_kat():
    fx = json.loads((GOLDEN / "opc_three.json").read_text())
    x = np.array(fx["positions_nm"])
    q = np.array(fx["charges_e"])
    box = np.array(fx["box_nm"])
    res = np.array(fx["residue"])
    n = len(q)
    pairs = [(i, j) for i in range(n) for j in range(i + 1, n) if res[i] == res[j]]
    beta = fx["beta_per_nm"]
    exp = fx["expected_kcal"]
    en, _, _ = O.nonbonded(x, q, np.zeros(n, int), np.full((1, 1), 0.3), np.zeros((1, 1)), box,
                           fx["cutoff_nm"], beta, O.rows_from_pairs(n, pairs))
    assert en["coulomb"] / O.KJ_PER_KCAL == pytest.approx(exp["direct"], abs=1e-8)
    e_ex, _, _ = O.excluded(x, q, pairs, box, beta)
    assert e_ex / O.KJ_PER_KCAL == pytest.approx(exp["excluded"], abs=1e-7)
    e_rec, _, _, _ = O.pme(x, q, box, fx["pme_grid"], fx["pme_order"], beta)
    # pme.test: the reciprocal sum to its six digits with 64 points, order 8
    assert e_rec / O.KJ_PER_KCAL == pytest.approx(exp["reciprocal"], abs=2e-6)
    es = O.self_energy(q, beta) + O.background_energy(q, box, beta)
    assert es / O.KJ_PER_KCAL == pytest.approx(exp["self"], abs=1e-7)


def test_pme_matches_ewald_sum_and_forces_are_gradients():
    rng = np.random.default_rng(0)
    n, L = 40, 2.0
    x = rng.uniform(0, L, size=(n, 3))
    q = rng.normal(size=n)
    q -= q.mean()
    box = np.array([L, L, L])
    beta = 3.0
    e, f, W, pot = O.pme(x, q, box, [32, 32, 32], 8, beta)
    assert e == pytest.approx(O.ewald_sum_reciprocal(x, q, box, beta), rel=2e-6)
    h = 1e-5
    for i, k in [(0, 0), (3, 1), (7, 2)]:
        xp, xm = x.copy(), x.copy()
        xp[i, k] += h
        xm[i, k] -= h
        fd = -(O.pme(xp, q, box, [32, 32, 32], 8, beta)[0] - O.pme(xm, q, box, [32, 32, 32], 8, beta)[0]) / (2 * h)
        assert f[i, k] == pytest.approx(fd, rel=1e-5, abs=1e-6)
    # dE/dq by differences
    qp, qm = q.copy(), q.copy()
    qp[5] += 1e-6
    qm[5] -= 1e-6
    fdq = (O.pme(x, qp, box, [32, 32, 32], 8, beta)[0] - O.pme(x, qm, box, [32, 32, 32], 8, beta)[0]) / 2e-6
    assert pot[5] == pytest.approx(fdq, rel=1e-5)


def test_beta_and_grid_of_the_water_box():
    beta = O.ewald_beta(0.9, 1e-5)
    assert beta == pytest.approx(3.4705, abs=1e-4)
    assert math.erfc(beta * 0.9) == pytest.approx(1e-5, rel=1e-9)
    L = (7850 / 33.4) ** (1 / 3)
    assert O.pme_grid([L] * 3, 0.1, 4) == [64, 64, 64]
    assert O.pme_grid([22.008] * 3, 0.1, 4) == [224, 224, 224]


def test_triclinic_pme_is_the_ewald_sum_and_its_gradient():
    """SPME in a triclinic cell (fractional spreading, m = H^-1 k): the
    energy is the Ewald sum over wave vectors, the forces are its central
    differences, and with no tilts it is the orthorhombic SPME."""
    rng = np.random.default_rng(11)
    cell = (2.4, 2.2, 2.1, -0.8, 0.9, -1.0)
    H = O.cell_matrix(cell)
    n = 24
    x = rng.uniform(0, 1, size=(n, 3)) @ H
    q = rng.normal(0, 0.5, size=n)
    q -= q.mean()
    beta, K, order = 3.0, (48, 48, 48), 8
    e, f, W, pot = O.pme_triclinic(x, q, cell, K, order, beta)
    e_ref = O.ewald_sum_reciprocal_triclinic(x, q, cell, beta)
    assert abs(e - e_ref) < 1e-5 * abs(e_ref), (e, e_ref)
    h = 1e-5
    for i in (0, 7):
        for a in range(3):
            xp, xm = x.copy(), x.copy()
            xp[i, a] += h
            xm[i, a] -= h
            fd = -(O.pme_triclinic(xp, q, cell, K, order, beta)[0] - O.pme_triclinic(xm, q, cell, K, order, beta)[0]) / (2 * h)
            assert abs(f[i, a] - fd) < 1e-6 * max(1.0, np.abs(f).max()), (i, a, f[i, a], fd)
    box = (2.4, 2.2, 2.1)
    e0, f0, W0, p0 = O.pme(x, q, box, K, order, beta)
    e1, f1, W1, p1 = O.pme_triclinic(x, q, box + (0.0, 0.0, 0.0), K, order, beta)
    assert abs(e0 - e1) < 1e-12 * abs(e0)
    np.testing.assert_allclose(f1, f0, rtol=1e-10, atol=1e-10)


def test_prune_lists_restatement():
    """oracle.prune_lists against a scalar restatement entry by entry, with
    empty places, images, entries that lose every member, and all classes."""
    rng = np.random.default_rng(8)
    G, C = 3, 40
    f32 = np.float32
    cell = (2.9, 3.1, 3.3, 0.4, -0.6, 0.5)
    frames = rng.uniform(-0.7, 0.7, size=(16 * G, 4)).astype(np.float32)
    order = np.arange(16 * G, dtype=np.int32)
    order[[5, 21, 40]] = -1  # empty places
    entries = np.zeros((G, C, 2), dtype=np.int32)
    counts = np.array([40, 17, 0], dtype=np.int32)
    for g in range(G):
        for e in range(counts[g]):
            n = rng.choice([-1, 0, 1], size=3, p=[0.1, 0.8, 0.1]) + 16
            code = int(n[0]) | (int(n[1]) << 5) | (int(n[2]) << 10)
            mask = int(rng.integers(1, 1 << 16))
            entries[g, e] = (rng.integers(0, 16 * G), mask | (int(code) << 16))
    rin = 1.0
    got = O.prune_lists(entries, counts, frames, order, cell, rin)
    ax, by, cz, bx, cx, cy = cell
    Rw = rin + 3e-6 * (ax + by + cz + abs(bx) + abs(cx) + abs(cy))
    rin2 = f32(Rw * Rw)
    for g in range(G):
        rows = []
        for e in range(counts[g]):
            q, bits = int(entries[g, e, 0]), int(entries[g, e, 1]) & 0xFFFFFFFF
            code = (bits >> 16) & 0x7FFF
            na, nb, nc = (f32((code >> s) & 31) - f32(16) for s in (0, 5, 10))
            t = ((na * f32(ax) + nb * f32(bx)) + nc * f32(cx), nb * f32(by) + nc * f32(cy), nc * f32(cz))
            j = [frames[q, k] + t[k] for k in range(3)]
            inner = 0
            for m in range(16):
                if not (bits >> m) & 1 or order[16 * g + m] < 0:
                    continue
                d = [frames[16 * g + m, k] - j[k] for k in range(3)]
                if (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2] <= rin2:
                    inner |= 1 << m
            if inner:
                rows.append((bin(inner).count("1"), q, inner | (bits & 0x7FFF0000)))
        want = [(q, b) for c in range(6) for (pc, q, b) in rows if (0 if pc > 5 else pc) == c]
        assert [tuple(map(int, r)) for r in got[g]] == want
    assert sum(len(r) for r in got) > 0 and any(len(r) < counts[g] for g, r in enumerate(got))


def test_argon_lattice_potential_is_mdir_argon_test():
    """examples/argon (864 atoms, LJ switched from 7.5 to 8.5 Å by the md
    dialect's quintic potential switch): step-0 potential -1304.88...
    kcal/mol (test/Driver/argon.test:9-14; -5459.64 kJ/mol in
    examples/argon/argon.mlir); fixture from tests/golden/make_argon_lattice.py.
    The forces are the energy's central differences."""
    import json
    d = json.load(open(Path(__file__).resolve().parent / "golden" / "argon_lattice.json"))
    x = np.array(d["positions_nm"])
    n = len(x)
    s = {"charges": np.zeros(n), "types": np.zeros(n, dtype=np.int32), "sigma": np.array([[d["sigma_nm"]]]),
         "epsilon": np.array([[d["epsilon_kj_mol"]]]), "box": np.array(d["box_nm"]), "cutoff": d["cutoff_nm"],
         "reach": d["cutoff_nm"] + 0.1, "pme": False, "beta": 0.0, "grid": None, "order": 4,
         "excluded_pairs": np.zeros((0, 2), dtype=np.int64), "lj_switch": 2, "switch": d["switch_nm"]}
    r = O.evaluate(s, x)
    kcal = r["terms"]["lj"] / O.KJ_PER_KCAL
    assert f"{kcal:.6f}".startswith(d["potential_kcal_mol_prefix"]), kcal
    assert f"{r['terms']['lj']:.4f}".startswith(f"{d['potential_kj_mol_argon_mlir']:.2f}")
    # central differences on atoms moved into the switching region
    rng = np.random.default_rng(2)
    xj = x + rng.uniform(-0.03, 0.03, size=x.shape)
    f = O.evaluate(s, xj)["forces"]
    h = 1e-6
    for a in (0, 100, 500):
        for k in range(3):
            up, dn = xj.copy(), xj.copy()
            up[a, k] += h
            dn[a, k] -= h
            fd = -(O.evaluate(s, up)["terms"]["lj"] - O.evaluate(s, dn)["terms"]["lj"]) / (2 * h)
            assert abs(fd - f[a, k]) <= 1e-5 * max(1.0, abs(f[a, k])), (a, k, fd, f[a, k])
