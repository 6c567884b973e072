"""Seeded synthetic systems for the short-range nonbonded + PME path.

MDIR measures on the Amber benchmark suite and TIP3P boxes that are not
available here; these generators build boxes of the same shapes, sizes
and densities (nm, ps, kJ/mol, e, amu):

- `argon`: 864 atoms on an FCC 6x6x6 lattice, L = 3.47 nm, +-0.01 nm
  uniform jitter, sigma 0.3405 nm, epsilon 0.996 kJ/mol, cutoff 1.0 nm with
  the dispersion correction;
- `tip3p`: rigid TIP3P waters on a jittered cubic lattice at 33.4 nm^-3
  with uniformly random orientations (O-H 0.09572 nm, H-O-H 104.52 deg,
  q O -0.834 / H +0.417, LJ on O only: sigma 0.315061 nm, epsilon
  0.6364 kJ/mol), cutoff 0.9 nm, PME order 4, 0.1 nm spacing, Ewald
  tolerance 1e-5;
- `solvated_frame`: a water box plus 5% solute atoms with charges
  N(0, 0.3) e renormalised to zero net charge and LJ sigma U[0.25, 0.40] nm,
  epsilon U[0.2, 1.0] kJ/mol over 7 solute types (type 0 is the water
  oxygen, the last type the water hydrogen with epsilon 0).

A system is a dict; `positions` are float64 (n, 3)."""

import math

import numpy as np

COULOMB = float.fromhex("0x1.15def44ac2182p+7")
KB = 0.0083144626181532  # kJ/mol/K (R)


def ewald_beta(rc, tol):
    """beta with erfc(beta rc) = tol by bisection (MDIR
    lib/Driver/TermNonbonded.cpp:779-795)."""
    low, high = 0.0, 1.0
    while math.erfc(high * rc) > tol:
        high *= 2.0
    for _ in range(100):
        mid = 0.5 * (low + high)
        if math.erfc(mid * rc) > tol:
            low = mid
        else:
            high = mid
    return 0.5 * (low + high)


def smooth_size(least):
    """The smallest even 2,3,5,7-smooth size >= least
    (TermNonbonded.cpp:755-766)."""
    size = max(int(least), 2)
    while True:
        if size % 2 == 0:
            rest = size
            for f in (2, 3, 5, 7):
                while rest % f == 0:
                    rest //= f
            if rest == 1:
                return size
        size += 1


def pme_grid(box, spacing=0.1, order=4):
    return [max(smooth_size(int(math.ceil(L / spacing - 1e-9))), 2 * order) for L in box]


def _lb_tables(sig, eps):
    """Lorentz-Berthelot sigma/epsilon tables from per-type values."""
    sig = np.asarray(sig, dtype=np.float64)
    eps = np.asarray(eps, dtype=np.float64)
    return 0.5 * (sig[:, None] + sig[None, :]), np.sqrt(eps[:, None] * eps[None, :])


def argon(seed=1, jitter=0.01, cells=6, length=3.47, cutoff=1.0, skin=0.1):
    rng = np.random.default_rng(seed)
    a = length / cells
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    idx = np.array([[i, j, k] for i in range(cells) for j in range(cells) for k in range(cells)])
    x = ((idx[:, None, :] + base[None, :, :]).reshape(-1, 3) + 0.25) * a
    x = x + rng.uniform(-jitter, jitter, size=x.shape)
    n = len(x)
    sigma, epsilon = _lb_tables([0.3405], [0.996])
    return {
        "name": f"argon-{n}", "positions": x, "box": np.array([length] * 3),
        "charges": np.zeros(n), "types": np.zeros(n, dtype=np.int32), "sigma": sigma,
        "epsilon": epsilon, "masses": np.full(n, 39.948), "cutoff": cutoff,
        "reach": cutoff + skin, "pme": False, "beta": 0.0, "grid": None, "order": 4,
        "excluded_pairs": np.zeros((0, 2), dtype=np.int64), "dispersion": True, "waters": None,
    }


def _random_rotations(rng, m):
    q = rng.normal(size=(m, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.empty((m, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


ROH, THETA = 0.09572, math.radians(104.52)
Q_O, Q_H = -0.834, 0.417
SIG_O, EPS_O = 0.315061, 0.6364


def _water_sites(rng, centers):
    m = len(centers)
    local = np.array([[0.0, 0.0, 0.0],
                      [ROH * math.sin(THETA / 2), ROH * math.cos(THETA / 2), 0.0],
                      [-ROH * math.sin(THETA / 2), ROH * math.cos(THETA / 2), 0.0]])
    R = _random_rotations(rng, m)
    return centers[:, None, :] + np.einsum("mij,kj->mki", R, local)


def tip3p(waters=7850, density=33.4, seed=3, jitter=0.02, cutoff=0.9, skin=0.1, tol=1e-5,
          spacing=0.1, order=4):
    rng = np.random.default_rng(seed)
    L = (waters / density) ** (1.0 / 3.0)
    m = int(math.ceil(waters ** (1.0 / 3.0) - 1e-9))
    sites = np.array([[i, j, k] for i in range(m) for j in range(m) for k in range(m)], dtype=np.float64)
    pick = np.sort(rng.permutation(len(sites))[:waters])
    centers = (sites[pick] + 0.5) * (L / m) + rng.uniform(-jitter, jitter, size=(waters, 3))
    x = _water_sites(rng, centers).reshape(-1, 3)
    n = 3 * waters
    q = np.tile([Q_O, Q_H, Q_H], waters)
    types = np.tile([0, 1, 1], waters).astype(np.int32)
    sigma, epsilon = _lb_tables([SIG_O, 0.1], [EPS_O, 0.0])
    o = 3 * np.arange(waters)
    excl = np.concatenate([np.stack([o, o + 1], 1), np.stack([o, o + 2], 1), np.stack([o + 1, o + 2], 1)])
    box = np.array([L, L, L])
    return {
        "name": f"tip3p-{n}", "positions": x, "box": box, "charges": q, "types": types,
        "sigma": sigma, "epsilon": epsilon, "masses": np.tile([15.9994, 1.008, 1.008], waters),
        "cutoff": cutoff, "reach": cutoff + skin, "pme": True, "beta": ewald_beta(cutoff, tol),
        "grid": pme_grid(box, spacing, order), "order": order, "excluded_pairs": excl,
        "dispersion": False, "waters": np.stack([o, o + 1, o + 2], 1),
    }


def solvated_frame(atoms, seed, solute_fraction=0.05, solute_types=7, cutoff=0.9, skin=0.1,
                   tol=1e-5, spacing=0.1, order=4, water_density=100.2, table=None):
    """A cubic box at water density holding `atoms` atoms (a multiple of 3):
    waters, of which 5% of the atoms are replaced by solute atoms with
    random charges (zero net) and LJ types 1..solute_types.  `table`
    (per-type sigma, epsilon of the solute types) is drawn from the frame's
    seed when not given."""
    rng = np.random.default_rng(seed)
    assert atoms % 3 == 0
    waters = atoms // 3
    L = (atoms / water_density) ** (1.0 / 3.0)
    sysw = tip3p(waters=waters, density=waters / L ** 3, seed=int(rng.integers(1 << 30)),
                 cutoff=cutoff, skin=skin, tol=tol, spacing=spacing, order=order)
    n = atoms
    nsol = int(round(solute_fraction * n))
    nsol_mol = nsol // 3
    chosen = np.sort(rng.permutation(waters)[:nsol_mol])
    q = sysw["charges"].copy()
    types = sysw["types"].copy()
    nt = solute_types + 2
    types[types == 1] = nt - 1  # water hydrogen: last type
    sol_atoms = (3 * chosen[:, None] + np.arange(3)[None, :]).reshape(-1)
    qs = rng.normal(0.0, 0.3, size=len(sol_atoms))
    qs -= qs.mean()
    q[sol_atoms] = qs
    types[sol_atoms] = rng.integers(1, solute_types + 1, size=len(sol_atoms))
    if table is None:
        table = (rng.uniform(0.25, 0.40, solute_types), rng.uniform(0.2, 1.0, solute_types))
    sig = np.concatenate([[SIG_O], table[0], [0.1]])
    eps = np.concatenate([[EPS_O], table[1], [0.0]])
    sigma, epsilon = _lb_tables(sig, eps)
    q -= q.mean()  # exact zero net charge of the frame
    s = dict(sysw)
    s.update({"name": f"frame-{n}", "charges": q, "types": types.astype(np.int32), "sigma": sigma,
              "epsilon": epsilon, "type_sigma": sig, "type_epsilon": eps})
    return s


def batch_frames(count=256, low=1000, high=8000, seed=4, solute_types=7, **kw):
    """`count` solvated frames with atom counts uniform in [low, high],
    multiples of 3, sharing one LJ type table (8 types with LJ: the water
    oxygen and `solute_types` solute types drawn once for the batch)."""
    rng = np.random.default_rng(seed)
    sizes = 3 * rng.integers(low // 3, high // 3 + 1, size=count)
    table = (rng.uniform(0.25, 0.40, solute_types), rng.uniform(0.2, 1.0, solute_types))
    return [solvated_frame(int(a), seed=int(rng.integers(1 << 30)), solute_types=solute_types, table=table, **kw)
            for a in sizes]


def force_matching(frames=64, waters=7850, types=8, seed=5, jitter=0.005, perturb=0.02, perturb_seed=6, **kw):
    """The force-matching workload: `frames` copies of the TIP3P box with
    every coordinate jittered by N(0, jitter) nm, the oxygens assigned
    round-robin to `types` LJ types (all at the TIP3P oxygen values,
    Lorentz-Berthelot tables) and the hydrogens to one more type with
    epsilon 0.  Returns (system, positions (frames, n, 3), target), where
    target holds the per-type sigma / epsilon and the charges of the target
    forces: each value times (1 + perturb s), s a seeded sign pattern."""
    base = tip3p(waters=waters, **kw)
    n = 3 * waters
    t = np.empty(n, dtype=np.int32)
    t[0::3] = np.arange(waters) % types
    t[1::3] = types
    t[2::3] = types
    sig = np.array([SIG_O] * types + [0.1])
    eps = np.array([EPS_O] * types + [0.0])
    sigma, epsilon = _lb_tables(sig, eps)
    system = dict(base)
    system.update({"name": f"tip3p-{n}-fm{types}", "types": t, "sigma": sigma, "epsilon": epsilon,
                   "type_sigma": sig, "type_epsilon": eps})
    rng = np.random.default_rng(seed)
    X = base["positions"][None, :, :] + rng.normal(0.0, jitter, size=(frames, n, 3))
    rs = np.random.default_rng(perturb_seed)
    target = {"sigma": sig * (1.0 + perturb * rs.choice([-1.0, 1.0], size=sig.shape)),
              "epsilon": eps * (1.0 + perturb * rs.choice([-1.0, 1.0], size=eps.shape)),
              "charges": base["charges"] * (1.0 + perturb * rs.choice([-1.0, 1.0], size=n))}
    return system, X, target


def maxwell_velocities(system, temperature, seed=2):
    rng = np.random.default_rng(seed)
    m = np.asarray(system["masses"])
    v = rng.normal(size=(len(m), 3)) * np.sqrt(KB * temperature / m)[:, None]
    v -= (m[:, None] * v).sum(0) / m.sum()
    return v
