"""FP64 CPU oracle of the short-range nonbonded + PME path (test infrastructure).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker.  It wraps oracle.c (pair sets, the
f64 pair term, B-spline spreading and gathering) and adds, in numpy, the
parts that MDIR computes on the host or through an FFT:

- the SPME influence function B C and the reciprocal energy and virial
  (docs/pme.md, Sections 1 and 1.2; lib/Conversion/MDExecToLoops/
  HostPMEConvolve.cpp), with numpy's FFT;
- beta by bisection of erfc(beta rc) = tol and the smooth grid size
  (lib/Driver/TermNonbonded.cpp:755-795 and 1104-1130);
- the self, background and dispersion-correction constants
  (TermNonbonded.cpp:601-637 and 651-668);
- the pruning of a dual list (lib/Conversion/MDExecToGPU/
  MDExecToGPU.cpp:9588, docs/neighbor-groups.md Section 6.2), restated in
  f32 on the lists and frames the device holds (`prune_lists`).

Units: nm, ps, kJ/mol, e.  COULOMB is MDIR's COULOMB_NATIVE
(scripts/mdir_physical_constants.py:16)."""

import ctypes
import math
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
COULOMB = float.fromhex("0x1.15def44ac2182p+7")
KJ_PER_KCAL = float.fromhex("0x1.0bc6a7ef9db23p+2")

_lib = None


def build():
    """Compiles liboracle.so and libcpu_port.so beside this file."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            build()
        _lib = ctypes.CDLL(str(path))
        d, i64, i32 = ctypes.c_double, ctypes.c_int64, ctypes.c_int32
        p = ctypes.c_void_p
        _lib.orc_pairset.restype = i64
        _lib.orc_pairset.argtypes = [i64, p, p, d, p, p, i64, p]
        _lib.orc_nonbonded.restype = None
        _lib.orc_nonbonded.argtypes = [i64, p, p, p, i32, p, p, p, d, d, d, i32, i32, d,
                                       p, p, p, p, p]
        _lib.orc_excluded.restype = None
        _lib.orc_excluded.argtypes = [i64, p, p, p, p, d, d, p, p, p]
        _lib.orc_pme_spread.argtypes = [i64, p, p, p, p, i32, p]
        _lib.orc_pme_gather.argtypes = [i64, p, p, p, p, i32, p, p, p]
        _lib.orc_bspline_moduli.argtypes = [i64, i32, p]
        _lib.orc_lcg_positions.argtypes = [i64, d, p]
        _lib.orc_widened_reach.restype = d
        _lib.orc_widened_reach.argtypes = [d, p]
        _lib.orc_lcg_positions_triclinic.argtypes = [i64, p, p]
        _lib.orc_widened_reach_triclinic.restype = d
        _lib.orc_widened_reach_triclinic.argtypes = [d, p]
        _lib.orc_pairset_triclinic.restype = i64
        _lib.orc_pairset_triclinic.argtypes = [i64, p, p, d, p, p, i32, i64, p, p]
        _lib.orc_pairset_triclinic_f32.restype = i64
        _lib.orc_pairset_triclinic_f32.argtypes = [i64, p, p, d, p, p, i32, i64, p]
        _lib.orc_nonbonded_triclinic.restype = None
        _lib.orc_nonbonded_triclinic.argtypes = [i64, p, p, p, i32, p, p, p, d, d, d, p, p, i32, p, p, p]
        _lib.orc_excluded_triclinic.restype = None
        _lib.orc_excluded_triclinic.argtypes = [i64, p, p, p, p, d, d, p, p, p]
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dtype):
    return None if a is None else np.ascontiguousarray(a, dtype=dtype)


# --------------------------------------------------------------------------
# Exclusions as ragged rows: offsets (n+1) and partners, each pair both ways.
# --------------------------------------------------------------------------
def rows_from_pairs(n, pairs):
    pairs = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    both = np.concatenate([pairs, pairs[:, ::-1]])
    order = np.lexsort((both[:, 1], both[:, 0]))
    both = both[order]
    counts = np.bincount(both[:, 0], minlength=n)
    off = np.zeros(n + 1, dtype=np.int32)
    off[1:] = np.cumsum(counts)
    return off, both[:, 1].astype(np.int32)


def lcg_positions(n, length):
    """The positions of MDIR's test/Runtime/neighbors-groups-gpu.mlir:47-80."""
    x = np.zeros((n, 3))
    lib().orc_lcg_positions(n, length, _ptr(x))
    return x


def lcg_positions_triclinic(n, cell):
    """The positions of MDIR's test/Runtime/neighbors-groups-triclinic-gpu.mlir:47-100
    in the cell (ax, by, cz, bx, cx, cy)."""
    x = np.zeros((n, 3))
    lib().orc_lcg_positions_triclinic(n, _ptr(_c(cell, np.float64)), _ptr(x))
    return x


def cell_matrix(cell):
    """The rows a, b, c of the lower-triangular cell (ax, by, cz, bx, cx, cy)."""
    ax, by, cz, bx, cx, cy = [float(v) for v in cell]
    return np.array([[ax, 0.0, 0.0], [bx, by, 0.0], [cx, cy, cz]])


def pairset_triclinic_f32(x, cell, reach, excl=None, want_list=True, span=3):
    """(count, rows (i, j, na, nb, nc)) of the canonical f32 pair test of a
    triclinic build (the widened reach; images relative to the raw
    positions); see oracle.c."""
    x = _c(x, np.float64)
    cell = _c(cell, np.float64)
    n = len(x)
    off, ex = (None, None) if excl is None else (_c(excl[0], np.int32), _c(excl[1], np.int32))
    count = lib().orc_pairset_triclinic_f32(n, _ptr(x), _ptr(cell), reach, _ptr(off), _ptr(ex), span, 0, None)
    if not want_list:
        return count, None
    out = np.zeros((max(count, 1), 5), dtype=np.int32)
    lib().orc_pairset_triclinic_f32(n, _ptr(x), _ptr(cell), reach, _ptr(off), _ptr(ex), span, count, _ptr(out))
    return count, out[:count]


def direct_triclinic(system, x, cell, span=2):
    """FP64 forces and energies of the pair term (every image within the
    cutoff) and of the excluded-pair correction in a triclinic cell, for a
    system dict as `evaluate` takes (no reciprocal, self or background
    terms): {"forces", "lj", "coulomb", "excluded", "virial"}."""
    x = _c(x, np.float64)
    cell = _c(cell, np.float64)
    n = len(x)
    q = _c(system["charges"], np.float64)
    t = _c(system["types"], np.int32)
    sig = _c(system["sigma"], np.float64)  # type-pair tables, as evaluate takes them
    eps = _c(system["epsilon"], np.float64)
    pairs = np.asarray(system.get("excluded_pairs", np.zeros((0, 2))), dtype=np.int32).reshape(-1, 2)
    off, ex = rows_from_pairs(n, pairs) if len(pairs) else (None, None)
    f = np.zeros((n, 3))
    e = np.zeros(2)
    w = np.zeros(9)
    lib().orc_nonbonded_triclinic(n, _ptr(x), _ptr(q), _ptr(t), sig.shape[0], _ptr(sig), _ptr(eps),
                                  _ptr(cell), system["cutoff"], system["beta"], system.get("coulomb", COULOMB),
                                  _ptr(None if off is None else _c(off, np.int32)),
                                  _ptr(None if ex is None else _c(ex, np.int32)), span, _ptr(f), _ptr(e), _ptr(w))
    ee = np.zeros(1)
    pp = _c(pairs, np.int32)
    lib().orc_excluded_triclinic(len(pp), _ptr(pp), _ptr(x), _ptr(q), _ptr(cell), system["beta"],
                                 system.get("coulomb", COULOMB), _ptr(f), _ptr(ee), _ptr(w))
    return {"forces": f, "lj": e[0], "coulomb": e[1], "excluded": ee[0], "virial": w.reshape(3, 3)}


def pairset_triclinic(x, cell, reach, excl=None, want_list=True, span=2):
    """(count, rows (i, j, na, nb, nc), pairs with several images) of every
    image of every pair within `reach` in f64 in a triclinic cell; see
    oracle.c."""
    x = _c(x, np.float64)
    cell = _c(cell, np.float64)
    n = len(x)
    off, ex = (None, None) if excl is None else (_c(excl[0], np.int32), _c(excl[1], np.int32))
    several = ctypes.c_int64(0)
    count = lib().orc_pairset_triclinic(n, _ptr(x), _ptr(cell), reach, _ptr(off), _ptr(ex), span, 0, None,
                                        ctypes.byref(several))
    if not want_list:
        return count, None, several.value
    out = np.zeros((max(count, 1), 5), dtype=np.int32)
    lib().orc_pairset_triclinic(n, _ptr(x), _ptr(cell), reach, _ptr(off), _ptr(ex), span, count, _ptr(out),
                                ctypes.byref(several))
    return count, out[:count], several.value


def prune_lists(entries, counts, frames, order, cell, pruned, sparse_bits=5):
    """The inner lists that a pruning leaves (MDIR: the inner mask = the
    outer mask and [r^2 <= R_in'^2] at the current frames, entries left with
    no member dropped; MDExecToGPU.cpp:9588), restated in f32 on the device's
    data: `entries` (G, C, 2) int32 outer entries (partner place, member bits
    | lattice-vector code << 16), `counts` (G,), `frames` (P, 4) f32 places,
    `order` (P,) atoms of the places (-1 empty), the cell (ax, by, cz[, bx, cx,
    cy]) and the pruned reach.  R_in' = R_in + 3e-6 (ax + by + cz + |bx| +
    |cx| + |cy|), squared in f64 and rounded to f32; the partner's image is
    its frame plus the lattice shift (na ax + nb bx) + nc cx, nb by + nc cy,
    nc cz; the distance is (m - j)^2 summed x, y then z; each of these f32
    operations rounded once.  Each list comes by member count, entries of
    more than `sparse_bits` members first, then 1, 2, ..., in the outer
    order within a count.  Returns a list of (n_g, 2) int64 arrays."""
    f32 = np.float32
    ax, by, cz, bx, cx, cy = (list(cell) + [0.0, 0.0, 0.0])[:6]
    Rw = pruned + 3e-6 * (ax + by + cz + abs(bx) + abs(cx) + abs(cy))
    rin2 = f32(Rw * Rw)
    frames = np.asarray(frames, dtype=np.float32)
    lists = []
    for g in range(len(counts)):
        ent = np.asarray(entries[g, : counts[g]])
        q = ent[:, 0].astype(np.int64)
        bits = ent[:, 1].astype(np.int64) & 0xFFFFFFFF
        live = int(sum(1 << m for m in range(16) if order[16 * g + m] >= 0))
        mask = bits & 0xFFFF & live
        code = (bits >> 16) & 0x7FFF
        na, nb, nc = (f32(v) for v in ((code & 31) - 16, ((code >> 5) & 31) - 16, ((code >> 10) & 31) - 16))
        tx = (na * f32(ax) + nb * f32(bx)) + nc * f32(cx)
        ty = nb * f32(by) + nc * f32(cy)
        tz = nc * f32(cz)
        jx, jy, jz = frames[q, 0] + tx, frames[q, 1] + ty, frames[q, 2] + tz
        inner = np.zeros(len(q), dtype=np.int64)
        for m in range(16):
            xm = frames[16 * g + m]
            dx, dy, dz = xm[0] - jx, xm[1] - jy, xm[2] - jz
            r2 = (dx * dx + dy * dy) + dz * dz
            inner |= (((mask >> m) & 1) & (r2 <= rin2)).astype(np.int64) << m
        keep = inner != 0
        kept = np.stack([q[keep], inner[keep] | (bits[keep] & 0x7FFF0000)], 1)
        pc = np.array([bin(int(v)).count("1") for v in inner[keep]], dtype=np.int64)
        cls = np.where(pc > sparse_bits, 0, pc)
        lists.append(np.concatenate([kept[cls == c] for c in range(sparse_bits + 1)])
                     if len(kept) else kept.reshape(0, 2))
    return lists


def chain_exclusions(n, degree):
    """The excluded pairs (i, (i + d) mod n), d = 1..degree, of
    neighbors-groups-gpu.mlir:200-260."""
    pairs = [(i, (i + d) % n) for i in range(n) for d in range(1, degree + 1)]
    pairs = {(min(a, b), max(a, b)) for a, b in pairs if a != b}
    return rows_from_pairs(n, sorted(pairs))


def pairset(x, box, reach, excl=None, want_list=True):
    """(count, array (count, 3) of (i, j, image code)) of the canonical f32
    pair test; see oracle.c."""
    x = _c(x, np.float64)
    box = _c(box, np.float64)
    n = len(x)
    off, ex = (None, None) if excl is None else (_c(excl[0], np.int32), _c(excl[1], np.int32))
    count = lib().orc_pairset(n, _ptr(x), _ptr(box), reach, _ptr(off), _ptr(ex), 0, None)
    if not want_list:
        return count, None
    out = np.zeros((max(count, 1), 3), dtype=np.int32)
    lib().orc_pairset(n, _ptr(x), _ptr(box), reach, _ptr(off), _ptr(ex), count, _ptr(out))
    return count, out[:count]


# --------------------------------------------------------------------------
# Ewald / PME parameters (TermNonbonded.cpp:755-795, 1104-1130)
# --------------------------------------------------------------------------
def ewald_beta(rc, tol):
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
    size = least
    while True:
        if size % 2 == 0:
            rest = size
            for f in (2, 3, 5, 7):
                while rest % f == 0:
                    rest //= f
            if rest == 1:
                return size
        size += 1


def pme_grid(box, spacing, order):
    return [max(smooth_size(int(math.ceil(L / spacing - 1e-9))), 2 * order) for L in box]


def bspline_moduli(K, order):
    out = np.zeros(K)
    lib().orc_bspline_moduli(K, order, _ptr(out))
    return out


def influence(box, K, order, beta, coulomb=COULOMB):
    """B C on the half-complex grid K0 x K1 x (K2//2 + 1), and the m vectors."""
    V = box[0] * box[1] * box[2]
    ms = []
    for a in range(3):
        idx = np.arange(K[a]) if a < 2 else np.arange(K[2] // 2 + 1)
        m = np.where(idx <= K[a] // 2, idx, idx - K[a]) / box[a]
        ms.append(m)
    mx, my, mz = np.meshgrid(ms[0], ms[1], ms[2], indexing="ij")
    m2 = mx * mx + my * my + mz * mz
    B = (bspline_moduli(K[0], order)[:, None, None] * bspline_moduli(K[1], order)[None, :, None]
         * bspline_moduli(K[2], order)[None, None, :K[2] // 2 + 1])
    with np.errstate(divide="ignore", invalid="ignore"):
        C = coulomb / (math.pi * V) * np.exp(-math.pi ** 2 * m2 / beta ** 2) / m2
    C[0, 0, 0] = 0.0
    return B * C, (mx, my, mz, m2)


def pme(x, q, box, K, order, beta, coulomb=COULOMB):
    """Reciprocal energy, forces (n, 3), virial (3, 3) and dE/dq (n,) by SPME."""
    x = _c(x, np.float64)
    q = _c(q, np.float64)
    box = _c(box, np.float64)
    Ka = np.asarray(K, dtype=np.int64)
    n = len(x)
    grid = np.zeros(tuple(K))
    lib().orc_pme_spread(n, _ptr(x), _ptr(q), _ptr(box), _ptr(Ka), order, _ptr(grid))
    bc, (mx, my, mz, m2) = influence(box, K, order, beta, coulomb)
    S = np.fft.rfftn(grid)
    power = (S.real ** 2 + S.imag ** 2)
    weight = np.full(bc.shape[2], 2.0)
    weight[0] = 1.0
    if K[2] % 2 == 0:
        weight[-1] = 1.0
    Em = 0.5 * bc * power * weight[None, None, :]
    energy = float(Em.sum())
    with np.errstate(divide="ignore", invalid="ignore"):
        f = -2.0 * (1.0 / m2 + math.pi ** 2 / beta ** 2)
    f[0, 0, 0] = 0.0
    mv = (mx, my, mz)
    W = np.zeros((3, 3))
    for a in range(3):
        for b in range(3):
            W[a, b] = float((Em * ((1.0 if a == b else 0.0) + f * mv[a] * mv[b])).sum())
    phi = np.fft.irfftn(bc * S, s=tuple(K), axes=(0, 1, 2)) * (K[0] * K[1] * K[2])
    phi = np.ascontiguousarray(phi)
    forces = np.zeros((n, 3))
    pot = np.zeros(n)
    lib().orc_pme_gather(n, _ptr(x), _ptr(q), _ptr(box), _ptr(Ka), order, _ptr(phi), _ptr(forces),
                         _ptr(pot))
    return energy, forces, W, pot


def pme_triclinic(x, q, cell, K, order, beta, coulomb=COULOMB):
    """SPME in a triclinic cell (ax, by, cz, bx, cx, cy): the spreading and
    gathering of `pme` on the fractional coordinates f = x H^-1, the wave
    vectors m = H^-1 k (the reciprocal vectors are the columns of H^-1),
    V = ax by cz; the gathered fractional forces taken to Cartesian ones by
    H^-1.  Returns (energy, forces, virial, dE/dq) as `pme`."""
    x = _c(x, np.float64)
    q = _c(q, np.float64)
    H = cell_matrix(cell)
    Hinv = np.linalg.inv(H)
    f = np.ascontiguousarray(x @ Hinv)
    unit = _c([1.0, 1.0, 1.0], np.float64)
    Ka = np.asarray(K, dtype=np.int64)
    n = len(x)
    grid = np.zeros(tuple(K))
    lib().orc_pme_spread(n, _ptr(f), _ptr(q), _ptr(unit), _ptr(Ka), order, _ptr(grid))
    V = float(cell[0] * cell[1] * cell[2])
    ks = []
    for a in range(3):
        idx = np.arange(K[a]) if a < 2 else np.arange(K[2] // 2 + 1)
        ks.append(np.where(idx <= K[a] // 2, idx, idx - K[a]).astype(np.float64))
    k0, k1, k2 = np.meshgrid(ks[0], ks[1], ks[2], indexing="ij")
    mx = Hinv[0, 0] * k0 + Hinv[0, 1] * k1 + Hinv[0, 2] * k2
    my = Hinv[1, 0] * k0 + Hinv[1, 1] * k1 + Hinv[1, 2] * k2
    mz = Hinv[2, 0] * k0 + Hinv[2, 1] * k1 + Hinv[2, 2] * k2
    m2 = mx * mx + my * my + mz * mz
    B = (bspline_moduli(K[0], order)[:, None, None] * bspline_moduli(K[1], order)[None, :, None]
         * bspline_moduli(K[2], order)[None, None, :K[2] // 2 + 1])
    with np.errstate(divide="ignore", invalid="ignore"):
        C = coulomb / (math.pi * V) * np.exp(-math.pi ** 2 * m2 / beta ** 2) / m2
    C[0, 0, 0] = 0.0
    bc = B * C
    S = np.fft.rfftn(grid)
    power = (S.real ** 2 + S.imag ** 2)
    weight = np.full(bc.shape[2], 2.0)
    weight[0] = 1.0
    if K[2] % 2 == 0:
        weight[-1] = 1.0
    Em = 0.5 * bc * power * weight[None, None, :]
    energy = float(Em.sum())
    with np.errstate(divide="ignore", invalid="ignore"):
        fm = -2.0 * (1.0 / m2 + math.pi ** 2 / beta ** 2)
    fm[0, 0, 0] = 0.0
    mv = (mx, my, mz)
    W = np.zeros((3, 3))
    for a in range(3):
        for b in range(3):
            W[a, b] = float((Em * ((1.0 if a == b else 0.0) + fm * mv[a] * mv[b])).sum())
    phi = np.ascontiguousarray(np.fft.irfftn(bc * S, s=tuple(K), axes=(0, 1, 2)) * (K[0] * K[1] * K[2]))
    ffrac = np.zeros((n, 3))
    pot = np.zeros(n)
    lib().orc_pme_gather(n, _ptr(f), _ptr(q), _ptr(unit), _ptr(Ka), order, _ptr(phi), _ptr(ffrac), _ptr(pot))
    return energy, ffrac @ Hinv.T, W, pot


def evaluate_triclinic(system, x, cell):
    """Every term of a system dict in a triclinic cell (pairs, excluded,
    reciprocal, self, background): as `evaluate`."""
    q = np.asarray(system["charges"], dtype=np.float64)
    d = direct_triclinic(system, x, cell)
    terms = {"lj": d["lj"], "coulomb": d["coulomb"], "excluded": d["excluded"]}
    forces = d["forces"].copy()
    W = d["virial"].copy()
    e_rec, f_rec, w_rec, pot = pme_triclinic(x, q, cell, system["grid"], system["order"], system["beta"])
    terms["reciprocal"] = e_rec
    forces += f_rec
    W += w_rec
    terms["self"] = self_energy(q, system["beta"])
    eb = background_energy(q, cell[:3], system["beta"])
    terms["background"] = eb
    W += np.eye(3) * eb
    return {"energy": sum(terms.values()), "terms": terms, "forces": forces, "virial": W, "potential": pot}


def ewald_sum_reciprocal(x, q, box, beta, coulomb=COULOMB, gauss=1e-18):
    """The reciprocal energy by the Ewald sum over wave vectors (the method of
    test/Driver/Inputs/ewald_reference.py), for small systems."""
    x = np.asarray(x, dtype=np.float64)
    q = np.asarray(q, dtype=np.float64)
    V = box[0] * box[1] * box[2]
    limit = beta * math.sqrt(-math.log(gauss)) / math.pi
    kmax = [int(limit * box[k]) + 1 for k in range(3)]
    e = 0.0
    for a in range(0, kmax[0] + 1):
        for b in range(-kmax[1], kmax[1] + 1):
            for c in range(-kmax[2], kmax[2] + 1):
                if a == 0 and (b < 0 or (b == 0 and c <= 0)):
                    continue
                m = np.array([a / box[0], b / box[1], c / box[2]])
                m2 = float(m @ m)
                if m2 > limit * limit:
                    continue
                ph = 2 * math.pi * (x @ m)
                re, im = float(q @ np.cos(ph)), float(q @ np.sin(ph))
                e += 2 * coulomb / (2 * math.pi * V) * math.exp(-math.pi ** 2 * m2 / beta ** 2) / m2 * (re * re + im * im)
    return e


def ewald_sum_reciprocal_triclinic(x, q, cell, beta, coulomb=COULOMB, gauss=1e-18):
    """The reciprocal energy by the Ewald sum over the wave vectors m = H^-1 k
    of a triclinic cell, for small systems (the check of pme_triclinic)."""
    x = np.asarray(x, dtype=np.float64)
    q = np.asarray(q, dtype=np.float64)
    H = cell_matrix(cell)
    Hinv = np.linalg.inv(H)
    V = float(cell[0] * cell[1] * cell[2])
    limit = beta * math.sqrt(-math.log(gauss)) / math.pi
    # |k_a| <= limit |a| bounds every k with |m| <= limit (m . a = k_a)
    kmax = [int(limit * np.linalg.norm(H[a])) + 1 for a in range(3)]
    e = 0.0
    for a in range(0, kmax[0] + 1):
        for b in range(-kmax[1], kmax[1] + 1):
            for c in range(-kmax[2], kmax[2] + 1):
                if a == 0 and (b < 0 or (b == 0 and c <= 0)):
                    continue
                m = Hinv @ np.array([a, b, c], dtype=np.float64)
                m2 = float(m @ m)
                if m2 > limit * limit:
                    continue
                ph = 2 * math.pi * (x @ m)
                re, im = float(q @ np.cos(ph)), float(q @ np.sin(ph))
                e += 2 * coulomb / (2 * math.pi * V) * math.exp(-math.pi ** 2 * m2 / beta ** 2) / m2 * (re * re + im * im)
    return e


def self_energy(q, beta, coulomb=COULOMB):
    return -coulomb * beta / math.sqrt(math.pi) * float(np.sum(np.asarray(q) ** 2))


def background_energy(q, box, beta, coulomb=COULOMB):
    V = box[0] * box[1] * box[2]
    Q = float(np.sum(q))
    return -coulomb * math.pi * Q * Q / (2.0 * V * beta * beta)


def dispersion_energy(types, sigma, epsilon, excluded_pairs, box, rc):
    """E_disp = -2 pi N^2 <C6> / (3 V rc^3), <C6> over the distinct pairs that
    are not excluded (TermNonbonded.cpp:613-637); its virial is 2 E_disp on
    each diagonal entry."""
    types = np.asarray(types)
    nt = sigma.shape[0]
    counts = np.bincount(types, minlength=nt).astype(np.float64)
    c6 = 4.0 * epsilon * sigma ** 6
    s = float(counts @ c6 @ counts - np.sum(counts * np.diag(c6)))
    for i, j in excluded_pairs:
        s -= 2.0 * c6[types[i], types[j]]
    n = float(len(types))
    pairs = n * (n - 1.0) - 2.0 * len(excluded_pairs)
    mean = s / pairs if pairs > 0 else 0.0
    V = box[0] * box[1] * box[2]
    return -2.0 * math.pi / (3.0 * V) * n * n * mean / rc ** 3


def nonbonded(x, q, types, sigma, epsilon, box, rc, beta, excl=None, coulomb=COULOMB,
              coulomb_shift=False, lj_switch=False, rs=0.0):
    """f64 LJ + Ewald direct: (energies {'lj', 'coulomb'}, forces, virial).
    lj_switch: False / 0 none, True / 1 the cubic switch in r^2 (MDIR's
    SQUARED_DISTANCE_SWITCH modifier, TermLennardJones.cpp:72-95), 2 the
    potential switch of MDIR's md dialect, quintic in r (ExpandTruncation.cpp:
    19-46), both from rs to rc."""
    x = _c(x, np.float64)
    q = _c(q, np.float64)
    t = _c(types, np.int32)
    sg = _c(sigma, np.float64)
    ep = _c(epsilon, np.float64)
    box = _c(box, np.float64)
    n = len(x)
    off, ex = (None, None) if excl is None else (_c(excl[0], np.int32), _c(excl[1], np.int32))
    forces = np.zeros((n, 3))
    energies = np.zeros(2)
    W = np.zeros(9)
    lib().orc_nonbonded(n, _ptr(x), _ptr(q), _ptr(t), sg.shape[0], _ptr(sg), _ptr(ep), _ptr(box),
                        rc, beta, coulomb, int(coulomb_shift), int(lj_switch), rs, _ptr(off),
                        _ptr(ex), _ptr(forces), _ptr(energies), _ptr(W))
    return {"lj": energies[0], "coulomb": energies[1]}, forces, W.reshape(3, 3)


def excluded(x, q, pairs, box, beta, coulomb=COULOMB):
    x = _c(x, np.float64)
    q = _c(q, np.float64)
    p = _c(np.asarray(pairs).reshape(-1, 2), np.int32)
    box = _c(box, np.float64)
    forces = np.zeros((len(x), 3))
    e = np.zeros(1)
    W = np.zeros(9)
    lib().orc_excluded(len(p), _ptr(p), _ptr(x), _ptr(q), _ptr(box), beta, coulomb,
                       _ptr(forces), _ptr(e), _ptr(W))
    return float(e[0]), forces, W.reshape(3, 3)


def evaluate(system, x, want_potential=False):
    """Every term of a system dict (see mdir_b200.systems) at positions x:
    returns dict with 'energy' (total), 'terms', 'forces' (n, 3), 'virial'."""
    box = np.asarray(system["box"], dtype=np.float64)
    q = np.asarray(system["charges"], dtype=np.float64)
    rc = system["cutoff"]
    pairs = np.asarray(system["excluded_pairs"]).reshape(-1, 2)
    rows = rows_from_pairs(len(q), pairs) if len(pairs) else None
    pme_on = system.get("pme", True)
    beta = system["beta"] if pme_on else 0.0
    terms = {}
    en, forces, W = nonbonded(x, q, system["types"], system["sigma"], system["epsilon"], box, rc,
                              beta, rows, coulomb_shift=system.get("coulomb_shift", False),
                              lj_switch=system.get("lj_switch", False), rs=system.get("switch", 0.0))
    terms.update(en)
    pot = None
    if pme_on:
        e_ex, f_ex, w_ex = excluded(x, q, pairs, box, beta)
        terms["excluded"] = e_ex
        forces += f_ex
        W += w_ex
        e_rec, f_rec, w_rec, pot = pme(x, q, box, system["grid"], system["order"], beta)
        terms["reciprocal"] = e_rec
        forces += f_rec
        W += w_rec
        terms["self"] = self_energy(q, beta)
        eb = background_energy(q, box, beta)
        terms["background"] = eb
        W += np.eye(3) * eb
    if system.get("dispersion", False):
        ed = dispersion_energy(np.asarray(system["types"]), np.asarray(system["sigma"]),
                               np.asarray(system["epsilon"]), pairs, box, rc)
        terms["dispersion"] = ed
        W += np.eye(3) * 2.0 * ed
    out = {"energy": sum(terms.values()), "terms": terms, "forces": forces, "virial": W}
    if want_potential:
        out["potential"] = pot
    return out
