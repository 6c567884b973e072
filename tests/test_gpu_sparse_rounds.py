"""Pruned (inner) lists hold their entries by member count, and the pair
kernel evaluates the entries of at most NB_SPARSE_BITS members member by
member (its sparse rounds).  Forces, energies and virial over such lists
must be those of the same pairs over one list, and the FP64 oracle's."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from mdir_b200 import NonbondedTerm, systems
from mdir_b200.frames import lorentz_berthelot

pytestmark = pytest.mark.gpu


def _term(s, sigma, epsilon, reach, pruned, deterministic):
    t = NonbondedTerm(len(s["charges"]))
    t.set_particles(s["charges"], s["types"], sigma, epsilon)
    t.set_exclusions(pairs=s["excluded_pairs"])
    t.set_interaction(s["cutoff"], reach, s["beta"])
    t.set_pme(s["grid"], s["order"])
    if deterministic:
        t.set_deterministic(True)
    if pruned:
        t.set_pruned_reach(pruned)
    return t


@pytest.mark.parametrize("table", [False, True])
@pytest.mark.parametrize("deterministic", [False, True])
def test_pruned_lists_give_the_forces_of_one_list(cuda, table, deterministic):
    s, X, target = systems.force_matching(frames=1, waters=1500)
    # one LJ type for all oxygens (the factor form of the pair kernel), or
    # 8 types at perturbed values (the table form)
    sig, eps = (target["sigma"], target["epsilon"]) if table else (s["type_sigma"], s["type_epsilon"])
    sigma, epsilon = lorentz_berthelot(sig, eps)
    box = list(s["box"])
    xd = torch.tensor(X[0], device=cuda)
    out = []
    for reach, pruned in ((1.0, 0.0), (1.4, 1.0)):
        t = _term(s, sigma, epsilon, reach, pruned, deterministic)
        t.build(xd, box)
        if pruned:
            t.prune(xd, box)
        f = t.force(xd, energy=True).cpu().numpy()
        out.append((f, t.energies()))
        if deterministic:  # bitwise again
            f2 = t.force(xd, energy=True).cpu().numpy()
            np.testing.assert_array_equal(f, f2)
        t.close()
    (f1, e1), (f2, e2) = out
    scale = np.sqrt(np.mean(np.sum(f1 ** 2, 1)))
    assert np.max(np.abs(f1 - f2)) <= 1e-5 * scale
    c = dict(s)
    c["sigma"], c["epsilon"] = sigma, epsilon
    ref = O.evaluate(c, X[0])
    err = np.sqrt(np.mean(np.sum((f2 - ref["forces"]) ** 2, 1)) / np.mean(np.sum(ref["forces"] ** 2, 1)))
    assert err < 1e-5, err
    # the real-space Coulomb sum is a small difference of large pair terms:
    # energies are held to 1e-6 of the terms' magnitudes
    terms = ref["terms"]
    scale = abs(terms["lj"]) + abs(terms["coulomb"]) + abs(terms["excluded"])
    for k in ("lj", "coulomb"):
        assert abs(e1[k] - e2[k]) <= 1e-6 * scale, (k, e1[k], e2[k])
        assert abs(e2[k] - terms[k]) <= 1e-6 * scale, (k, e2[k], terms[k])
    w1, w2 = e1["virial_pair"], e2["virial_pair"]
    assert np.max(np.abs(w1 - w2)) <= 1e-6 * np.max(np.abs(w1))


@pytest.mark.parametrize("case", ["water", "triclinic"])
def test_pruned_lists_are_the_host_restatement(cuda, case):
    """Bit for bit: the inner lists after a pruning equal the oracle's
    restatement of the pruning's f32 test (oracle.prune_lists), in its
    order, at the build's positions and again after the atoms moved."""
    from mdir_b200 import _lib as L
    if case == "water":
        s = systems.tip3p(waters=1500, seed=11)
        cell = list(s["box"])
    else:
        from tests.test_gpu_triclinic import CELLS, charged_lattice
        cell = list(CELLS[0])
        s = charged_lattice(cell)
    n = len(s["charges"])
    t = NonbondedTerm(n)
    t.set_particles(s["charges"], s["types"], s["sigma"], s["epsilon"])
    t.set_exclusions(pairs=s["excluded_pairs"])
    rin = 1.0
    t.set_interaction(0.9, 1.25 if case == "water" else 1.1, 0.0)
    t.set_pruned_reach(rin)
    x = np.asarray(s["positions"], dtype=np.float64)
    rng = np.random.default_rng(4)
    for step in range(2):
        xd = torch.tensor(x, device=cuda)
        if step == 0:
            sizes = t.build(xd, cell)
        t.prune(xd, cell[:3])
        torch.cuda.synchronize()
        cap = t.info()["list_capacity"]
        G = int(sizes[L.SIZE_GROUPS])
        ref = O.prune_lists(t.buffer(L.SLOT_ENTRIES, np.int32, 2)[: G * cap].reshape(G, cap, 2),
                            t.buffer(L.SLOT_COUNTS, np.int32)[:G], t.buffer(L.SLOT_PLACED, np.float32, 4),
                            t.buffer(L.SLOT_ORDER, np.int32), cell, rin)
        got_c = t.buffer(L.SLOT_INNER_COUNTS, np.int32)[:G]
        got_e = t.buffer(L.SLOT_INNER_ENTRIES, np.int32, 2)[: G * cap].reshape(G, cap, 2)
        assert sum(len(r) for r in ref) > 0
        for g in range(G):
            assert got_c[g] == len(ref[g]), (step, g)
            got = got_e[g, : got_c[g]].astype(np.int64)
            got[:, 1] &= 0xFFFFFFFF
            np.testing.assert_array_equal(got, ref[g])
        x = x + rng.normal(0.0, 0.01, size=x.shape)  # within half the skin of the build
    t.close()


def test_pruning_in_the_pair_kernel_is_the_pruning_then_the_pairs(cuda):
    """MDRT_NB_PRUNE on a force call: the pruning and the pairs of the fresh
    inner lists in one kernel (MDIR D284) leave the inner lists of the
    pruning kernel bit for bit, and the forces of pruning then pairing."""
    from mdir_b200 import _lib as L
    s = systems.tip3p(waters=1500, seed=17)
    box = list(s["box"])
    x0 = np.asarray(s["positions"])
    x1 = x0 + np.random.default_rng(6).normal(0.0, 0.01, size=x0.shape)

    def term():
        t = NonbondedTerm(len(s["charges"]))
        t.set_particles(s["charges"], s["types"], s["sigma"], s["epsilon"])
        t.set_exclusions(pairs=s["excluded_pairs"])
        t.set_interaction(s["cutoff"], 1.3, s["beta"])
        t.set_pruned_reach(1.0)
        t.set_pme(s["grid"], s["order"])
        sizes = t.build(torch.tensor(x0, device=cuda), box)
        return t, int(sizes[L.SIZE_GROUPS])

    (a, G), (b, _) = term(), term()
    for x in (x0, x1):
        xd = torch.tensor(x, device=cuda)
        a.prune(xd, box)
        fa = a.force(xd).cpu().numpy()
        fb = b.force(xd, prune=True).cpu().numpy()
        ca = a.buffer(L.SLOT_INNER_COUNTS, np.int32)[:G]
        cb = b.buffer(L.SLOT_INNER_COUNTS, np.int32)[:G]
        np.testing.assert_array_equal(ca, cb)
        cap = a.info()["list_capacity"]
        ea = a.buffer(L.SLOT_INNER_ENTRIES, np.int32, 2)
        eb = b.buffer(L.SLOT_INNER_ENTRIES, np.int32, 2)
        for g in range(G):
            np.testing.assert_array_equal(ea[g * cap: g * cap + ca[g]], eb[g * cap: g * cap + cb[g]])
        err = np.sqrt(np.mean(np.sum((fb - fa) ** 2, 1)) / np.mean(np.sum(fa ** 2, 1)))
        assert err < 1e-6, err
        ref = O.evaluate(s, x)["forces"]
        assert np.sqrt(np.mean(np.sum((fb - ref) ** 2, 1)) / np.mean(np.sum(ref ** 2, 1))) < 1e-5
        # the next force call without a pruning reads the inner lists and units the kernel left
        fc = b.force(xd).cpu().numpy()
        assert np.sqrt(np.mean(np.sum((fc - fa) ** 2, 1)) / np.mean(np.sum(fa ** 2, 1))) < 1e-6
    a.close()
    b.close()


def test_md_step_with_the_pruning_in_the_pair_kernel(cuda):
    """The MD step with its prunings inside the pair kernel (tuning
    fused_prune 1) follows the step with a pruning launch of its own (2):
    the same prunings and rebuilds, and positions that part no faster than
    two runs of the step with its own pruning launch part from each other
    (f32 sums in the order the atomics land, amplified by the dynamics)."""
    from mdir_b200.md import Integrator
    s = systems.tip3p(waters=1500, seed=19)
    out = []
    for fused in (2, 2, 1):
        t = NonbondedTerm(len(s["charges"]))
        t.set_particles(s["charges"], s["types"], s["sigma"], s["epsilon"])
        t.set_exclusions(pairs=s["excluded_pairs"])
        t.set_interaction(s["cutoff"], 1.3, s["beta"])
        t.set_pruned_reach(0.95)
        t.set_pme(s["grid"], s["order"])
        t.set_tuning(fused_prune=fused)
        md = Integrator(t, s["masses"], s["waters"])
        md.thermostat(300.0, 0.0, 1)
        x = torch.tensor(s["positions"], device=cuda)
        v = torch.tensor(systems.maxwell_velocities(s, 300.0, seed=2), device=cuda)
        md.build(x, s["box"])
        md.run(x, v, s["box"], 0.002, 60, unroll=10)
        th = md.thermo()
        out.append((x.cpu().numpy(), th["prunes"], th["builds"]))
        assert t.status() == 0
    (xa, pa, ba), (xc, pc, bc), (xb, pb, bb) = out
    assert pa == pb == pc and pa >= 10 and ba == bb == bc
    control = np.abs(xa - xc).max()
    assert np.abs(xa - xb).max() < 1e-4 or np.abs(xa - xb).max() < 10 * control, (np.abs(xa - xb).max(), control)


@pytest.mark.parametrize("deterministic", [False, True])
def test_staging_depth_changes_no_force(cuda, deterministic):
    """The pair kernel's staging depth 2 (the next unit's entries in flight)
    gives the forces and energies of depth 1: bit for bit in the
    deterministic mode, to the order of f32 sums otherwise."""
    s = systems.tip3p(waters=1500, seed=23)
    box = list(s["box"])
    xd = torch.tensor(s["positions"], device=cuda)
    out = []
    for depth in (1, 2):
        t = _term(s, s["sigma"], s["epsilon"], 1.3, 1.0, deterministic)
        t.set_tuning(staging_depth=depth)
        t.build(xd, box)
        t.prune(xd, box)
        f = t.force(xd, energy=True).cpu().numpy()
        out.append((f, t.energies()))
        t.close()
    (f1, e1), (f2, e2) = out
    if deterministic:
        np.testing.assert_array_equal(f1, f2)
        assert e1["lj"] == e2["lj"] and e1["coulomb"] == e2["coulomb"]
    else:
        assert np.sqrt(np.mean(np.sum((f2 - f1) ** 2, 1)) / np.mean(np.sum(f1 ** 2, 1))) < 1e-6
        assert abs(e1["coulomb"] - e2["coulomb"]) <= 1e-9 * abs(e1["coulomb"])
