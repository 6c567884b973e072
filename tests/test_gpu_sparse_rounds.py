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
