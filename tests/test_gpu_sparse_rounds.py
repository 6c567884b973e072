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
