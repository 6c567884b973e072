"""Host logic of the differentiation form (no GPU): the Lorentz-Berthelot
chain rule from table gradients to per-type gradients, the gradient of the
dispersion correction, and the force-matching workload."""

import numpy as np

from mdir_b200 import systems
from mdir_b200.frames import (diagonal_types, dispersion_table_gradient, lorentz_berthelot,
                              lorentz_berthelot_chain)
from oracle import oracle


def test_lorentz_berthelot_chain_matches_differences():
    rng = np.random.default_rng(11)
    nt = 5
    sig = rng.uniform(0.25, 0.4, nt)
    eps = rng.uniform(0.2, 1.0, nt)
    eps[-1] = 0.0  # a type without LJ
    A = rng.normal(size=(2, nt, nt))

    def f(s, e):
        ts, te = lorentz_berthelot(s, e)
        return float((A[0] * ts).sum() + (A[1] * te).sum())

    ds, de = lorentz_berthelot_chain(A, sig, eps)
    h = 1e-6
    for a in range(nt):
        sp, sm = sig.copy(), sig.copy()
        sp[a] += h
        sm[a] -= h
        assert abs((f(sp, eps) - f(sm, eps)) / (2 * h) - ds[a]) < 1e-7
        if eps[a] > 0:
            ep, em = eps.copy(), eps.copy()
            ep[a] += h
            em[a] -= h
            assert abs((f(sig, ep) - f(sig, em)) / (2 * h) - de[a]) < 1e-6
        else:
            assert de[a] == 0.0


def test_lorentz_berthelot_chain_on_the_device_side_is_the_host_chain():
    """FrameEvaluator.lorentz_berthelot_chain_device (the autograd op's chain,
    torch ops on the evaluator's device; here the CPU) equals the host chain,
    and takes new weights when the parameters change."""
    import types
    import torch
    from mdir_b200.frames import FrameEvaluator
    rng = np.random.default_rng(12)
    nt = 6
    ev = types.SimpleNamespace(version=0, device=torch.device("cpu"), epsilon=rng.uniform(0.2, 1.0, nt))
    ev.epsilon[2] = 0.0
    for version in range(2):
        ev.version = version
        ev.epsilon = ev.epsilon * (1.0 + 0.1 * version)
        A = rng.normal(size=(2, nt, nt))
        ds, de = FrameEvaluator.lorentz_berthelot_chain_device(ev, torch.tensor(A))
        hs, he = lorentz_berthelot_chain(A, np.full(nt, 0.3), ev.epsilon)
        assert np.allclose(ds.numpy(), hs, rtol=1e-14, atol=0)
        assert np.allclose(de.numpy(), he, rtol=1e-14, atol=0)


def test_dispersion_gradient_matches_oracle_differences():
    s = systems.solvated_frame(1200, seed=3)
    s["dispersion"] = True
    sig, eps = diagonal_types(s)
    box = np.asarray(s["box"])
    ts, te = lorentz_berthelot(sig, eps)
    G = dispersion_table_gradient(s, ts, te, box)
    pairs = np.asarray(s["excluded_pairs"]).reshape(-1, 2)

    def energy(ts_, te_):
        return oracle.dispersion_energy(np.asarray(s["types"]), ts_, te_, pairs, box, s["cutoff"])

    h = 1e-7
    for part, base in ((0, ts), (1, te)):
        for a, b in ((0, 0), (0, 3), (2, 5)):
            up, dn = base.copy(), base.copy()
            # one entry of the table, as the gradient counts each ordered entry
            up[a, b] += h
            dn[a, b] -= h
            args_up = (up, te) if part == 0 else (ts, up)
            args_dn = (dn, te) if part == 0 else (ts, dn)
            fd = (energy(*args_up) - energy(*args_dn)) / (2 * h)
            assert abs(fd - G[part, a, b]) <= 1e-6 * max(1.0, abs(fd)), (part, a, b, fd, G[part, a, b])


def test_force_matching_workload_shapes():
    s, X, target = systems.force_matching(frames=3, waters=300, types=8)
    n = 900
    assert X.shape == (3, n, 3)
    t = np.asarray(s["types"])
    assert t.max() == 8 and np.all(t[1::3] == 8) and set(np.unique(t[0::3])) == set(range(8))
    sig, eps = diagonal_types(s)
    assert len(sig) == 9 and eps[-1] == 0.0
    rel = target["charges"] / s["charges"] - 1.0
    assert np.allclose(np.abs(rel), 0.02)
    # the same seeds give the same workload
    s2, X2, _ = systems.force_matching(frames=3, waters=300, types=8)
    assert np.array_equal(X, X2)


def test_batch_shards_balance_atoms():
    from mdir_b200.batch import shard
    rng = np.random.default_rng(4)
    atoms = 3 * rng.integers(333, 2667, size=256)
    for ranks in (1, 2, 4, 8):
        parts = shard(atoms, ranks)
        assert sorted(f for p in parts for f in p) == list(range(256))
        loads = [int(atoms[p].sum()) for p in parts]
        assert max(loads) - min(loads) <= int(atoms.max())
