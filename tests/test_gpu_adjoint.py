"""The parameter gradients of the device path (the differentiation form)
against central finite differences of the FP64 oracle, h = 1e-5: the
force-matching product sum_i g_i . dF_i/dtheta, the energy gradient, the
gradient of a force-matching loss through torch autograd, and the frame
schedule of the evaluator (MDIR's scenarios: test/Driver/Inputs/
python_tunable_gradient.py `lj`, `pme`, `charges`; python_frame_product.py).

The product and the energy gradient are linear in the cotangent and exact
in the parameters up to f32 arithmetic, so they meet GRAD_TOL per element
against the oracle at fixed cotangent.  The loss gradient also carries the
f32 error of the forward forces inside its cotangent F - F_ref: it meets
GRAD_TOL norm-wise per parameter group (and per element for sigma and
epsilon)."""

import numpy as np
import pytest
import torch

from oracle import oracle as O
from mdir_b200 import FrameEvaluator, systems
from mdir_b200 import torch as mtorch
from mdir_b200.frames import lorentz_berthelot

pytestmark = pytest.mark.gpu
GRAD_TOL = 1e-4
H = 1e-5


def with_params(s, sig, eps, q):
    c = dict(s)
    c["sigma"], c["epsilon"] = lorentz_berthelot(sig, eps)
    c["charges"] = np.asarray(q, dtype=np.float64)
    return c


def rel_err(a, fd):
    """The largest error relative to each finite difference, with a floor
    of 1e-3 of the largest one (a gradient near zero is compared to that)."""
    a = np.asarray(a, dtype=np.float64)
    fd = np.asarray(fd, dtype=np.float64)
    floor = 1e-3 * np.max(np.abs(fd))
    return float(np.max(np.abs(a - fd) / np.maximum(np.abs(fd), floor)))


def central(phi, sig, eps, q, lj_types, atoms, h=H):
    """Central differences of phi(sig, eps, q) in sigma and epsilon of the
    types `lj_types` and in the charges of `atoms`."""
    out = {"sigma": [], "epsilon": [], "charges": []}
    for name, base, idx in (("sigma", sig, lj_types), ("epsilon", eps, lj_types), ("charges", q, atoms)):
        for a in idx:
            up, dn = base.copy(), base.copy()
            up[a] += h
            dn[a] -= h
            args_up = {"sigma": sig, "epsilon": eps, "charges": q}
            args_dn = dict(args_up)
            args_up[name] = up
            args_dn[name] = dn
            out[name].append((phi(**args_up) - phi(**args_dn)) / (2 * h))
    return {k: np.array(v) for k, v in out.items()}


@pytest.fixture(scope="module")
def small():
    return systems.force_matching(frames=2, waters=600)


def _params(s):
    return (np.asarray(s["type_sigma"], dtype=np.float64).copy(),
            np.asarray(s["type_epsilon"], dtype=np.float64).copy(),
            np.asarray(s["charges"], dtype=np.float64).copy())


def test_product_matches_oracle_differences(cuda, small):
    s, X, _ = small
    sig, eps, q = _params(s)
    ev = FrameEvaluator(s)
    rng = np.random.default_rng(21)
    G = rng.normal(size=X.shape)
    dq, dt = ev.product(torch.tensor(X, device=cuda), torch.tensor(G, device=cuda))
    got = ev.per_type(dq, dt)

    def phi(sigma, epsilon, charges):
        sys_ = with_params(s, sigma, epsilon, charges)
        return sum(float(np.sum(G[k] * O.evaluate(sys_, X[k])["forces"])) for k in range(len(X)))

    atoms = rng.choice(len(q), 12, replace=False)
    fd = central(phi, sig, eps, q, range(8), atoms)
    for name, idx in (("sigma", range(8)), ("epsilon", range(8)), ("charges", atoms)):
        err = rel_err(got[name][list(idx)], fd[name])
        assert err <= GRAD_TOL, (name, err, got[name][list(idx)], fd[name])
    # the hydrogen type has no LJ term
    assert got["epsilon"][8] == 0.0 and abs(got["sigma"][8]) == 0.0


def test_energy_gradient_matches_oracle_differences(cuda, small):
    s, X, _ = small
    sig, eps, q = _params(s)
    ev = FrameEvaluator(s)
    out = ev.evaluate(torch.tensor(X, device=cuda), gradients=("tunables", "positions"))
    tun = out.gradients["tunables"]

    def phi(sigma, epsilon, charges):
        sys_ = with_params(s, sigma, epsilon, charges)
        return sum(O.evaluate(sys_, X[k])["energy"] for k in range(len(X)))

    rng = np.random.default_rng(22)
    atoms = rng.choice(len(q), 12, replace=False)
    fd = central(phi, sig, eps, q, range(8), atoms)
    assert rel_err(tun["sigma"].sum(0)[:8], fd["sigma"]) <= GRAD_TOL
    assert rel_err(tun["epsilon"].sum(0)[:8], fd["epsilon"]) <= GRAD_TOL
    assert rel_err(tun["charges"].sum(0)[atoms], fd["charges"]) <= GRAD_TOL
    # the positions gradient is -F, and the energies match the oracle
    ref = [O.evaluate(s, X[k]) for k in range(len(X))]
    for k in range(len(X)):
        assert abs(out.energy[k] - ref[k]["energy"]) <= 1e-6 * sum(abs(v) for v in ref[k]["terms"].values())
        Fk = -out.gradients["positions"][k].cpu().numpy()
        rms = np.sqrt(np.mean((Fk - ref[k]["forces"]) ** 2) / np.mean(ref[k]["forces"] ** 2))
        assert rms <= 1e-5


def test_vjp_is_the_product_with_the_sign_of_dU_dx(cuda, small):
    s, X, _ = small
    ev = FrameEvaluator(s)
    Xd = torch.tensor(X, device=cuda)
    rng = np.random.default_rng(23)
    Gbar = rng.normal(size=X.shape)
    out = ev.evaluate(Xd, gradients=("tunables",))
    v = out.vjp(positions=Gbar)
    dq, dt = ev.product(Xd, -torch.tensor(Gbar, device=cuda))
    ref = ev.per_type(dq, dt)
    # the same product, up to the order of the floating-point atomics of two runs
    for name in ("sigma", "epsilon", "charges"):
        assert np.allclose(v[name], ref[name], rtol=1e-5, atol=1e-6 * np.max(np.abs(ref[name])))
    # with a cotangent on the energies, the energy gradient is added
    w = out.vjp(np.array([1.0, 2.0]), positions=Gbar)
    tun = out.gradients["tunables"]
    e_part = tun["sigma"][0] + 2.0 * tun["sigma"][1]
    assert np.allclose(w["sigma"] - v["sigma"], e_part, rtol=1e-5, atol=1e-6 * np.max(np.abs(e_part)))


def test_force_matching_loss_gradient_through_autograd(cuda, small):
    s, X, target = small
    sig, eps, q = _params(s)
    ref_sys = with_params(s, target["sigma"], target["epsilon"], target["charges"])
    F_ref = np.stack([O.evaluate(ref_sys, X[k])["forces"] for k in range(len(X))])
    ev = FrameEvaluator(s)
    ts = torch.tensor(sig, device=cuda, requires_grad=True)
    te = torch.tensor(eps, device=cuda, requires_grad=True)
    tq = torch.tensor(q, device=cuda, requires_grad=True)
    Xd = torch.tensor(X, device=cuda)
    Fr = torch.tensor(F_ref, device=cuda)
    F = mtorch.forces(ev, ts, te, tq, Xd)
    loss = ((F - Fr) ** 2).sum() / len(X)
    loss.backward()

    def phi(sigma, epsilon, charges):
        sys_ = with_params(s, sigma, epsilon, charges)
        return sum(float(np.sum((O.evaluate(sys_, X[k])["forces"] - F_ref[k]) ** 2)) for k in range(len(X))) / len(X)

    rng = np.random.default_rng(24)
    atoms = rng.choice(len(q), 12, replace=False)
    fd = central(phi, sig, eps, q, range(8), atoms)
    got = {"sigma": ts.grad.cpu().numpy()[:8], "epsilon": te.grad.cpu().numpy()[:8],
           "charges": tq.grad.cpu().numpy()[atoms]}
    # Norm-wise within GRAD_TOL for each group.  Per element, the cotangent
    # 2 (F - F_ref)/K holds the f32 error of the forward forces (about 3e-6
    # of |F|) against a difference of about 2% of |F|, some 1.5e-4 per
    # component; the LJ gradients average it over thousands of pairs, the
    # gradient of one charge over its few hundred neighbours only.
    for name, per_element in (("sigma", GRAD_TOL), ("epsilon", GRAD_TOL), ("charges", 1e-3)):
        a, f = got[name], fd[name]
        assert np.linalg.norm(a - f) <= GRAD_TOL * np.linalg.norm(f), (name, a, f)
        assert rel_err(a, f) <= per_element, (name, rel_err(a, f))
    assert abs(loss.item() - phi(sig, eps, q)) <= 1e-3 * loss.item()


def test_frames_beyond_the_skin_get_a_new_build(cuda):
    s, X, _ = systems.force_matching(frames=3, waters=600, jitter=0.005)
    X = X.copy()
    X[1] += np.array([0.08, 0.0, 0.0])  # a translation beyond half the skin (0.05 nm)
    ev = FrameEvaluator(s)
    F = ev.forces(torch.tensor(X, device=cuda)).cpu().numpy()
    assert ev.builds == 3  # frame 0, frame 1 (moved), frame 2 (far from frame 1)
    for k in range(3):
        ref = O.evaluate(s, X[k])["forces"]
        rms = np.sqrt(np.mean((F[k] - ref) ** 2) / np.mean(ref ** 2))
        assert rms <= 1e-5
    # frames that stay within half the skin share one build
    ev2 = FrameEvaluator(s)
    ev2.forces(torch.tensor(X[[0, 2]], device=cuda))
    assert ev2.builds == 1


def test_product_at_the_full_water_box(cuda):
    """One frame of the 23,550-atom box (8 oxygen types), the 16 LJ
    parameters and 6 charges against the FP64 oracle."""
    s, X, _ = systems.force_matching(frames=1, waters=7850)
    sig, eps, q = _params(s)
    ev = FrameEvaluator(s)
    rng = np.random.default_rng(26)
    G = rng.normal(size=X.shape)
    dq, dt = ev.product(torch.tensor(X, device=cuda), torch.tensor(G, device=cuda))
    got = ev.per_type(dq, dt)

    def phi(sigma, epsilon, charges):
        return float(np.sum(G[0] * O.evaluate(with_params(s, sigma, epsilon, charges), X[0])["forces"]))

    atoms = rng.choice(len(q), 6, replace=False)
    fd = central(phi, sig, eps, q, range(8), atoms)
    assert rel_err(got["sigma"][:8], fd["sigma"]) <= GRAD_TOL
    assert rel_err(got["epsilon"][:8], fd["epsilon"]) <= GRAD_TOL
    assert rel_err(got["charges"][atoms], fd["charges"]) <= GRAD_TOL


def test_lanes_give_the_results_of_one_lane(cuda):
    """Frames spread over 4 contexts on their own streams (one moved beyond
    half the skin, so that the lanes build again in the middle of a call)
    give the forces, energies and gradients of one context."""
    s, X, _ = systems.force_matching(frames=7, waters=600, jitter=0.005)
    X = X.copy()
    X[4] += np.array([0.08, 0.0, 0.0])
    Xd = torch.tensor(X, device=cuda)
    G = torch.tensor(np.random.default_rng(3).normal(size=X.shape), device=cuda)
    out = []
    for lanes in (1, 4):
        ev = FrameEvaluator(s, lanes=lanes)
        F, E = ev.forces(Xd, energy=True)
        dq, dt = ev.product(Xd, G)
        eq, et = ev.energy_gradient(Xd)
        out.append((F.cpu().numpy(), E, dq.cpu().numpy(), dt.cpu().numpy(), eq.cpu().numpy(), et.cpu().numpy(),
                    ev.builds))
    one, four = out
    # each call: frames 0-3 on the build in force, frame 4 (moved), frame 5 (far from frame 4)
    assert one[6] == four[6] == 7
    for a, b in zip(one[:6], four[:6]):
        scale = np.max(np.abs(a))
        assert np.max(np.abs(a - b)) <= 1e-6 * scale


def test_kept_potential_grids_give_the_recomputed_gradient(cuda):
    """The product with each frame's reciprocal potential grid kept from the
    forward (mdrtPmePotentialGrid, mdrtNbParameterGradientPotential) against
    the product that runs the reciprocal forward again, over 4 lanes with a
    build in the middle of the call; and the autograd op both ways."""
    s, X, _ = systems.force_matching(frames=7, waters=600, jitter=0.005)
    X = X.copy()
    X[4] += np.array([0.08, 0.0, 0.0])
    Xd = torch.tensor(X, device=cuda)
    G = torch.tensor(np.random.default_rng(5).normal(size=X.shape), device=cuda)
    ev = FrameEvaluator(s, lanes=4)
    P = ev.potential_buffers(len(X))
    ev.forces(Xd, potentials=P)
    kept = ev.product(Xd, G, potentials=P)
    again = ev.product(Xd, G)
    for a, b in zip(kept, again):
        a, b = a.cpu().numpy(), b.cpu().numpy()
        assert np.max(np.abs(a - b)) <= 1e-6 * np.max(np.abs(b))
    sig, eps, q = _params(s)
    grads = []
    for keep in (True, False):
        ev = FrameEvaluator(s, lanes=4, keep_potentials=keep)
        ts = torch.tensor(sig, device=cuda, requires_grad=True)
        te = torch.tensor(eps, device=cuda, requires_grad=True)
        tq = torch.tensor(q, device=cuda, requires_grad=True)
        Fk = mtorch.forces(ev, ts, te, tq, Xd)
        (Fk ** 2).sum().backward()
        grads.append([ts.grad.cpu().numpy(), te.grad.cpu().numpy(), tq.grad.cpu().numpy()])
    for a, b in zip(*grads):
        assert np.max(np.abs(a - b)) <= 1e-6 * np.max(np.abs(b))
