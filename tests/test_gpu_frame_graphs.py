"""The CUDA graphs of the frames entries (mdrtNbForceFrames and the product
mode of mdrtNbParameterGradientFrames): a replayed graph gives the forces
of the launches it holds bit for bit (deterministic mode), follows new
positions and new parameters written into the same buffers, is captured
again after a build, and gives the product of the launches; and the
force-matching loss through torch autograd gives the same gradient with and
without graphs."""

import numpy as np
import pytest
import torch

from mdir_b200 import FrameEvaluator, systems
from mdir_b200 import torch as mtorch

pytestmark = pytest.mark.gpu


def pair(lanes, frames=8, waters=900, deterministic=False):
    s, X, target = systems.force_matching(frames=frames, waters=waters)
    on = FrameEvaluator(s, lanes=lanes)
    off = FrameEvaluator(s, lanes=lanes, frame_graphs=False)
    if deterministic:
        on.term.set_deterministic(True)
        off.term.set_deterministic(True)
    return s, X, target, on, off


def test_replays_are_the_launches_bit_for_bit():
    s, X, target, on, off = pair(lanes=1, deterministic=True)
    Xd = torch.tensor(X, device="cuda")
    ref = off.forces(Xd)
    F = torch.empty_like(Xd)
    for _ in range(5):
        on.forces(Xd, out=F)
        assert torch.equal(F, ref)
    captures, replays = on.term.frame_graph_info()
    assert captures >= 1 and replays >= 2
    assert off.term.frame_graph_info() == (0, 0)

    # new positions in the same buffer (within the skin: no build)
    before = on.builds
    Xd.add_(torch.randn_like(Xd) * 1e-3)
    on.forces(Xd, out=F)
    assert on.builds == before
    assert on.term.frame_graph_info()[1] > replays
    assert torch.equal(F, off.forces(Xd))

    # new parameters: the graph reads the particle tables at its launch.
    # (The first change makes the LJ table one that does not factorize, a
    # new kernel form and so a new key; the second keeps that form.)
    for scale in (1.0, 1.01):
        sig, eps, q = target["sigma"] * scale, target["epsilon"] / scale, target["charges"] * scale
        on.set_parameters(sig, eps, q)
        off.set_parameters(sig, eps, q)
        replays = on.term.frame_graph_info()[1]
        for _ in range(3 if scale == 1.0 else 1):
            on.forces(Xd, out=F)
        assert on.term.frame_graph_info()[1] > replays
        assert torch.equal(F, off.forces(Xd))

    # frames that moved past half the skin: a build, then new captures
    Xd.add_(0.3)
    for _ in range(4):
        on.forces(Xd, out=F)
    assert on.builds > before
    assert on.term.frame_graph_info()[0] > captures
    assert torch.equal(F, off.forces(Xd))


@pytest.mark.parametrize("lanes", [1, 3])
def test_product_replays_match_the_launches(lanes):
    s, X, target, on, off = pair(lanes=lanes, frames=7)
    Xd = torch.tensor(X, device="cuda")
    G = torch.randn_like(Xd) * 0.1
    P_on, P_off = on.potential_buffers(7), off.potential_buffers(7)
    off.forces(Xd, potentials=P_off)
    dq0, dt0 = off.product(Xd, G, potentials=P_off)
    for _ in range(4):
        on.forces(Xd, potentials=P_on)
        dq, dt = on.product(Xd, G, potentials=P_on, run=on.last_run)
        # the type-pair sums are f32 atomics within a block: their order,
        # not the graph, makes the difference between two runs
        assert (dq - dq0).abs().max().item() <= 1e-6 * dq0.abs().max().item()
        assert (dt - dt0).abs().max().item() <= 1e-5 * dt0.abs().max().item()
    assert sum(t.frame_graph_info()[1] for t in on._lane_terms) > 0


def test_loss_gradient_with_and_without_graphs():
    s, X, target, on, off = pair(lanes=2, frames=6)
    Xd = torch.tensor(X, device="cuda")
    grads = []
    for ev in (on, off):
        ev.set_parameters(target["sigma"], target["epsilon"], target["charges"])
        F_ref = ev.forces(Xd).clone()
        ev.set_parameters(s["type_sigma"], s["type_epsilon"], s["charges"])
        sig = torch.tensor(s["type_sigma"], device="cuda", requires_grad=True)
        eps = torch.tensor(s["type_epsilon"], device="cuda", requires_grad=True)
        q = torch.tensor(s["charges"], device="cuda", requires_grad=True)
        for _ in range(4):
            for t in (sig, eps, q):
                t.grad = None
            F = mtorch.forces(ev, sig, eps, q, Xd)
            loss = ((F - F_ref) ** 2).sum() / X.shape[0]
            loss.backward()
        grads.append([t.grad.cpu().numpy() for t in (sig, eps, q)])
    for a, b in zip(*grads):
        assert np.max(np.abs(a - b)) <= 1e-5 * np.max(np.abs(b))

