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


def test_lists_put_lj_partners_first():
    """A build without a pruned reach orders each group's entries with the
    partners that have Lennard-Jones terms first (the adjoint skips its LJ
    terms in the rounds after them), and the pair set stays the oracle's."""
    from mdir_b200 import NonbondedTerm
    from mdir_b200 import _lib as L
    from oracle import oracle as O
    s = systems.tip3p(waters=600)
    x = np.asarray(s["positions"])
    t = NonbondedTerm(len(x))
    t.set_particles(s["charges"], s["types"], s["sigma"], s["epsilon"])
    t.set_exclusions(pairs=s["excluded_pairs"])
    t.set_interaction(s["cutoff"], s["reach"], s["beta"])
    sizes = t.build(torch.tensor(x, device="cuda"), s["box"])
    G = int(sizes[L.SIZE_GROUPS])
    cap = t.info()["list_capacity"]
    entries = t.buffer(L.SLOT_ENTRIES, np.int32, 2)[: G * cap].reshape(G, cap, 2)
    counts = t.buffer(L.SLOT_COUNTS, np.int32)[:G]
    order = t.buffer(L.SLOT_ORDER, np.int32)
    eps = np.asarray(s["epsilon"])
    lj_type = np.any(eps != 0.0, axis=1)
    types = np.asarray(s["types"])
    assert lj_type.any() and not lj_type.all()
    mixed = 0
    for g in range(G):
        partners = entries[g, : counts[g], 0]
        flags = lj_type[types[order[partners]]]
        # every LJ partner before every other one
        assert not np.any(flags[1:] & ~flags[:-1]), g
        mixed += bool(flags.any() and not flags.all())
    assert mixed > 0
    got = np.asarray(t.pair_set(sizes), dtype=np.int64)
    count, ref = O.pairset(x, s["box"], s["reach"], O.rows_from_pairs(len(x), s["excluded_pairs"]))
    ref = np.asarray(ref, dtype=np.int64)
    assert len(got) == count
    key = lambda p: p[np.lexsort((p[:, 2], p[:, 1], p[:, 0]))]
    np.testing.assert_array_equal(key(got), key(ref))
    t.close()


def test_frames_past_the_skin_mid_call_are_evaluated_again():
    """The frames of a call go on the build in force while their test runs;
    when frames from the middle of the call on moved past half the skin,
    those are evaluated again after a build.  Each frame's forces equal
    those of the frame evaluated alone, with lists built at it."""
    s, X, target = systems.force_matching(frames=8, waters=900)
    X = X.copy()
    X[5:] += 0.3  # every atom of frames 5.. moved 0.52 nm, past half the skin
    ev = FrameEvaluator(s, lanes=3)
    Xd = torch.tensor(X, device="cuda")
    for _ in range(2):
        ev.forces(Xd[:1])  # a build at frame 0
        F = ev.forces(Xd).cpu().numpy()
    for k in range(8):
        one = FrameEvaluator(s, lanes=1, frame_graphs=False)
        ref = one.forces(Xd[k:k + 1]).cpu().numpy()[0]
        err = np.sqrt(np.mean(np.sum((F[k] - ref) ** 2, 1)) / np.mean(np.sum(ref ** 2, 1)))
        assert err < 1e-6, (k, err)
