"""The frame evaluator as operations of PyTorch (the differentiation form).

`forces(evaluator, sigma, epsilon, charges, positions)` returns the forces
(K, n, 3) of the frames; autograd differentiates them in the per-type LJ
sigma / epsilon and the per-atom charges through the hand-written adjoint
of libmdrt_nb.so (`mdrtNbParameterGradientPotential`, the product mode),
which recomputes the pair geometry and reads each frame's reciprocal
potential grid as the forward kept it (4 bytes a grid point a frame;
`FrameEvaluator(keep_potentials=False)` recomputes it instead).  A
force-matching loss (1/K) sum |F - F_ref|^2 therefore costs one forward and
one adjoint pass per frame.

`evaluate(evaluator, theta, positions)` returns the energies (K,),
differentiable in theta = {"sigma", "epsilon", "charges"} (the energy mode)
and in the positions (dU/dx = -F).  MDIR: mdir.torch.evaluate
(python/mdir/torch.py), a custom op whose backward is the vector-Jacobian
product of the evaluator.  Forward mode is not implemented, and a second
derivative in the positions (forces that require a gradient in the
positions) is refused, as MDIR refuses it for the reciprocal sum."""

import numpy as np
import torch

from .frames import UnsupportedError, lorentz_berthelot_chain

__all__ = ["forces", "evaluate"]


def _host(t):
    return t.detach().to("cpu", torch.float64).numpy()


_PINNED = {}


def _host_params(sigma, epsilon, charges):
    """The three parameter tensors on the host (f64 copies): three
    asynchronous copies into a pinned buffer and one wait."""
    parts = [t.detach().reshape(-1) for t in (sigma, epsilon, charges)]
    sizes = [p.numel() for p in parts]
    total = sum(sizes)
    key = (total, parts[0].device)
    buf = _PINNED.get(key)
    if buf is None:
        buf = torch.empty(total, dtype=torch.float64, pin_memory=parts[0].is_cuda)
        _PINNED[key] = buf
    at = 0
    for p, k in zip(parts, sizes):
        buf[at:at + k].copy_(p, non_blocking=True)
        at += k
    if parts[0].is_cuda:
        torch.cuda.current_stream(parts[0].device).synchronize()
    flat = buf.numpy().copy()
    return flat[:sizes[0]], flat[sizes[0]:sizes[0] + sizes[1]], flat[sizes[0] + sizes[1]:]


class _Forces(torch.autograd.Function):
    @staticmethod
    def forward(ctx, evaluator, positions, sigma, epsilon, charges):
        # the host copies are taken once, before the forward is queued, so
        # that the host goes on to queue the loss and the backward while the
        # forward runs
        params = _host_params(sigma, epsilon, charges)
        evaluator.set_parameters(*params)
        X = evaluator.frames(positions.detach())
        P = evaluator.potential_buffers(X.shape[0]) if evaluator.keep_potentials else None
        F = evaluator.forces(X, potentials=P)
        ctx.evaluator = evaluator
        ctx.params = params
        ctx.potentials = P
        ctx.run = evaluator.last_run
        ctx.save_for_backward(X)
        return F.reshape(positions.shape)

    @staticmethod
    def backward(ctx, grad):
        if ctx.needs_input_grad[1]:
            raise UnsupportedError("the derivative of the forces in the positions is not implemented")
        ev = ctx.evaluator
        (X,) = ctx.saved_tensors
        ev.set_parameters(*ctx.params)
        dq, dt = ev.product(X, grad.reshape(X.shape), potentials=ctx.potentials, run=ctx.run)
        ctx.potentials = None
        # the per-type gradients on the device (no wait for the product)
        ds, de = ev.lorentz_berthelot_chain_device(dt)
        return (None, None, ds.to(grad.dtype) if ctx.needs_input_grad[2] else None,
                de.to(grad.dtype) if ctx.needs_input_grad[3] else None,
                dq if ctx.needs_input_grad[4] else None)


def forces(evaluator, sigma, epsilon, charges, positions):
    """Forces (K, n, 3) at the given per-type sigma / epsilon (nt,) and
    charges (n,), differentiable in the three."""
    return _Forces.apply(evaluator, positions, sigma, epsilon, charges)


class _Energies(torch.autograd.Function):
    @staticmethod
    def forward(ctx, evaluator, positions, sigma, epsilon, charges):
        evaluator.set_parameters(_host(sigma), _host(epsilon), _host(charges))
        X = evaluator.frames(positions.detach())
        F, E = evaluator.forces(X, energy=True)
        ctx.evaluator = evaluator
        ctx.params = (_host(sigma), _host(epsilon), _host(charges))
        ctx.save_for_backward(X, F)
        ctx.shape = positions.shape
        return torch.as_tensor(E, dtype=torch.float64, device=X.device)

    @staticmethod
    def backward(ctx, grad):
        ev = ctx.evaluator
        X, F = ctx.saved_tensors
        ev.set_parameters(*ctx.params)
        g = grad.detach().to(torch.float64)
        out_x = (-(g[:, None, None] * F)).reshape(ctx.shape) if ctx.needs_input_grad[1] else None
        ds = de = dq = None
        if any(ctx.needs_input_grad[2:]):
            q, t = ev.energy_gradient(X)
            gq = (g[:, None] * q).sum(0)
            gt = (g[:, None, None, None] * t).sum(0)
            s_, e_ = lorentz_berthelot_chain(gt.cpu().numpy(), ev.sigma, ev.epsilon)
            ds = torch.as_tensor(s_, device=grad.device)
            de = torch.as_tensor(e_, device=grad.device)
            dq = gq
        return None, out_x, ds, de, dq


def evaluate(evaluator, theta, positions):
    """Energies (K,) of the frames at theta = {"sigma", "epsilon",
    "charges"} (tensors; missing entries take the evaluator's values)."""
    dev = evaluator.device
    sigma = theta.get("sigma", torch.as_tensor(evaluator.sigma, device=dev))
    epsilon = theta.get("epsilon", torch.as_tensor(evaluator.epsilon, device=dev))
    charges = theta.get("charges", torch.as_tensor(evaluator.charges, device=dev))
    return _Energies.apply(evaluator, positions, sigma, epsilon, charges)
