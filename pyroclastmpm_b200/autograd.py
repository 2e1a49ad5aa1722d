"""torch.autograd wrapper of the differentiable USL rollout.

``rollout(sim, youngs, friction, nsteps, checkpoint_every)`` runs `nsteps`
steps of `sim` from its current state with per-particle Drucker-Prager
Young's modulus and friction angle (CUDA float32 tensors [n], particle id
order) and returns the final positions [n, dim] as a CUDA tensor.  Its
backward runs the checkpointed adjoint in the native library and returns the
gradients of the two parameter tensors, so a calibration loop is plain torch:

    E = torch.full((n,), 5e6, device="cuda", requires_grad=True)
    phi = torch.full((n,), 25.0, device="cuda", requires_grad=True)
    x = rollout(sim, E, phi, 500, 25)
    loss = ((x - target) ** 2).mean()
    loss.backward()                  # E.grad, phi.grad

Each forward starts from the state the first rollout started from (the
simulation is reset to it), so repeated calls evaluate the same map.
PyTorch is plumbing here: no torch operator runs on the step.
"""
from __future__ import annotations

import torch

from ._capi import Simulation


class _Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, youngs, friction, sim: Simulation, nsteps: int, checkpoint_every: int):
        if not (youngs.is_cuda and friction.is_cuda):
            raise ValueError("parameters must be CUDA tensors")
        n, d = sim.n, sim.dim
        E = youngs.detach().to(torch.float32).contiguous()
        phi = friction.detach().to(torch.float32).contiguous()
        if E.numel() != n or phi.numel() != n:
            raise ValueError("one parameter per particle expected")
        if getattr(sim, "_rollout_started", False):
            sim.rollout_reset()
        torch.cuda.current_stream().synchronize()
        sim.set_ptr("youngs_modulus", E.data_ptr(), 4 * n, on_device=True)
        sim.set_ptr("friction_angle", phi.data_ptr(), 4 * n, on_device=True)
        sim.rollout_forward(nsteps, checkpoint_every)
        sim._rollout_started = True
        x = torch.empty((n, d), dtype=torch.float32, device=youngs.device)
        sim.get_ptr("positions", x.data_ptr(), 4 * n * d, on_device=True)
        ctx.sim = sim
        return x

    @staticmethod
    def backward(ctx, grad_x):
        sim = ctx.sim
        n = sim.n
        g = grad_x.detach().to(torch.float32).contiguous()
        gE = torch.empty(n, dtype=torch.float32, device=g.device)
        gphi = torch.empty(n, dtype=torch.float32, device=g.device)
        torch.cuda.current_stream().synchronize()
        sim.rollout_backward_ptr(g.data_ptr(), gE.data_ptr(), gphi.data_ptr())
        return gE, gphi, None, None, None


def rollout(sim: Simulation, youngs: torch.Tensor, friction: torch.Tensor, nsteps: int,
            checkpoint_every: int = 25) -> torch.Tensor:
    """Final positions after `nsteps` steps, differentiable in the per-particle
    Young's modulus and friction angle (degrees)."""
    return _Rollout.apply(youngs, friction, sim, int(nsteps), int(checkpoint_every))


def calibrate(sim: Simulation, target: torch.Tensor, youngs0, friction0, nsteps: int, checkpoint_every: int = 25,
              iterations: int = 40, lr_log_youngs: float = 0.05, lr_friction: float = 0.5):
    """Per-particle calibration of Young's modulus and friction angle to a
    target final configuration: Adam on (log E, friction angle in degrees),
    the loss being the mean squared distance of the final positions from
    `target` [n, dim] (a CUDA tensor).  Returns (E, friction, losses): the
    parameters after the last iteration and the loss of every iteration."""
    dev = target.device
    logE = torch.log(torch.as_tensor(youngs0, dtype=torch.float32, device=dev)).clone().requires_grad_(True)
    phi = torch.as_tensor(friction0, dtype=torch.float32, device=dev).clone().requires_grad_(True)
    opt = torch.optim.Adam([{"params": [logE], "lr": lr_log_youngs}, {"params": [phi], "lr": lr_friction}])
    losses = []
    n = target.shape[0]
    scale = None
    for _ in range(iterations):
        opt.zero_grad()
        x = rollout(sim, torch.exp(logE), phi, nsteps, checkpoint_every)
        loss = ((x.double() - target.double()) ** 2).sum() / n
        # the loss (m^2) and its per-particle gradients are tiny; scaled by
        # the first loss, the gradients stay far above Adam's epsilon
        if scale is None:
            scale = 1.0 / max(float(loss.item()), 1e-300)
        (loss * scale).backward()
        opt.step()
        losses.append(float(loss.item()))
    return torch.exp(logE).detach(), phi.detach(), losses
