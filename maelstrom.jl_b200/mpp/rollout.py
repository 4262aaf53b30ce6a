"""Rollouts of semi-Lagrangian advection + projection and their gradient.

One step is ``advect!`` of the face velocities through themselves (src/flip.jl:495-497,
the velocity part of a FlipBasin step) followed by ``project!`` (src/flip.jl:1144-1156)
on the basin's fixed cell classes and level set. :class:`Rollout` keeps one velocity
checkpoint per step (the state each step starts from) and runs the reverse pass with
libmpp's adjoint kernels: the projection's (``mpp_project_vjp``) and the advection's
(``mpp_advect_vjp``), recomputing each step's trajectories from its checkpoint.
:class:`AdvectFunction` is the same advection adjoint as a ``torch.autograd.Function``,
so ``adjoint.project`` and it compose under autograd as well.
"""
from __future__ import annotations

import torch

from . import FlipBasin, _raise_or_warn


class Rollout:
    """``steps`` steps of advect + project on ``basin`` (its types, phi, volume0 and
    solver context), with per-step velocity checkpoints for :meth:`backward`."""

    def __init__(self, basin: FlipBasin, steps: int, dt: float, recover: float = 0.5):
        self.s, self.steps, self.dt, self.recover = basin, int(steps), float(dt), float(recover)
        dev = basin.P.device
        self.ckpt = [[torch.empty_like(a) for a in (basin.u, basin.v, basin.w)] for _ in range(self.steps + 1)]
        self.work = [torch.empty_like(a) for a in (basin.u, basin.v, basin.w)]
        self.grad = [torch.empty_like(a) for a in (basin.u, basin.v, basin.w)]
        self.mu = torch.zeros(basin.grid.ncells, dtype=torch.float32, device=dev)
        self.iterations, self.adjoint_iterations = [], []

    def forward(self, u, v, w):
        """Run the rollout from (u, v, w): returns the final (u, v, w) (views of the last
        checkpoint)."""
        s, p = self.s, self.s.projector
        for c, a in zip(self.ckpt[0], (u, v, w)):
            c.copy_(a)
        self.iterations = []
        for n in range(self.steps):
            p.advect(*self.ckpt[n], self.dt, out=self.work)
            res = p.project(*self.work, s.fu, s.fv, s.fw, s.P, s.types, s.phi, s.volume0, self.dt, self.recover)
            _raise_or_warn(res)
            self.iterations.append(res.iterations + res.fallback_iterations)
            for c, a in zip(self.ckpt[n + 1], self.work):
                c.copy_(a)
        return self.ckpt[self.steps]

    def backward(self, gu, gv, gw):
        """The cotangent of the final (u, v, w) in; the initial (u, v, w)'s out."""
        s, p = self.s, self.s.projector
        for c, a in zip(self.grad, (gu, gv, gw)):
            c.copy_(a)
        self.adjoint_iterations = []
        for n in reversed(range(self.steps)):
            res = p.project_vjp(*self.grad, self.mu, s.types, s.phi)
            _raise_or_warn(res)
            self.adjoint_iterations.append(res.iterations + res.fallback_iterations)
            p.advect_vjp(*self.grad, *self.ckpt[n], self.dt, out=self.grad)
        return self.grad


class AdvectFunction(torch.autograd.Function):
    """advect! of the face velocities as a differentiable op; saves its input velocity
    (the step's checkpoint) for the backward pass."""

    @staticmethod
    def forward(ctx, u, v, w, basin: FlipBasin, dt: float):
        p = basin.projector
        outs = p.advect(u.detach().contiguous(), v.detach().contiguous(), w.detach().contiguous(), dt)
        ctx.save_for_backward(u.detach(), v.detach(), w.detach())
        ctx.basin, ctx.dt = basin, dt
        return tuple(outs)

    @staticmethod
    def backward(ctx, gu, gv, gw):
        u, v, w = ctx.saved_tensors
        gs = [torch.zeros_like(a) if g is None else g.detach().contiguous() for g, a in zip((gu, gv, gw), (u, v, w))]
        outs = ctx.basin.projector.advect_vjp(*gs, u, v, w, ctx.dt)
        return outs[0], outs[1], outs[2], None, None


def advect(u, v, w, basin: FlipBasin, dt: float):
    return AdvectFunction.apply(u, v, w, basin, dt)
