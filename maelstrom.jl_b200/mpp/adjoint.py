"""project! as a differentiable operation (the counterpart of a ChainRulesCore.rrule).

:class:`ProjectFunction` is a ``torch.autograd.Function``: its forward runs
``mpp_project`` on copies of the input faces, its backward runs ``mpp_project_vjp``
(beta = dx G^T g, the same preconditioned solve on the cotangent, g_in = g + D^T mu).
Both run in libmpp's CUDA kernels. The basin's cell classes and level set are the ones
at forward time and must not change before the backward pass.
"""
from __future__ import annotations

import torch

from . import FlipBasin, _raise_or_warn


class ProjectFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u, v, w, basin: FlipBasin, dt: float, recover: float = 0.5):
        uo, vo, wo = (a.detach().clone().contiguous() for a in (u, v, w))
        p = basin.projector
        res = p.project(uo, vo, wo, basin.fu, basin.fv, basin.fw, basin.P, basin.types, basin.phi, basin.volume0, dt,
                        recover)
        basin.iterations.append(res.iterations + res.fallback_iterations)
        basin.last = res
        _raise_or_warn(res)
        ctx.basin = basin
        return uo, vo, wo

    @staticmethod
    def backward(ctx, gu, gv, gw):
        s = ctx.basin
        g = s.grid
        dev = s.P.device
        outs = []
        for a, axis in ((gu, 0), (gv, 1), (gw, 2)):
            n = 1
            for e in g.face_shape(axis):
                n *= e
            outs.append(torch.zeros(n, dtype=torch.float32, device=dev) if a is None
                        else a.detach().to(torch.float32).contiguous().clone())
        if getattr(s, "mu", None) is None:
            s.mu = torch.zeros(g.ncells, dtype=torch.float32, device=dev)
        res = s.projector.project_vjp(*outs, s.mu, s.types, s.phi)
        s.last_vjp = res
        _raise_or_warn(res)
        return outs[0], outs[1], outs[2], None, None, None


def project(u, v, w, basin: FlipBasin, dt: float, recover: float = 0.5):
    """Differentiable ``project!``: returns the projected (u, v, w)."""
    return ProjectFunction.apply(u, v, w, basin, dt, recover)
