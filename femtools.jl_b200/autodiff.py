"""Reverse-mode differentiation of the Stokes DR solve through the device adjoint.

The reference differentiates its solve with a frozen-operator adjoint
(solve_adjoint!, src/stokes/solvers/DR_adjoint.jl:396-433) and exposes per-element
or per-phase material gradients (examples/miniapps/stokes/.../sinking_block_adj.jl:117-239,
DR_adjoint.jl:495-531). A Julia caller binds that pair as a ChainRulesCore rrule;
here the same pair is a torch.autograd.Function: the forward solves the Stokes
problem for a per-element log-viscosity δ (η_q = η0_q·exp(δ_e)), checkpoints the
converged DR state, and the backward restores the checkpoint, solves the adjoint
(dR/du)ᵀλ = −∂L/∂v on the device and returns dL/dδ_e = Σ_q η_q·λ·∂R/∂η_q.

`DRCheckpoint` snapshots and restores the pseudo-time state of a StokesDR (fields
and, optionally, a host copy) so that a solve can be resumed or its converged state
reused without re-solving.
"""
from __future__ import annotations

from typing import Optional

import torch

from . import solver as _solver

_FIELDS = ("v", "rate", "P", "gammaP", "M_P", "Pnum", "viscosity_ip")


class DRCheckpoint:
    """Copy of a StokesDR's pseudo-time state: velocity, rate, pressure, the pressure
    scaling, Pnum and the viscosity field; on the device, or spilled to pinned host
    memory with `host=True`."""

    def __init__(self, dr: "_solver.StokesDR", host: bool = False):
        self.host = host
        self.data = {}
        for name in _FIELDS:
            x = getattr(dr, name)
            if x is None:
                self.data[name] = None
            elif isinstance(x, list):
                self.data[name] = [self._copy(t) for t in x]
            else:
                self.data[name] = self._copy(x)

    def _copy(self, t):
        if self.host:
            out = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
            out.copy_(t, non_blocking=True)
            return out
        return t.clone()

    def restore(self, dr: "_solver.StokesDR"):
        for name in _FIELDS:
            x = self.data[name]
            if x is None:
                if name == "viscosity_ip":
                    dr.viscosity_ip = None
                continue
            cur = getattr(dr, name)
            if isinstance(x, list):
                for dst, src in zip(cur, x):
                    dst.copy_(src, non_blocking=True)
            elif cur is None or cur.shape != x.shape:
                setattr(dr, name, x.to(dr.device).clone())
            else:
                cur.copy_(x, non_blocking=True)


class StokesLogViscositySolve(torch.autograd.Function):
    """v = solve(δ): the converged velocity (3·nnodes, component-major) of the Stokes
    problem in `dr` with viscosity η_q = eta0_ip_q·exp(δ_e(q)) at every integration point."""

    @staticmethod
    def forward(ctx, delta, dr, bc_v, dt, eta0_ip, solve_kw, adjoint_kw):
        nq = dr.mesh.nq
        dr.viscosity_ip = (eta0_ip * torch.repeat_interleave(torch.exp(delta.detach()), nq)).contiguous()
        st = _solver.solve(dr, bc_v, dt, **(solve_kw or {}))
        ctx.stats = st
        ctx.dr, ctx.bc, ctx.dt, ctx.adjoint_kw = dr, bc_v, dt, adjoint_kw or {}
        ctx.ck = DRCheckpoint(dr)
        return torch.cat([x.clone() for x in dr.v])

    @staticmethod
    def backward(ctx, grad_v):
        dr = ctx.dr
        ctx.ck.restore(dr)
        nn = dr.mesh.nnodes
        obj = [grad_v[c * nn:(c + 1) * nn].contiguous().to(dr.dtype) for c in range(3)]
        lam_v, lam_P, st = _solver.solve_adjoint(dr, ctx.bc, ctx.dt, obj, **ctx.adjoint_kw)
        ctx.adjoint_stats = st
        sens = _solver.viscosity_sensitivity(dr, ctx.dt, lam_v, lam_P)
        g = (dr.viscosity_ip * sens).reshape(dr.mesh.nels, dr.mesh.nq).sum(dim=1)
        return g, None, None, None, None, None, None


def solve_log_viscosity(delta: torch.Tensor, dr, bc_v, dt, eta0_ip: torch.Tensor, solve_kw: Optional[dict] = None,
                        adjoint_kw: Optional[dict] = None) -> torch.Tensor:
    """Differentiable Stokes solve in the per-element log-viscosity δ (see the class)."""
    return StokesLogViscositySolve.apply(delta, dr, bc_v, dt, eta0_ip, solve_kw, adjoint_kw)
