"""Lithostatic pressure: LithostaticPressureDR
(src/lithostatic_pressure/types/lithostatic_pressure_types.jl), its assembler
(assembly/residual_atomics.jl) and solve! (solvers/DR.jl), on the device through
libfemtools_b200. The steady Poisson problem ∫ ∇P·∇v dΩ = ∫ ρ(T, P) g·∇v dΩ for a nodal
P on the velocity mesh, ρ = ρ0 (1 − α (T − Tref) + P/K), relaxed by the same dynamic
relaxation as the thermal problem; its usual role is the initial pressure guess of a
Stokes solve.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _abi as abi
from . import problem as prob


class LithostaticPressureDR:
    """Device state: P (the unknown), its pseudo-transient rate, R, R0, the Jacobian
    row sums and diagonal, the temperature T (an EOS coefficient, zero by default) and
    one phase per node (1 by default). `rho0`, `alpha`, `K` are per phase, as in the
    ThermalMaterial the reference takes them from."""

    def __init__(self, mesh, rho0=(1.0,), alpha=(0.0,), K=(math.inf,), phases=None, CFL=0.98, c_fact=0.9,
                 eps=1e-6):
        import torch
        from . import solver
        solver._require_cuda()
        n = len(rho0)
        if len(alpha) != n or len(K) != n or not 1 <= n <= abi.MAX_PHASES:
            raise ValueError("material property tuples must have the same length (1..16)")
        self.mesh = mesh
        dev = torch.device("cuda")
        self.device, self.dtype = dev, torch.float64
        nn = mesh.nnodes
        for name in ("P", "rate", "R", "R0", "dRdP", "PC", "T"):
            setattr(self, name, torch.zeros(nn, dtype=torch.float64, device=dev))
        ph = np.ones(nn, dtype=np.int32) if phases is None else np.asarray(phases, dtype=np.int32).ravel()
        if len(ph) != nn or ph.min() < 1 or ph.max() > n:
            raise ValueError(f"phases must hold one value in 1:{n} per node")
        self.phases = torch.as_tensor(ph, device=dev)
        self.rho0, self.alpha, self.K = tuple(map(float, rho0)), tuple(map(float, alpha)), tuple(map(float, K))
        self.CFL, self.c_fact, self.eps = CFL, c_fact, eps
        self.el2n = torch.as_tensor(np.ascontiguousarray(mesh.el2n, dtype=np.int32), device=dev)
        self.geo = torch.as_tensor(np.ascontiguousarray(mesh.geo_v, dtype=np.float64), device=dev)
        self._keep = []

    def problem(self, bc=None) -> abi.LithostaticProblemC:
        import torch
        from . import solver
        p = abi.LithostaticProblemC()
        d = self.mesh.dim
        p.dim, p.nv, p.nq = (3, 27, 27) if d == 3 else (2, 9, 9)
        p.nels, p.nnodes = self.mesh.nels, self.mesh.nnodes
        p.el2n, p.geo = solver._ptr(self.el2n), solver._ptr(self.geo)
        for name in ("P", "rate", "R", "R0", "dRdP", "PC", "T"):
            setattr(p, name, solver._ptr(getattr(self, name)))
        p.phases, p.phases_layout, p.nphases = solver._ptr(self.phases), abi.PHASE_NODAL, len(self.rho0)
        for i in range(abi.MAX_PHASES):
            p.rho0[i] = self.rho0[i] if i < len(self.rho0) else 1.0
            p.alpha[i] = self.alpha[i] if i < len(self.alpha) else 0.0
            p.K[i] = self.K[i] if i < len(self.K) else math.inf
        self._keep = []
        if bc is not None:
            dofs = bc.DoFs if isinstance(bc, prob.DirichletBoundaryCondition) else bc[0]
            vals = bc.vals if isinstance(bc, prob.DirichletBoundaryCondition) else bc[1]
            dt_ = torch.as_tensor(np.asarray(dofs, dtype=np.int32), device=self.device).contiguous()
            vt = torch.as_tensor(np.asarray(vals, dtype=np.float64), device=self.device).reshape(-1).contiguous()
            self._keep = [dt_, vt]
            p.bc_dofs, p.bc_vals, p.bc_n = solver._ptr(dt_), solver._ptr(vt), dt_.numel()
        p.cfl, p.c_fact, p.eps = self.CFL, self.c_fact, self.eps
        return p


def _gravity(dr, g):
    d = dr.mesh.dim
    if g is None:
        if d != 2:
            raise ValueError("3-D lithostatic pressure needs g (the default (0, −9.81) is a 2-D body force)")
        g = (0.0, -9.81)
    if len(g) != d:
        raise ValueError(f"g must have {d} components")
    return (C.c_double * 3)(*(list(map(float, g)) + [0.0] * (3 - d)))


def assemble_lithostatic_pressure(dr: LithostaticPressureDR, Tref=273.0, g=None, compute_jacobian=False):
    """assemble_lithostatic_pressure_matrices_atomix! (assembly/residual_atomics.jl:1-19):
    fills dr.R and, with compute_jacobian, dr.dRdP (absolute row sums) and dr.PC (|diagonal|)."""
    from . import solver
    lib, h = solver._Handle.get()
    p = dr.problem()
    solver._check(lib, h, lib.femb200_lithostatic_residual(h, C.byref(p), float(Tref), _gravity(dr, g),
                                                          1 if compute_jacobian else 0))
    return dr.R


def solve_lithostatic(dr: LithostaticPressureDR, bc, Tref=273.0, g=None, tolerance=None, max_iterations=10_000,
                      check_interval=100, throw_on_failure=True):
    """solve!(dr::LithostaticPressureDR, mesh, bc; tolerance=dr.ϵ, max_iterations,
    check_interval, throw_on_failure, Tref, g) (solvers/DR.jl:21-44): dr.P in place from
    its current value; returns (converged, iterations, residual)."""
    from . import solver
    lib, h = solver._Handle.get()
    p = dr.problem(bc)
    c = abi.LithostaticControlsC()
    c.Tref = float(Tref)
    gg = _gravity(dr, g)
    for k in range(3):
        c.g[k] = gg[k]
    c.tolerance = dr.eps if tolerance is None else tolerance
    c.max_iterations, c.check_interval = max_iterations, check_interval
    c.throw_on_failure = 1 if throw_on_failure else 0
    st = abi.ThermalStatsC()
    solver._check(lib, h, lib.femb200_solve_lithostatic(h, C.byref(p), C.byref(c), C.byref(st)))
    return {"converged": bool(st.converged), "iterations": st.iterations, "residual": st.residual}
