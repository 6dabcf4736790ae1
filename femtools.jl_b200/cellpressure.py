"""Viscous Hex27 Stokes with four cell-local pressure modes (1, ξ, η, ζ) per cell:
CellPressureStokesDR (src/stokes/types/stokes_types.jl:567-613), its assemblers
(src/stokes/assemblers/momentum_residuals.jl:618-745, pressure_residual.jl:330-364) and
solve! (src/stokes/solvers/DR.jl:960-1057), on the device through libfemtools_b200.

The whole Arrow–Hurwicz loop runs inside `femb200_solve_cell_pressure`; only the
convergence checks synchronise.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional, Sequence

import numpy as np

from . import _abi as abi
from . import problem as prob


class CellPressureStokesDR:
    """State of the viscous 3-D Stokes solver on a Hex27 mesh: continuous Q2 velocity
    `v` and the 4 × nels cell pressure `P` (mode fastest), both starting at zero; the
    residuals, the Jacobi preconditioner and the lumped pressure mass. `material` gives
    the phase viscosities η, densities ρ0 and the three-component gravity; finite G or
    K and nonzero α are rejected (the discretisation is purely viscous and
    incompressible). `phases` assigns one 1-based phase per cell (default 1)."""

    def __init__(self, mesh, material: prob.StokesMaterial, phases=None):
        import torch
        from . import solver
        solver._require_cuda()
        if mesh.dim != 3 or mesh.el2n.shape[1] != 27:
            raise ValueError("CellPressureStokesDR requires a Hex27 mesh")
        if len(material.g) != 3:
            raise ValueError("material gravity must have 3 components")
        if not (all(math.isinf(x) for x in material.G) and all(math.isinf(x) for x in material.K)
                and all(x == 0 for x in material.alpha)):
            raise ValueError("CellPressureStokesDR is purely viscous and incompressible; G and K must be Inf and α zero")
        n = len(material.eta)
        if phases is None:
            phases = np.ones(mesh.nels, dtype=np.int32)
        phases = np.asarray(phases.cpu() if hasattr(phases, "cpu") else phases).astype(np.int32).ravel()
        if len(phases) != mesh.nels:
            raise ValueError(f"phases has {len(phases)} entries but the mesh has {mesh.nels} cells")
        if phases.min() < 1 or phases.max() > n:
            raise ValueError(f"phases must lie in 1:{n}, got {phases.min()}:{phases.max()}")
        self.mesh, self.material = mesh, material
        dev = torch.device("cuda")
        self.device, self.dtype = dev, torch.float64
        z = lambda k: torch.zeros(k, dtype=torch.float64, device=dev)
        nn, ne = mesh.nnodes, mesh.nels
        self.v = [z(nn) for _ in range(3)]
        self.P = z(4 * ne)
        self.Rv = [z(nn) for _ in range(3)]
        self.RP = z(4 * ne)
        self.diagonal = [z(nn) for _ in range(3)]
        self.pressure_mass = z(4 * ne)
        self.phases = torch.as_tensor(phases, device=dev)
        self.el2n = torch.as_tensor(np.ascontiguousarray(mesh.el2n, dtype=np.int32), device=dev)
        self.geo_v = torch.as_tensor(np.ascontiguousarray(mesh.geo_v, dtype=np.float64), device=dev)
        self._keep = []

    def problem(self, bc_v: Optional[Sequence] = None, load=None) -> abi.CellPressureProblemC:
        import torch
        from . import solver
        p = abi.CellPressureProblemC()
        p.nels, p.nnodes = self.mesh.nels, self.mesh.nnodes
        p.el2n, p.geo_v, p.phases = solver._ptr(self.el2n), solver._ptr(self.geo_v), solver._ptr(self.phases)
        m = self.material
        p.nphases = len(m.eta)
        for i in range(len(m.eta)):
            p.eta[i], p.rho[i] = m.eta[i], m.rho0[i]
        for c in range(3):
            p.g[c] = m.g[c]
            p.v[c], p.Rv[c], p.diagonal[c] = (solver._ptr(self.v[c]), solver._ptr(self.Rv[c]),
                                              solver._ptr(self.diagonal[c]))
        p.P, p.RP, p.pressure_mass = solver._ptr(self.P), solver._ptr(self.RP), solver._ptr(self.pressure_mass)
        keep = []
        if load is not None:
            for c in range(3):
                t = torch.as_tensor(np.asarray(load[c].cpu() if hasattr(load[c], "cpu") else load[c]),
                                    dtype=torch.float64, device=self.device).contiguous()
                keep.append(t)
                p.load[c] = solver._ptr(t)
        if bc_v is not None:
            for c in range(3):
                bc = bc_v[c]
                if bc is None:
                    continue
                dofs = bc.DoFs if isinstance(bc, prob.DirichletBoundaryCondition) else bc[0]
                vals = bc.vals if isinstance(bc, prob.DirichletBoundaryCondition) else bc[1]
                d = torch.as_tensor(np.asarray(dofs.cpu() if hasattr(dofs, "cpu") else dofs, dtype=np.int32),
                                    device=self.device).contiguous()
                vv = torch.as_tensor(np.asarray(vals.cpu() if hasattr(vals, "cpu") else vals, dtype=np.float64),
                                     device=self.device).reshape(-1).contiguous()
                if vv.numel() == 1 and d.numel() != 1:
                    vv = vv.expand(d.numel()).contiguous()
                keep += [d, vv]
                p.bc_dofs[c], p.bc_vals[c], p.bc_n[c] = solver._ptr(d), solver._ptr(vv), d.numel()
        self._keep = keep
        return p


def stokes_preconditioner_3d(dr: CellPressureStokesDR):
    """stokes_preconditioner_3d!(diagonal, pressure_mass, mesh, phases, η)
    (momentum_residuals.jl:703-745): fills dr.diagonal and dr.pressure_mass."""
    from . import solver
    lib, h = solver._Handle.get()
    p = dr.problem()
    solver._check(lib, h, lib.femb200_cell_pressure_preconditioner(h, C.byref(p)))
    return dr.diagonal, dr.pressure_mass


def assemble_stokes_pressure_residual_3d(dr: CellPressureStokesDR):
    """assemble_stokes_pressure_residual_3d!(RP, v, mesh) (pressure_residual.jl:330-364)."""
    from . import solver
    lib, h = solver._Handle.get()
    p = dr.problem()
    solver._check(lib, h, lib.femb200_cell_pressure_residuals(h, C.byref(p), 1))
    return dr.RP


def assemble_stokes_momentum_residual_3d(dr: CellPressureStokesDR):
    """assemble_stokes_momentum_residual_3d!(R, v, P, mesh, phases, η, ρ, g)
    (momentum_residuals.jl:644-700)."""
    from . import solver
    lib, h = solver._Handle.get()
    p = dr.problem()
    solver._check(lib, h, lib.femb200_cell_pressure_residuals(h, C.byref(p), 2))
    return dr.Rv


def solve_cell_pressure(dr: CellPressureStokesDR, bc_v, tolerance=1e-5, max_iterations=3000, check_interval=100,
                        velocity_step=0.6, pressure_step=0.2, throw_on_failure=True, collect_history=False,
                        load=None):
    """solve!(dr::CellPressureStokesDR, mesh, bc_v; tolerance, max_iterations,
    check_interval, velocity_step, pressure_step, collect_history, throw_on_failure)
    (DR.jl:980-1002): Arrow–Hurwicz relaxation of dr.v and dr.P in place from their
    current values. `bc_v` holds one DirichletBoundaryCondition (or (DoFs, vals)) per
    component; `load` an optional momentum right-hand side subtracted from Rv. Returns
    the reference's stats (converged, iterations, residual, history, err_v, err_P,
    iter, err, reached_total_iter); a solve that does not converge raises
    FemB200Error unless throw_on_failure is False."""
    from . import solver
    lib, h = solver._Handle.get()
    p = dr.problem(bc_v, load)
    c = abi.CellPressureControlsC()
    c.tolerance, c.max_iterations, c.check_interval = tolerance, max_iterations, check_interval
    c.velocity_step, c.pressure_step, c.throw_on_failure = velocity_step, pressure_step, 1 if throw_on_failure else 0
    cap = max_iterations // max(check_interval, 1) + 2 if collect_history else 0
    hist = (C.c_double * (3 * cap))() if cap else None
    c.history = C.cast(hist, C.POINTER(C.c_double)) if cap else None
    c.history_capacity = cap
    st = abi.CellPressureStatsC()
    solver._check(lib, h, lib.femb200_solve_cell_pressure(h, C.byref(p), C.byref(c), C.byref(st)))
    history = [(int(hist[3 * i]), hist[3 * i + 1], hist[3 * i + 2]) for i in range(st.history_len)] if cap else []
    return {"converged": bool(st.converged), "iterations": st.iterations, "residual": st.residual,
            "history": history, "err_v": st.err_v, "err_P": st.err_P, "iter": st.iterations, "err": st.residual,
            "reached_total_iter": bool(st.reached_total_iter)}


def solve_adjoint_cell_pressure(dr: CellPressureStokesDR, bc_v, objective_v, lam_v=None, lam_P=None,
                                throw_on_failure=True, tolerance=1e-5, max_iterations=3000, check_interval=100,
                                velocity_step=0.6, pressure_step=0.2):
    """solve_adjoint!(dr::CellPressureStokesDR, mesh, bc_v; objective_v, λv, λP)
    (src/stokes/solvers/DR_adjoint.jl:446-484): the viscous operator is symmetric and linear,
    so the adjoint (∂R/∂u)ᵀλ = ∂J/∂u is the forward relaxation with `objective_v` (three nodal
    arrays) as the momentum load, zero density and gravity and homogeneous conditions on
    the nodes of `bc_v`. `lam_v` (three nodal arrays) and `lam_P` (4·nels) are the initial
    iterate and are overwritten (zeros when omitted); dr.v and dr.P are left unchanged.
    Returns (lam_v, lam_P, stats)."""
    import torch
    from . import solver
    dev = dr.device
    lam_v = [torch.zeros(dr.mesh.nnodes, dtype=torch.float64, device=dev) for _ in range(3)] if lam_v is None else lam_v
    lam_P = torch.zeros(4 * dr.mesh.nels, dtype=torch.float64, device=dev) if lam_P is None else lam_P
    if len(objective_v) != 3 or any(len(o) != dr.mesh.nnodes for o in objective_v):
        raise ValueError("objective_v must have mesh.nnodes entries per component")
    lib, h = solver._Handle.get()
    zero_bc = []
    for c in range(3):
        bc = bc_v[c]
        dofs = bc.DoFs if isinstance(bc, prob.DirichletBoundaryCondition) else bc[0]
        zero_bc.append((np.asarray(dofs.cpu() if hasattr(dofs, "cpu") else dofs), np.zeros(len(dofs))))
    p = dr.problem(zero_bc, load=objective_v)
    for i in range(abi.MAX_PHASES):
        p.rho[i] = 0.0
    for c in range(3):
        p.g[c] = 0.0
        p.v[c] = solver._ptr(lam_v[c])
    p.P = solver._ptr(lam_P)
    c = abi.CellPressureControlsC()
    c.tolerance, c.max_iterations, c.check_interval = tolerance, max_iterations, check_interval
    c.velocity_step, c.pressure_step, c.throw_on_failure = velocity_step, pressure_step, 0
    st = abi.CellPressureStatsC()
    solver._check(lib, h, lib.femb200_solve_cell_pressure(h, C.byref(p), C.byref(c), C.byref(st)))
    stats = {"converged": bool(st.converged), "iterations": st.iterations, "residual": st.residual,
             "err_v": st.err_v, "err_P": st.err_P, "iter": st.iterations, "err": st.residual,
             "reached_total_iter": bool(st.reached_total_iter)}
    if not st.converged and throw_on_failure:
        raise abi.FemB200Error(abi.ENOTCONV, f"3-D Stokes adjoint solve did not converge after {st.iterations} "
                                             f"iterations (residual = {st.residual:g}, tolerance = {tolerance:g})")
    return lam_v, lam_P, stats


def stokes_material_gradient_3d(dr: CellPressureStokesDR, adjoint_velocity):
    """stokes_material_gradient_3d(dr::CellPressureStokesDR, mesh, adjoint_velocity)
    (src/stokes/solvers/DR_adjoint.jl:486-531): per phase, the adjoint contracted with the
    derivative of the momentum residual in that phase's density (the load at v = 0, P = 0
    with ρ = e_phase) and in its viscosity (the viscous residual of dr.v with η = e_phase,
    no load): density_gradient[p] = −λ·∂R/∂ρ_p, viscosity_gradient[p] = −λ·∂R/∂η_p.
    Both residuals are device assemblies; the contractions are device dot products."""
    import torch
    from . import solver
    lib, h = solver._Handle.get()
    n = len(dr.material.eta)
    nn, ne = dr.mesh.nnodes, dr.mesh.nels
    zero_v = [torch.zeros(nn, dtype=torch.float64, device=dr.device) for _ in range(3)]
    zero_P = torch.zeros(4 * ne, dtype=torch.float64, device=dr.device)
    R = [torch.empty(nn, dtype=torch.float64, device=dr.device) for _ in range(3)]
    lam = [torch.as_tensor(x, dtype=torch.float64, device=dr.device).reshape(-1) for x in adjoint_velocity]

    def contract(v, eta, rho, g):
        p = dr.problem()
        for i in range(abi.MAX_PHASES):
            p.eta[i] = eta[i] if i < n else 0.0
            p.rho[i] = rho[i] if i < n else 0.0
        for c in range(3):
            p.g[c] = g[c]
            p.v[c], p.Rv[c] = solver._ptr(v[c]), solver._ptr(R[c])
        p.P = solver._ptr(zero_P)
        solver._check(lib, h, lib.femb200_cell_pressure_residuals(h, C.byref(p), 2))
        return -float(sum(torch.dot(lam[c], R[c]) for c in range(3)))

    unit = lambda k: [1.0 if i == k else 0.0 for i in range(n)]
    dens = tuple(contract(zero_v, dr.material.eta, unit(k), dr.material.g) for k in range(n))
    visc = tuple(contract(dr.v, unit(k), [0.0] * n, (0.0, 0.0, 0.0)) for k in range(n))
    return {"density_gradient": dens, "viscosity_gradient": visc}
