"""Device-side StokesDR / ThermalDiffusionDR states and the solve API over libfemtools_b200.

Mirrors the reference's user API (src/stokes/solvers/DR.jl:89, :241, :302;
src/heat_diffusion/solvers/DR.jl:50): `solve`, `solve_stokes_dyrel`,
`solve_coupled`, `solve_thermal` and the low-level assemblers. State lives in
torch CUDA tensors (torch is used for device memory and streams only); every
computation is a libfemtools_b200 kernel. There is no CPU fallback: without the
library or a CUDA device these calls raise.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional, Sequence

import numpy as np

from . import _abi as abi
from . import problem as prob
from .mesh import MixedMesh

try:
    import torch
except ImportError:  # pragma: no cover - torch is part of the image
    torch = None


def _require_cuda():
    if torch is None or not torch.cuda.is_available():
        raise RuntimeError("libfemtools_b200 needs a CUDA device (sm_100a); no CPU fallback exists")


class _Handle:
    """One femb200_handle per process (created on the current CUDA device)."""
    _h = None

    @classmethod
    def get(cls):
        _require_cuda()
        lib = abi.load_library()
        if cls._h is None:
            h = C.c_void_p()
            rc = lib.femb200_create(C.byref(h))
            if rc != abi.OK:
                raise abi.FemB200Error(rc, "femb200_create failed (no usable CUDA device?)")
            cls._h = h
        lib.femb200_set_stream(cls._h, C.c_void_p(torch.cuda.current_stream().cuda_stream))
        return lib, cls._h


def _check(lib, h, rc):
    if rc != abi.OK:
        raise abi.FemB200Error(rc, lib.femb200_last_error(h).decode())


def _ptr(t):
    if t is None:
        return 0
    if isinstance(t, torch.Tensor):
        assert t.is_cuda and t.is_contiguous(), "device arrays must be contiguous CUDA tensors"
        return t.data_ptr()
    raise TypeError(f"expected a CUDA tensor, got {type(t)}")


_DT = {torch.float64: abi.F64, torch.float32: abi.F32} if torch is not None else {}


class StokesDR:
    """Stokes DR state on the device (StokesDR, src/stokes/types/stokes_types.jl:197-298).

    Velocity-node fields v, rate (∂v∂τ), Rv, Rv0, dRdv (∂Rv∂v), PC; pressure-DoF fields
    P, P0, gammaP (γP), T, T0, Q, Pf, RP, M_P, Pnum; integration-point stress history
    tau_old and current stress tau (nq × nels, assembler order).
    """

    def __init__(self, mesh: MixedMesh, material: prob.StokesMaterial, plastic: Optional[prob.DruckerPrager] = None,
                 phases_v=None, phases_v_layout=abi.PHASE_NODAL, phases_P=None, phases_P_layout=abi.PHASE_NODAL,
                 dtype=None, geometry_dtype=None, stress=True, CFL_v=0.98, c_fact=0.9):
        _require_cuda()
        if material.dim != mesh.dim:
            raise ValueError(f"material gravity must have {mesh.dim} components")
        self.mesh = mesh
        self.material = material
        self.plastic = plastic
        self.dtype = dtype or torch.float64
        self.geometry_dtype = geometry_dtype or self.dtype
        self.CFL_v, self.c_fact = CFL_v, c_fact
        dev = torch.device("cuda")
        self.device = dev
        dim, nn, nP = mesh.dim, mesh.nnodes, mesh.nnodesP
        z = lambda n: torch.zeros(n, dtype=self.dtype, device=dev)
        self.v = [z(nn) for _ in range(dim)]
        self.rate = [z(nn) for _ in range(dim)]
        self.Rv = [z(nn) for _ in range(dim)]
        self.Rv0 = [z(nn) for _ in range(dim)]
        self.dRdv = [z(nn) for _ in range(dim)]
        self.PC = [z(nn) for _ in range(dim)]
        for name in ("P", "P0", "gammaP", "T", "T0", "Q", "Pf", "RP", "M_P", "Pnum"):
            setattr(self, name, z(nP))
        nt = 6 if dim == 3 else 3
        nqe = mesh.nq * mesh.nels
        self.tau_old = [z(nqe) for _ in range(nt)] if stress else None
        self.tau = [z(nqe) for _ in range(nt)] if stress else None
        i32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.int32), device=dev)
        self.phases_v = i32(phases_v) if phases_v is not None else torch.ones(nn, dtype=torch.int32, device=dev)
        self.phases_v_layout = phases_v_layout if phases_v is not None else abi.PHASE_NODAL
        self.phases_P = i32(phases_P) if phases_P is not None else torch.ones(nP, dtype=torch.int32, device=dev)
        self.phases_P_layout = phases_P_layout if phases_P is not None else abi.PHASE_NODAL
        gdt = self.geometry_dtype
        self._mesh = {
            "dim": dim, "nels": mesh.nels, "nnodes": nn, "nnodesP": nP,
            "el2n": i32(mesh.el2n), "dofsP": i32(mesh.dofsP), "el2nP": i32(mesh.el2nP),
            "geo_v": torch.as_tensor(mesh.geo_v, device=dev).to(gdt).contiguous(),
            "geo_P": torch.as_tensor(mesh.geo_P, device=dev).to(gdt).contiguous(),
        }
        self.P_old = None
        self.P_old_layout = abi.FIELD_NODAL
        self.viscosity_ip = None
        self.body_force = None
        self._use_Q = False
        self._use_Pf = False

    # ---- helpers ----
    def tensor(self, x, dtype=None):
        return torch.as_tensor(np.asarray(x), dtype=dtype or self.dtype, device=self.device).contiguous()

    def set_velocity(self, comps):
        for c, x in enumerate(comps):
            self.v[c].copy_(self.tensor(x))

    def _state(self):
        return {
            "v": self.v, "rate": self.rate, "Rv": self.Rv, "Rv0": self.Rv0, "dRdv": self.dRdv, "PC": self.PC,
            "P": self.P, "P0": self.P0, "gammaP": self.gammaP, "T": self.T, "T0": self.T0,
            "Q": self.Q if self._use_Q else None, "Pf": self.Pf if self._use_Pf else None,
            "RP": self.RP, "M_P": self.M_P, "Pnum": self.Pnum,
            "phases_v": self.phases_v, "phases_v_layout": self.phases_v_layout,
            "phases_P": self.phases_P, "phases_P_layout": self.phases_P_layout,
            "tau_old": self.tau_old, "tau": self.tau,
            "tau_old_layout": abi.FIELD_IP if self.tau_old is not None else abi.FIELD_NONE,
            "P_old": self.P_old, "P_old_layout": self.P_old_layout,
            "viscosity_ip": self.viscosity_ip, "body_force": self.body_force,
        }

    def problem(self, bc_v: Optional[Sequence] = None, scaling_viscosity=None) -> abi.StokesProblemC:
        s = abi.StokesProblemC()
        mat = prob.material_struct(self.material, self.plastic, scaling_viscosity)
        bcs = []
        for c in range(self.mesh.dim):
            if bc_v is None or c >= len(bc_v) or bc_v[c] is None:
                bcs.append(None)
                continue
            bc = bc_v[c]
            dofs = bc.DoFs if isinstance(bc, prob.DirichletBoundaryCondition) else bc[0]
            vals = bc.vals if isinstance(bc, prob.DirichletBoundaryCondition) else bc[1]
            bcs.append((self.tensor(dofs, torch.int32) if not isinstance(dofs, torch.Tensor) else dofs,
                        self.tensor(vals) if not isinstance(vals, torch.Tensor) else vals))
        self._keep = bcs   # keep the device copies alive while the struct is in use
        prob.fill_stokes_problem(s, self._mesh, self._state(), mat, bcs, _ptr, _DT[self.dtype],
                                 _DT[self.geometry_dtype])
        return s


def assemble_pressure_residual(dr: StokesDR, dt, finite_K=False):
    """assemble_pressure_residual_kernel! (pressure_residual.jl:256) into dr.RP."""
    lib, h = _Handle.get()
    _check(lib, h, lib.femb200_pressure_residual(h, C.byref(dr.problem()), float(dt), int(finite_K)))


def assemble_momentum_residual(dr: StokesDR, dt, with_pnum=False):
    """assemble_momentum_residual_kernel! (momentum_residuals.jl:417) into dr.Rv (Pnum = dr.Pnum or nothing)."""
    lib, h = _Handle.get()
    _check(lib, h, lib.femb200_momentum_residual(h, C.byref(dr.problem()), float(dt), int(with_pnum)))


def assemble_stokes_residuals(dr: StokesDR, dt, finite_K=False):
    """Fused DR sweep: RP, Pnum = γP·RP/M_P and Rv in one pass (DR.jl:665-684)."""
    lib, h = _Handle.get()
    _check(lib, h, lib.femb200_stokes_residuals(h, C.byref(dr.problem()), float(dt), int(finite_K)))


def assemble_augmented_momentum_jacobian(dr: StokesDR, dt, finite_K=False):
    """assemble_augmented_momentum_jacobian_matrices_atomix! (momentum_residuals.jl:998) into dr.dRdv, dr.PC."""
    lib, h = _Handle.get()
    _check(lib, h, lib.femb200_jacobian_diagnostics(h, C.byref(dr.problem()), float(dt), int(finite_K)))


def assemble_viscosity_weighted_pressure_scaling(dr: StokesDR, pressure_factor, dt, finite_K=False,
                                                 scaling_viscosity=None):
    """assemble_viscosity_weighted_pressure_scaling! (pressure_scaling.jl:118) into dr.M_P, dr.gammaP."""
    lib, h = _Handle.get()
    _check(lib, h, lib.femb200_pressure_scaling(h, C.byref(dr.problem(scaling_viscosity=scaling_viscosity)),
                                                float(pressure_factor), float(dt), int(finite_K)))


def update_stokes_current_stress(dr: StokesDR, dt):
    """update_stokes_current_stress! (DR.jl:820): integration-point stress into dr.tau."""
    lib, h = _Handle.get()
    _check(lib, h, lib.femb200_store_stress(h, C.byref(dr.problem()), float(dt)))


def assemble_shear_heating(dr: StokesDR, dt, phi=None):
    """assemble_shear_heating! (shear_heating.jl:18): Φ at every velocity quadrature point."""
    lib, h = _Handle.get()
    if phi is None:
        phi = torch.zeros(dr.mesh.nq * dr.mesh.nels, dtype=dr.dtype, device=dr.device)
    _check(lib, h, lib.femb200_shear_heating(h, C.byref(dr.problem()), float(dt), C.c_void_p(_ptr(phi))))
    return phi


def _controls(dt, **kw):
    history_capacity = kw.pop("history_capacity", 0)
    dim = kw.pop("_dim", 3)
    hist = np.zeros((history_capacity, 4 + dim)) if history_capacity else None
    c = prob.controls_struct(dt, history=hist, **kw)
    return c, hist


def solve(dr: StokesDR, bc_v, dt, pressure_factor=50.0, tolerance=1e-6, max_iterations=50_000, check_interval=50,
          throw_on_failure=True, finite_K=False, scaling_viscosity=None, history_capacity=0, precision="fp64",
          ordered_scatter=False, **kwargs):
    """solve!(dr::StokesDR, mesh, bc_v; dt, …) (src/stokes/solvers/DR.jl:302-337).

    Assembles M_P and γP, then runs the Powell–Hestenes/DYREL iteration. Returns
    the statistics as a dict; raises FemB200Error when the solve does not converge
    and `throw_on_failure` is set, with the reference's message. With
    precision="mixed", ordered_scatter=True makes the solve reproducible bit for bit
    (femb200_set_ordered_scatter: colour-ordered scatter, about a third slower).
    """
    return _solve(dr, bc_v, dt, True, pressure_factor=pressure_factor, tolerance=tolerance,
                  max_iterations=max_iterations, check_interval=check_interval, throw_on_failure=throw_on_failure,
                  finite_K=finite_K, scaling_viscosity=scaling_viscosity, history_capacity=history_capacity,
                  precision=precision, ordered_scatter=ordered_scatter, **kwargs)


def solve_stokes_dyrel(dr: StokesDR, bc_v, dt, ncheck=50, eps_tol=1e-6, iterMax=50_000, total_iterMax=50_000,
                       max_ph_iterations=1000, rel_drop0=1e-2, history_capacity=0, **kwargs):
    """solve_stokes_dyrel!(dr, mesh, bc_v, Δt, γP; …) (DR.jl:241) with dr.M_P, dr.gammaP prepared."""
    return _solve(dr, bc_v, dt, False, check_interval=ncheck, tolerance=eps_tol, iter_max=iterMax,
                  max_iterations=total_iterMax, max_ph_iterations=max_ph_iterations, rel_drop0=rel_drop0,
                  throw_on_failure=False, history_capacity=history_capacity, **kwargs)


def _solve(dr, bc_v, dt, assemble_scaling, scaling_viscosity=None, history_capacity=0, precision="fp64",
           ordered_scatter=False, **kw):
    lib, h = _Handle.get()
    kw.setdefault("cfl_v", dr.CFL_v)
    kw.setdefault("c_fact", dr.c_fact)
    c, hist = _controls(dt, assemble_scaling=assemble_scaling, history_capacity=history_capacity,
                        _dim=dr.mesh.dim,
                        precision=abi.PRECISION_MIXED if precision == "mixed" else abi.PRECISION_FP64, **kw)
    st = abi.StokesStatsC()
    s = dr.problem(bc_v, scaling_viscosity)
    _check(lib, h, lib.femb200_set_ordered_scatter(h, 1 if ordered_scatter else 0))
    try:
        rc = lib.femb200_solve_stokes(h, C.byref(s), C.byref(c), C.byref(st))
    finally:
        lib.femb200_set_ordered_scatter(h, 0)
    _check(lib, h, rc)
    out = prob.stats_dict(st)
    out["iterations"] = out["iter"]
    out["residual"] = out["err_abs"]
    if hist is not None:
        out["history"] = hist[: st.history_len]
    return out


# ---- adjoint (src/stokes/solvers/DR_adjoint.jl) ----------------------------------

def _vec3(ts):
    return (C.c_void_p * 3)(*[C.c_void_p(_ptr(t)) for t in ts])


def assemble_adjoint_residual(dr: StokesDR, dt, lam_v, lam_P, finite_K=False, with_pnum=True):
    """(dR/du)ᵀλ at dr's state for the augmented residual (Pnum = γP·RP/M_P inline):
    returns (dv components, dP). The matrix-free apply of the reference's frozen
    adjoint operator (apply_adjoint_operator!, adjoint_operator.jl:640-660)."""
    lib, h = _Handle.get()
    z = lambda n: torch.zeros(n, dtype=dr.dtype, device=dr.device)
    dv = [z(dr.mesh.nnodes) for _ in range(3)]
    dP = z(dr.mesh.nnodesP)
    _check(lib, h, lib.femb200_stokes_adjoint_residual(h, C.byref(dr.problem()), float(dt), int(finite_K),
                                                        int(with_pnum), _vec3(lam_v), C.c_void_p(_ptr(lam_P)),
                                                        _vec3(dv), C.c_void_p(_ptr(dP))))
    return dv, dP


def viscosity_sensitivity(dr: StokesDR, dt, lam_v, lam_P, finite_K=False, with_pnum=True):
    """λ·∂R/∂η at every integration point (nq × nels): the gradient of λᵀR(u, η) in the
    viscosity field; per-element or per-phase gradients follow by the chain rule."""
    lib, h = _Handle.get()
    out = torch.zeros(dr.mesh.nq * dr.mesh.nels, dtype=dr.dtype, device=dr.device)
    _check(lib, h, lib.femb200_stokes_viscosity_sensitivity(h, C.byref(dr.problem()), float(dt), int(finite_K),
                                                             int(with_pnum), _vec3(lam_v), C.c_void_p(_ptr(lam_P)),
                                                             C.c_void_p(_ptr(out))))
    return out


def solve_adjoint(dr: StokesDR, bc_v, dt, objective_v, lam_v=None, lam_P=None, tolerance=1e-6,
                  max_iterations=50_000, check_interval=50, iter_max=50_000, max_ph_iterations=100, rel_drop=0.1,
                  throw_on_failure=True, finite_K=False):
    """solve_adjoint!(dr, mesh, bc_v; dt, objective_v, λv, λP, …) (DR_adjoint.jl:396-433).

    Solves (dR/du)ᵀλ = −objective_v at the converged forward state in `dr` (dr.gammaP
    and dr.M_P as in the forward solve) with the frozen-operator PH/DYREL iteration.
    Returns (λv, λP, stats). With J(u(m)) and R(u, m) = 0, dJ/dm = λᵀ ∂R/∂m.
    """
    lib, h = _Handle.get()
    z = lambda n: torch.zeros(n, dtype=dr.dtype, device=dr.device)
    lam_v = [z(dr.mesh.nnodes) for _ in range(3)] if lam_v is None else lam_v
    lam_P = z(dr.mesh.nnodesP) if lam_P is None else lam_P
    obj = [o.contiguous() for o in objective_v]
    c, _ = _controls(dt, tolerance=tolerance, max_iterations=max_iterations, check_interval=check_interval,
                     iter_max=iter_max, max_ph_iterations=max_ph_iterations, rel_drop0=rel_drop,
                     throw_on_failure=throw_on_failure, finite_K=finite_K, cfl_v=dr.CFL_v, c_fact=dr.c_fact)
    st = abi.StokesStatsC()
    rc = lib.femb200_solve_stokes_adjoint(h, C.byref(dr.problem(bc_v)), C.byref(c), _vec3(obj), _vec3(lam_v),
                                          C.c_void_p(_ptr(lam_P)), C.byref(st))
    _check(lib, h, rc)
    return lam_v, lam_P, prob.stats_dict(st)


def _device_coords(coords, dim):
    """Node coordinates as a contiguous FP64 device array, nnodes × dim (x fastest)."""
    c = coords if isinstance(coords, torch.Tensor) else torch.as_tensor(np.asarray(coords, dtype=np.float64))
    c = c.to(device="cuda", dtype=torch.float64).reshape(-1, dim).contiguous()
    return c


def precompute_geometry(coords, el2n, dim, geometry_dtype=None, with_P=True):
    """precompute_geometry (src/mesh/mesh.jl:592-606) and the mixed-mesh geometry
    (mixed_mesh.jl:358-392) on the device: returns (geo_v, geo_P), nels × nq × (dim² + 1)
    and nels × nq, with J⁻¹ (column-major) and |det J|·ω at every velocity integration
    point. `geometry_dtype` is the stored precision (torch.float64 or torch.float32, the
    reference's geometry_precision); J is inverted in FP64 either way."""
    lib, h = _Handle.get()
    gdt = geometry_dtype or torch.float64
    c = _device_coords(coords, dim)
    e2n = el2n if isinstance(el2n, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(el2n, dtype=np.int32))
    e2n = e2n.to(device="cuda", dtype=torch.int32).contiguous()
    nv = 27 if dim == 3 else 9
    nels = e2n.numel() // nv
    geo_v = torch.empty((nels, nv, dim * dim + 1), dtype=gdt, device="cuda")
    geo_P = torch.empty((nels, nv), dtype=gdt, device="cuda") if with_P else None
    _check(lib, h, lib.femb200_precompute_geometry(h, dim, nels, c.shape[0], _ptr(c), _ptr(e2n), _ptr(geo_v),
                                                   _ptr(geo_P), _DT[gdt]))
    return geo_v, geo_P


def update_geometry(state, coords):
    """update_geometry!(mesh) (src/mesh/mesh.jl:640-650, mixed_mesh.jl:337-345): recompute
    the geometry a StokesDR or ThermalDiffusionDR state holds, in place (the arrays keep
    their identity), from moved node coordinates (host or device, nnodes × dim)."""
    lib, h = _Handle.get()
    mesh = state.mesh
    c = _device_coords(coords, mesh.dim)
    if c.shape[0] != mesh.nnodes:
        raise ValueError(f"coords has {c.shape[0]} nodes; expected {mesh.nnodes}")
    if isinstance(state, StokesDR):
        e2n, geo_v, geo_P = state._mesh["el2n"], state._mesh["geo_v"], state._mesh["geo_P"]
    else:
        e2n, geo_v, geo_P = state.el2n, state.geo, None
    _check(lib, h, lib.femb200_precompute_geometry(h, mesh.dim, mesh.nels, mesh.nnodes, _ptr(c), _ptr(e2n),
                                                   _ptr(geo_v), _ptr(geo_P), _DT[geo_v.dtype]))
    return state


class ThermalDiffusionDR:
    """Thermal DR state on the device (heat_diffusion_types.jl:90-132)."""

    def __init__(self, mesh: MixedMesh, k=(1.0,), Cp=(1.0,), rho0=(1.0,), alpha=(0.0,), K=(math.inf,), phases=None,
                 CFL=0.98, c_fact=0.9, eps=1e-6, dtype=None):
        _require_cuda()
        self.mesh = mesh
        self.dtype = dtype or torch.float64
        dev = torch.device("cuda")
        self.device = dev
        nn = mesh.nnodes
        for name in ("T", "T0", "rate", "R", "R0", "dRdT", "PC", "P", "source"):
            setattr(self, name, torch.zeros(nn, dtype=self.dtype, device=dev))
        self.phases = (torch.as_tensor(np.ascontiguousarray(phases, dtype=np.int32), device=dev) if phases is not None
                       else torch.ones(nn, dtype=torch.int32, device=dev))
        self.mat = dict(k=tuple(k), Cp=tuple(Cp), rho0=tuple(rho0), alpha=tuple(alpha), K=tuple(K))
        self.CFL, self.c_fact, self.eps = CFL, c_fact, eps
        self.source_ip = None
        self.el2n = torch.as_tensor(np.ascontiguousarray(mesh.el2n, dtype=np.int32), device=dev)
        self.geo = torch.as_tensor(mesh.geo_v, device=dev).to(self.dtype).contiguous()
        self.bc = None

    def set_bc(self, bc: prob.DirichletBoundaryCondition):
        self.bc = (torch.as_tensor(np.asarray(bc.DoFs, dtype=np.int32), device=self.device),
                   torch.as_tensor(np.asarray(bc.vals), dtype=self.dtype, device=self.device))

    def problem(self) -> abi.ThermalProblemC:
        t = abi.ThermalProblemC()
        t.dim, t.dtype, t.geo_dtype = self.mesh.dim, _DT[self.dtype], _DT[self.dtype]
        t.nv, t.nq = (27, 27) if self.mesh.dim == 3 else (9, 9)
        t.nels, t.nnodes = self.mesh.nels, self.mesh.nnodes
        t.el2n, t.geo = _ptr(self.el2n), _ptr(self.geo)
        for name in ("T", "T0", "rate", "R", "R0", "dRdT", "PC", "P", "source"):
            setattr(t, name, _ptr(getattr(self, name)))
        t.source_ip = _ptr(self.source_ip)
        t.phases, t.phases_layout = _ptr(self.phases), abi.PHASE_NODAL
        if self.bc is not None:
            t.bc_dofs, t.bc_vals, t.bc_n = _ptr(self.bc[0]), _ptr(self.bc[1]), len(self.bc[0])
        n = len(self.mat["k"])
        t.nphases = n
        for name, fill in (("k", 1.0), ("Cp", 1.0), ("rho0", 1.0), ("alpha", 0.0), ("K", math.inf)):
            arr = getattr(t, name)
            vals = self.mat[name]
            for i in range(abi.MAX_PHASES):
                arr[i] = vals[i] if i < n else fill
        t.cfl, t.c_fact, t.eps = self.CFL, self.c_fact, self.eps
        return t


def assemble_thermal_residual(th: ThermalDiffusionDR, dt, Tref=273.0, compute_jacobian=False):
    lib, h = _Handle.get()
    _check(lib, h, lib.femb200_thermal_residual(h, C.byref(th.problem()), float(dt), float(Tref), int(compute_jacobian)))


def assemble_diffusion_matrices_colored(th: ThermalDiffusionDR, groups, dt, Tref=273.0, compute_jacobian=False):
    """assemble_diffusion_matrices_colored! (heat_diffusion/assembly/residual_colored.jl:10):
    one launch per colour group of `groups` (coloring.ElementGroups), plain adds."""
    lib, h = _Handle.get()
    dev = getattr(groups, "_device", None)
    if dev is None:
        dev = torch.as_tensor(groups.elements, device=th.device)
        groups._device = dev
    _check(lib, h, lib.femb200_thermal_residual_colored(h, C.byref(th.problem()), float(dt), float(Tref),
                                                        int(compute_jacobian), C.c_void_p(_ptr(dev)),
                                                        groups.offsets.ctypes.data, groups.ncolors))


def solve_thermal(th: ThermalDiffusionDR, bc, dt, Tref=273.0, tolerance=None, max_iterations=10_000,
                  check_interval=100, throw_on_failure=True):
    """solve!(dr::ThermalDiffusionDR, mesh, bc; dt) (heat_diffusion/solvers/DR.jl:50)."""
    lib, h = _Handle.get()
    th.set_bc(bc)
    c = abi.ThermalControlsC()
    c.dt, c.Tref = float(dt), float(Tref)
    c.tolerance = th.eps if tolerance is None else float(tolerance)
    c.max_iterations, c.check_interval, c.throw_on_failure = int(max_iterations), int(check_interval), int(throw_on_failure)
    st = abi.ThermalStatsC()
    _check(lib, h, lib.femb200_solve_thermal(h, C.byref(th.problem()), C.byref(c), C.byref(st)))
    return {"converged": bool(st.converged), "iterations": st.iterations, "residual": st.residual}


def solve_coupled(thermal: ThermalDiffusionDR, stokes: StokesDR, bc_T, bc_v, dt, Tref=273.0, shear_heating=False,
                  pressure_factor=50.0, tolerance=1e-6, max_iterations=50_000, check_interval=50,
                  throw_on_failure=True, history_capacity=0, **kw):
    """solve_coupled!(thermal, stokes, thermal_mesh, stokes_mesh, bc_T, bc_v; dt, …) (DR.jl:89-135)."""
    lib, h = _Handle.get()
    thermal.set_bc(bc_T)
    kw.setdefault("cfl_v", stokes.CFL_v)
    kw.setdefault("c_fact", stokes.c_fact)
    c, hist = _controls(dt, pressure_factor=pressure_factor, tolerance=tolerance, max_iterations=max_iterations,
                        check_interval=check_interval, throw_on_failure=throw_on_failure,
                        history_capacity=history_capacity, _dim=stokes.mesh.dim, assemble_scaling=True, **kw)
    phi = torch.zeros(stokes.mesh.nq * stokes.mesh.nels, dtype=stokes.dtype, device=stokes.device) if shear_heating else None
    st = abi.StokesStatsC()
    t = thermal.problem()
    rc = lib.femb200_solve_coupled(h, C.byref(t), C.byref(stokes.problem(bc_v)), C.byref(c), float(Tref),
                                   int(shear_heating), C.c_void_p(_ptr(phi)), C.byref(st))
    _check(lib, h, rc)
    out = prob.stats_dict(st)
    out["iterations"] = out["iter"]
    out["residual"] = out["err_abs"]
    if hist is not None:
        out["history"] = hist[: st.history_len]
    return out, phi
