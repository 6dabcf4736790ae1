"""Seeded synthetic configurations (the benchmark workloads and test problems).

Each case holds host (numpy) inputs and materialises them as a device StokesDR;
`host_state(binding)` builds the same problem through any host binding with the
HostStokes interface (the tests pass the CPU oracle's), so both sides see
bit-identical inputs.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _abi as abi
from . import mesh as _mesh
from . import problem as _problem


class _Fem:
    """Namespace shim: the builders below use the package's public names."""
    structured_mixed_mesh = staticmethod(_mesh.structured_mixed_mesh)
    element_tables = staticmethod(_mesh.element_tables)
    StokesMaterial = _problem.StokesMaterial
    DruckerPrager = _problem.DruckerPrager
    DirichletBoundaryCondition = _problem.DirichletBoundaryCondition
    mesh = _mesh


fem = _Fem


@dataclass
class StokesCase:
    mesh: object
    material: object
    plastic: object
    dt: float
    phases_v: Optional[np.ndarray] = None
    phases_v_layout: int = abi.PHASE_NODAL
    phases_P: Optional[np.ndarray] = None
    phases_P_layout: int = abi.PHASE_NODAL
    v: list = field(default_factory=list)
    P: Optional[np.ndarray] = None
    P0: Optional[np.ndarray] = None
    T: Optional[np.ndarray] = None
    T0: Optional[np.ndarray] = None
    tau_old: Optional[list] = None
    bc: list = field(default_factory=list)    # (dofs 1-based, vals) per component
    gammaP: Optional[np.ndarray] = None
    M_P: Optional[np.ndarray] = None
    Pnum: Optional[np.ndarray] = None

    def device_state(self, fem_=None, dtype=None, geometry_dtype=None):
        import torch
        from .solver import StokesDR
        dr = StokesDR(self.mesh, self.material, self.plastic, phases_v=self.phases_v,
                           phases_v_layout=self.phases_v_layout, phases_P=self.phases_P,
                           phases_P_layout=self.phases_P_layout, dtype=dtype, geometry_dtype=geometry_dtype)
        for c, x in enumerate(self.v):
            dr.v[c].copy_(dr.tensor(x))
        for name in ("P", "P0", "T", "T0", "gammaP", "M_P", "Pnum"):
            x = getattr(self, name)
            if x is not None:
                getattr(dr, name).copy_(dr.tensor(x))
        if self.tau_old is not None:
            for c, x in enumerate(self.tau_old):
                dr.tau_old[c].copy_(dr.tensor(x))
        torch.cuda.synchronize()
        return dr

    def bc_device(self):
        return [fem.DirichletBoundaryCondition(d, v) for d, v in self.bc]

    def host_state(self, oh):
        hs = oh.HostStokes(self.mesh, self.material, self.plastic, phases_v=self.phases_v,
                           phases_v_layout=self.phases_v_layout, phases_P=self.phases_P,
                           phases_P_layout=self.phases_P_layout)
        for c, x in enumerate(self.v):
            hs.v[c][:] = x
        for name in ("P", "P0", "T", "T0", "gammaP", "M_P", "Pnum"):
            x = getattr(self, name)
            if x is not None:
                getattr(hs, name)[:] = x
        if self.tau_old is not None:
            for c, x in enumerate(self.tau_old):
                hs.tau_old[c][:] = x
        hs.set_bc(self.bc)
        return hs


def vep_layers_case(n=4, seed=0, dt=0.1, eta_reg=1e-2, Kb=10.0, bulk=10.0, plastic=True):
    """3-D Hex27/P1-disc visco-elasto-plastic Stokes on the unit cube, n³ cells:
    three horizontal layers with interfaces z1 < z2 ~ U(0.3, 0.7), per-phase
    η = 10^U(0,3), G = 1, cohesion U(0.1, 1), ϕ = 30°, ψ = 0, ρ0 = 1, g = (0,0,−1),
    pure-shear wall velocities vx = x − ½, vy = 0, vz = −(z − ½) (ε̇ = 1), seeded.

    Fixed here (the configuration leaves them open): Δt = 0.1 and η_reg = 1e-2, the
    values of the reference's visco-elasto-plastic shear-band example
    (examples/miniapps/stokes/vevp/stokes_2D_shear_bands_triangle.jl:51-76), and a
    storage modulus ηb = K = Kb = 10 (the example's 100 needs ~5× more Powell–Hestenes
    iterations at 64³; the StokesMaterial default is ηb = 1). Kb must be finite because
    ψ = 0 makes Kb·Δt·sinΨ·sinϕ = Inf·0 otherwise."""
    rng = np.random.default_rng(seed)
    z1, z2 = np.sort(rng.uniform(0.3, 0.7, size=2))
    eta = tuple(10.0 ** rng.uniform(0.0, 3.0, size=3))
    C = tuple(rng.uniform(0.1, 1.0, size=3))
    mesh = fem.structured_mixed_mesh(3, (n, n, n))
    zc = fem.mesh.cell_centroids(mesh)[:, 2]
    phase = np.where(zc < z1, 1, np.where(zc < z2, 2, 3)).astype(np.int32)
    mat = fem.StokesMaterial(eta=eta, eta_b=(bulk,) * 3, G=(1.0,) * 3, alpha=(0.0,) * 3, rho0=(1.0,) * 3,
                             K=(bulk,) * 3, g=(0.0, 0.0, -1.0), Tref=0.0)
    pl = fem.DruckerPrager.from_angles((math.radians(30),) * 3, (0.0,) * 3, C, (eta_reg,) * 3, (Kb,) * 3) \
        if plastic else None
    x, y, z = mesh.coords.T
    fields = [x - 0.5, np.zeros_like(y), -(z - 0.5)]
    b = mesh.boundary_nodes
    bc = [(b, f[b - 1].copy()) for f in fields]
    case = StokesCase(mesh, mat, pl, dt, phases_v=phase, phases_v_layout=abi.PHASE_CELL, phases_P=phase,
                      phases_P_layout=abi.PHASE_CELL, v=[f.copy() for f in fields],
                      P=np.zeros(mesh.nnodesP), P0=np.zeros(mesh.nnodesP), T=np.zeros(mesh.nnodesP),
                      T0=np.zeros(mesh.nnodesP), tau_old=[np.zeros(mesh.nq * mesh.nels) for _ in range(6)], bc=bc)
    case.meta = dict(z1=z1, z2=z2, eta=eta, C=C)
    return case


def inclusion_2d_case(n=64, dt=1.0):
    """2-D Q9/P1-disc plane-strain viscous Stokes on the unit square: circular inclusion
    r = 0.1 at (½, ½) with η = 1e3, ρ = 1.1 in a matrix η = 1, ρ = 1; g = (0, −1); free
    slip on all walls (vx = 0 on x ∈ {0,1}, vy = 0 on y ∈ {0,1})."""
    mesh = fem.structured_mixed_mesh(2, (n, n))
    c = fem.mesh.cell_centroids(mesh)
    phase = np.where(np.hypot(c[:, 0] - 0.5, c[:, 1] - 0.5) < 0.1, 2, 1).astype(np.int32)
    mat = fem.StokesMaterial(eta=(1.0, 1e3), eta_b=(math.inf, math.inf), G=(math.inf, math.inf), alpha=(0.0, 0.0),
                             rho0=(1.0, 1.1), K=(math.inf, math.inf), g=(0.0, -1.0))
    bx = fem.mesh.wall_nodes(mesh, 0)
    by = fem.mesh.wall_nodes(mesh, 1)
    bc = [(bx, np.zeros(len(bx))), (by, np.zeros(len(by)))]
    return StokesCase(mesh, mat, None, dt, phases_v=phase, phases_v_layout=abi.PHASE_CELL, phases_P=phase,
                      phases_P_layout=abi.PHASE_CELL, v=[np.zeros(mesh.nnodes)] * 2, P=np.zeros(mesh.nnodesP),
                      P0=np.zeros(mesh.nnodesP), T=np.zeros(mesh.nnodesP), T0=np.zeros(mesh.nnodesP),
                      tau_old=[np.zeros(mesh.nq * mesh.nels) for _ in range(3)], bc=bc)


def random_state_case(dim=3, n=3, seed=0, phases="nodal", plastic=True, nphases=3, elastic=True, distort=True):
    """Random fields for element-level parity: random v, P, P0, T, T0, τ_old, γP, M_P
    and phases in one of the three layouts, on a structured mesh whose interior nodes
    are perturbed (non-affine cells, `distort`) or sheared (affine cells)."""
    rng = np.random.default_rng(seed)
    mesh = fem.structured_mixed_mesh(dim, (n,) * dim)
    coords = mesh.coords.copy()
    if distort:
        # distort interior nodes (keeps elements valid) so J⁻¹ varies within a cell
        h = 1.0 / (2 * n)
        interior = np.all((coords > 1e-12) & (coords < 1 - 1e-12), axis=1)
        coords[interior] += rng.uniform(-0.15 * h, 0.15 * h, size=(interior.sum(), dim))
    else:
        # an affine shear keeps every cell a parallelepiped with a full J⁻¹
        coords[:, 0] += 0.2 * coords[:, 1]
        if dim == 3:
            coords[:, 1] += 0.1 * coords[:, 2]
    geo_v, geo_P = fem.mesh.precompute_geometry(coords, mesh.el2n, fem.element_tables(dim))
    mesh.coords, mesh.geo_v, mesh.geo_P = coords, geo_v, geo_P
    ph = nphases
    mat = fem.StokesMaterial(eta=tuple(10 ** rng.uniform(0, 2, ph)), eta_b=tuple(rng.uniform(5, 50, ph)),
                             G=tuple(rng.uniform(0.5, 3, ph)) if elastic else (math.inf,) * ph,
                             alpha=tuple(rng.uniform(0, 0.1, ph)), rho0=tuple(rng.uniform(1, 2, ph)),
                             K=tuple(rng.uniform(10, 100, ph)), g=(0.0, -1.0) if dim == 2 else (0.0, 0.3, -1.0),
                             Tref=0.1)
    pl = fem.DruckerPrager.from_angles(tuple(rng.uniform(0.3, 0.6, ph)), tuple(rng.uniform(0.0, 0.2, ph)),
                                       tuple(rng.uniform(0.05, 0.3, ph)), tuple(rng.uniform(0.01, 0.1, ph)),
                                       tuple(rng.uniform(1, 10, ph))) if plastic else None
    nv, npd = mesh.nv, mesh.np_
    if phases == "nodal":
        pv, lv = rng.integers(1, ph + 1, mesh.nnodes).astype(np.int32), abi.PHASE_NODAL
        pp, lp = rng.integers(1, ph + 1, mesh.nnodesP).astype(np.int32), abi.PHASE_NODAL
    elif phases == "cell":
        pv = rng.integers(1, ph + 1, mesh.nels).astype(np.int32)
        lv, pp, lp = abi.PHASE_CELL, pv, abi.PHASE_CELL
    else:
        pv, lv = rng.integers(1, ph + 1, (mesh.nels, nv)).astype(np.int32), abi.PHASE_ELEMENT_NODE
        pp, lp = rng.integers(1, ph + 1, (mesh.nels, npd)).astype(np.int32), abi.PHASE_ELEMENT_NODE
    nt = 6 if dim == 3 else 3
    case = StokesCase(mesh, mat, pl, 0.7, phases_v=pv, phases_v_layout=lv, phases_P=pp, phases_P_layout=lp,
                      v=[rng.standard_normal(mesh.nnodes) for _ in range(dim)],
                      P=rng.standard_normal(mesh.nnodesP) * 0.3, P0=rng.standard_normal(mesh.nnodesP) * 0.3,
                      T=rng.standard_normal(mesh.nnodesP), T0=rng.standard_normal(mesh.nnodesP),
                      tau_old=[rng.standard_normal(mesh.nq * mesh.nels) * 0.3 for _ in range(nt)],
                      gammaP=rng.uniform(1, 5, mesh.nnodesP), M_P=rng.uniform(0.01, 0.1, mesh.nnodesP),
                      Pnum=rng.standard_normal(mesh.nnodesP) * 0.1,
                      bc=[(mesh.boundary_nodes, np.zeros(len(mesh.boundary_nodes)))] * dim)
    return case


@dataclass
class AdjointCase:
    """Stokes part of the adjoint workload: a forward StokesCase with the viscosity
    given per integration point as η_q = exp(−0.1·T_q)·exp(δ_e) (δ_e one log-viscosity
    per element), an objective J = Σ_top |v − v_target|² over the top-surface nodes,
    and the temperature frozen on the pressure DoFs."""
    case: StokesCase
    T_ip: np.ndarray        # temperature at the integration points (nq × nels)
    delta: np.ndarray       # per-element log-viscosity perturbation
    top: np.ndarray         # 1-based top-surface nodes
    v_target: list          # target velocity per component on all nodes (zero off the top)

    def eta_ip(self, delta=None):
        d = self.delta if delta is None else delta
        nq = self.case.mesh.nq
        return np.exp(-0.1 * self.T_ip) * np.repeat(np.exp(d), nq)

    def objective(self, v):
        """J and ∂J/∂v (numpy or torch velocity components)."""
        top = self.top - 1
        J = 0.0
        grad = []
        for c in range(3):
            x = v[c].detach().double().cpu().numpy() if hasattr(v[c], "detach") else np.asarray(v[c])
            diff = np.zeros_like(x)
            diff[top] = x[top] - self.v_target[c][top]
            J += float(np.sum(diff[top] ** 2))
            grad.append(2.0 * diff)
        return J, grad


def adjoint_case(n=4, seed=0, eta_b=10.0, alpha=0.1):
    """3-D Hex27/P1-disc viscous Stokes on the unit cube for the adjoint gradient:
    temperature linear from 1 at the bottom to 0 at the top plus N(0, 0.01²) noise on
    the pressure DoFs (frozen), ρ = ρ0(1 − α(T − 0)), g = (0, 0, −1), viscosity
    η = exp(−0.1·T)·exp(δ_e) with δ_e ~ N(0, 0.1²) per element; free slip on the
    sides and the bottom, a free top surface; J = Σ_top |v − v_target|² with a seeded
    target. Fixed here (the configuration leaves them open): ηb = 10, α = 0.1, Δt = 1."""
    rng = np.random.default_rng(seed)
    mesh = fem.structured_mixed_mesh(3, (n, n, n))
    nels, nq = mesh.nels, mesh.nq
    zc = fem.mesh.cell_centroids(mesh)[:, 2]
    h = 1.0 / n
    # P1-disc DoFs of T = 1 − z: the centre value and the centre plus one half-cell slope
    Tdof = np.zeros((nels, 4))
    Tc = 1.0 - zc
    Tdof[:, 0] = Tc
    Tdof[:, 1] = Tc
    Tdof[:, 2] = Tc
    Tdof[:, 3] = Tc - 0.5 * h
    Tdof += rng.normal(0.0, 0.01, size=Tdof.shape)
    T = np.zeros(mesh.nnodesP)
    T[mesh.dofsP.reshape(-1) - 1] = Tdof.reshape(-1)
    tabs = fem.element_tables(3)
    T_ip = (Tdof @ tabs.NP.T).reshape(-1)          # nels × nq, element-major
    delta = rng.normal(0.0, 0.1, size=nels)
    mat = fem.StokesMaterial(eta=(1.0,), eta_b=(eta_b,), G=(math.inf,), alpha=(alpha,), rho0=(1.0,), K=(math.inf,),
                             g=(0.0, 0.0, -1.0), Tref=0.0)
    bx = fem.mesh.wall_nodes(mesh, 0)
    by = fem.mesh.wall_nodes(mesh, 1)
    bz = fem.mesh.wall_nodes(mesh, 2, hi=-1.0)   # bottom only
    bc = [(bx, np.zeros(len(bx))), (by, np.zeros(len(by))), (bz, np.zeros(len(bz)))]
    z = mesh.coords[:, 2]
    top = (np.nonzero(np.abs(z - 1.0) < 1e-12)[0] + 1).astype(np.int32)
    v_target = [np.zeros(mesh.nnodes) for _ in range(3)]
    for c in range(3):
        v_target[c][top - 1] = rng.normal(0.0, 0.01, size=len(top))
    case = StokesCase(mesh, mat, None, 1.0, v=[np.zeros(mesh.nnodes) for _ in range(3)], P=np.zeros(mesh.nnodesP),
                      P0=np.zeros(mesh.nnodesP), T=T, T0=T.copy(), tau_old=[np.zeros(nq * nels) for _ in range(6)],
                      bc=bc)
    return AdjointCase(case, T_ip, delta, top, v_target)


def shear_band_2d_case(n=256, seed=0, dt=0.1, eta_reg=1.0, Kb=10.0, bulk=10.0):
    """2-D plane-strain Q9/P1-disc visco-elasto-plastic shear-band experiment on the unit
    square, n² cells: matrix η = 1e2 with a seeded weak inclusion of radius 0.02 and
    η = 1 (position uniform in [0.4, 0.6]²), G = 1, cohesion 0.5, ϕ = 30°, ψ = 0,
    simple-shear boundary velocities vx = y − ½, vy = 0 on all walls.

    Fixed here (the configuration leaves them open): Δt = 0.1, Kb = ηb = K = 10 (the
    3-D layered case's values) and the Perzyna viscosity η_reg = 1: the reference's
    shear-band example notes that values well below it diverge the DR iteration on
    fine meshes (examples/miniapps/stokes/vevp/stokes_2D_shear_bands_triangle.jl:42-44),
    and 1e-2 does so here once the first points yield."""
    rng = np.random.default_rng(seed)
    cx, cy = rng.uniform(0.4, 0.6, size=2)
    mesh = fem.structured_mixed_mesh(2, (n, n))
    c = fem.mesh.cell_centroids(mesh)
    phase = np.where(np.hypot(c[:, 0] - cx, c[:, 1] - cy) < 0.02, 2, 1).astype(np.int32)
    mat = fem.StokesMaterial(eta=(1e2, 1.0), eta_b=(bulk, bulk), G=(1.0, 1.0), alpha=(0.0, 0.0), rho0=(1.0, 1.0),
                             K=(bulk, bulk), g=(0.0, 0.0), Tref=0.0)
    pl = fem.DruckerPrager.from_angles((math.radians(30),) * 2, (0.0,) * 2, (0.5, 0.5), (eta_reg,) * 2, (Kb,) * 2)
    x, y = mesh.coords.T
    b = mesh.boundary_nodes
    fields = [y - 0.5, np.zeros_like(y)]
    bc = [(b, f[b - 1].copy()) for f in fields]
    case = StokesCase(mesh, mat, pl, dt, phases_v=phase, phases_v_layout=abi.PHASE_CELL, phases_P=phase,
                      phases_P_layout=abi.PHASE_CELL, v=[f.copy() for f in fields], P=np.zeros(mesh.nnodesP),
                      P0=np.zeros(mesh.nnodesP), T=np.zeros(mesh.nnodesP), T0=np.zeros(mesh.nnodesP),
                      tau_old=[np.zeros(mesh.nq * mesh.nels) for _ in range(3)], bc=bc)
    case.meta = dict(center=(cx, cy))
    return case


@dataclass
class CellPressureCase:
    """A sinking-block configuration of the cell-pressure Hex27 solver: mesh, material,
    one phase per cell and free-slip walls (wall-normal velocity fixed to zero)."""
    mesh: object
    material: object
    phases: np.ndarray
    bc: list            # per component: (DoFs, vals)


def cell_pressure_case(n=4, seed=0, distort=True, eta=(1.0, 100.0), rho=(1.0, 1.5), half_width=0.25):
    """Hex27 n³ on the unit cube (interior nodes perturbed by up to 15 % of the node
    spacing when `distort`), a dense viscous block |x − ½|, |y − ½|, |z − ½| < half_width
    (phase 2, by cell centroid) in a phase-1 matrix, g = (0, 0, −1), free slip on every wall
    (the setup of the reference's 3-D sinking-block example, on a structured mesh)."""
    rng = np.random.default_rng(seed)
    mesh = _mesh.structured_mixed_mesh(3, (n, n, n))
    coords = mesh.coords.copy()
    if distort:
        h = 1.0 / (2 * n)
        interior = np.all((coords > 1e-12) & (coords < 1 - 1e-12), axis=1)
        coords[interior] += rng.uniform(-0.15 * h, 0.15 * h, size=(interior.sum(), 3))
        geo_v, geo_P = _mesh.precompute_geometry(coords, mesh.el2n, _mesh.element_tables(3))
        mesh.coords, mesh.geo_v, mesh.geo_P = coords, geo_v, geo_P
    cen = _mesh.cell_centroids(mesh)
    inside = np.all(np.abs(cen - 0.5) < half_width, axis=1)
    phases = np.where(inside, 2, 1).astype(np.int32)
    material = _problem.StokesMaterial(eta=eta, rho0=rho, g=(0.0, 0.0, -1.0))
    tol = 32 * np.finfo(float).eps
    bc = []
    for d in range(3):
        on = (np.abs(mesh.coords[:, d]) <= tol) | (np.abs(mesh.coords[:, d] - 1.0) <= tol)
        dofs = (np.nonzero(on)[0] + 1).astype(np.int32)
        bc.append((dofs, np.zeros(len(dofs))))
    return CellPressureCase(mesh, material, phases, bc)
