"""Material/plasticity descriptions and the packing of a solve into the C-ABI structs.

`StokesMaterial` and `DruckerPrager` mirror src/stokes/types/stokes_types.jl:19
and :388/:415. `fill_stokes_problem` packs mesh, state and boundary arrays into a
`femb200_stokes_problem`; it is array-library agnostic (the caller supplies the
pointer function), so the same packing serves device tensors and host arrays.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Optional, Sequence

from . import _abi as abi


def _tuple(x, n=None):
    if isinstance(x, (int, float)):
        return (float(x),) * (n or 1)
    return tuple(float(v) for v in x)


@dataclass
class StokesMaterial:
    """Per-phase Stokes material (StokesMaterial, stokes_types.jl:19-60); defaults as there."""
    eta: Sequence[float] = (1.0,)
    eta_b: Optional[Sequence[float]] = None
    G: Optional[Sequence[float]] = None
    alpha: Optional[Sequence[float]] = None
    rho0: Optional[Sequence[float]] = None
    K: Optional[Sequence[float]] = None
    g: Sequence[float] = (0.0, 0.0)
    Tref: float = 0.0

    def __post_init__(self):
        self.eta = _tuple(self.eta)
        n = len(self.eta)
        self.eta_b = _tuple(1.0 if self.eta_b is None else self.eta_b, n)
        self.G = _tuple(math.inf if self.G is None else self.G, n)
        self.alpha = _tuple(0.0 if self.alpha is None else self.alpha, n)
        self.rho0 = _tuple(1.0 if self.rho0 is None else self.rho0, n)
        self.K = _tuple(math.inf if self.K is None else self.K, n)
        self.g = tuple(float(x) for x in self.g)
        for name in ("eta_b", "G", "alpha", "rho0", "K"):
            if len(getattr(self, name)) != n:
                raise ValueError("Stokes material property tuples must have the same length")
        if len(self.g) not in (2, 3):
            raise ValueError(f"gravity must have 2 or 3 components, got {len(self.g)}")
        if n > abi.MAX_PHASES:
            raise ValueError(f"at most {abi.MAX_PHASES} phases are supported")

    @property
    def nphases(self):
        return len(self.eta)

    @property
    def dim(self):
        return len(self.g)


@dataclass
class DruckerPrager:
    """Drucker–Prager parameters (stokes_types.jl:388-423): cos/sin of the angles stored."""
    cos_phi: Sequence[float]
    sin_phi: Sequence[float]
    sin_psi: Sequence[float]
    C: Sequence[float]
    eta_reg: Sequence[float]
    Kb: Sequence[float]

    @classmethod
    def from_angles(cls, phi, psi, C, eta_reg, Kb):
        """DruckerPrager(ϕ, Ψ, C, η_reg, Kb) with angles in radians."""
        phi, psi = _tuple(phi), _tuple(psi)
        return cls(tuple(math.cos(x) for x in phi), tuple(math.sin(x) for x in phi),
                   tuple(math.sin(x) for x in psi), _tuple(C), _tuple(eta_reg), _tuple(Kb))


@dataclass
class DirichletBoundaryCondition:
    """Constrained DoFs (1-based) and prescribed values (boundary_conditions.jl:30-42)."""
    DoFs: object
    vals: object

    def __post_init__(self):
        if len(self.DoFs) != len(self.vals):
            raise ValueError("boundary indices and values must have the same length")


def material_struct(mat: StokesMaterial, plastic: Optional[DruckerPrager] = None,
                    scaling_eta=None) -> abi.StokesMaterialC:
    m = abi.StokesMaterialC()
    n = mat.nphases
    m.nphases = n

    def put(dst, vals, fill):
        for i in range(abi.MAX_PHASES):
            dst[i] = vals[i] if i < n else fill

    put(m.eta, mat.eta, 1.0)
    put(m.eta_b, mat.eta_b, math.inf)
    put(m.G, mat.G, math.inf)
    put(m.alpha, mat.alpha, 0.0)
    put(m.rho0, mat.rho0, 0.0)
    put(m.K, mat.K, math.inf)
    for i in range(3):
        m.g[i] = mat.g[i] if i < len(mat.g) else 0.0
    m.Tref = mat.Tref
    if plastic is not None:
        m.plastic = 1
        for name in ("cos_phi", "sin_phi", "sin_psi", "C", "eta_reg", "Kb"):
            vals = _tuple(getattr(plastic, name), n)
            if len(vals) != n:
                raise ValueError("DruckerPrager parameters must have one entry per phase")
            put(getattr(m, name), vals, 0.0)
    if scaling_eta is not None:
        m.use_scaling_eta = 1
        put(m.scaling_eta, _tuple(scaling_eta, n), 1.0)
    return m


def fill_stokes_problem(s: abi.StokesProblemC, mesh: dict, state: dict, mat: abi.StokesMaterialC,
                        bcs: Sequence, ptr: Callable, dtype: int = abi.F64, geo_dtype: int = abi.F64):
    """Pack arrays into a femb200_stokes_problem.

    `mesh` holds el2n, dofsP, el2nP, geo_v, geo_P and the sizes; `state` the named
    state arrays (v, rate, Rv, Rv0, dRdv, PC as lists per component; P, P0, …);
    `bcs` one (dofs, vals) pair per velocity component; `ptr(x)` returns the
    address of an array (0 for None).
    """
    dim = mesh["dim"]
    s.dim = dim
    s.nv, s.np, s.nq = (27, 4, 27) if dim == 3 else (9, 3, 9)
    s.dtype, s.geo_dtype = dtype, geo_dtype
    s.nels, s.nnodes, s.nnodesP = mesh["nels"], mesh["nnodes"], mesh["nnodesP"]
    for name in ("el2n", "dofsP", "el2nP", "geo_v", "geo_P"):
        setattr(s, name, ptr(mesh[name]))
    for name in ("v", "rate", "Rv", "Rv0", "dRdv", "PC"):
        arr = getattr(s, name)
        comps = state[name]
        for c in range(3):
            arr[c] = ptr(comps[c]) if c < dim else 0
    for name in ("P", "P0", "gammaP", "T", "T0", "Q", "Pf", "RP", "M_P", "Pnum"):
        setattr(s, name, ptr(state.get(name)))
    s.phases_v = ptr(state.get("phases_v"))
    s.phases_v_layout = state.get("phases_v_layout", abi.PHASE_NODAL)
    s.phases_P = ptr(state.get("phases_P"))
    s.phases_P_layout = state.get("phases_P_layout", abi.PHASE_NODAL)
    told = state.get("tau_old")
    nt = 6 if dim == 3 else 3
    for c in range(6):
        s.tau_old[c] = ptr(told[c]) if (told is not None and c < nt) else 0
    s.tau_old_layout = state.get("tau_old_layout", abi.FIELD_IP if told is not None else abi.FIELD_NONE)
    tau = state.get("tau")
    for c in range(6):
        s.tau[c] = ptr(tau[c]) if (tau is not None and c < nt) else 0
    s.P_old = ptr(state.get("P_old"))
    s.P_old_layout = state.get("P_old_layout", abi.FIELD_NODAL)
    s.viscosity_ip = ptr(state.get("viscosity_ip"))
    bf = state.get("body_force")
    for c in range(3):
        s.body_force[c] = ptr(bf[c]) if (bf is not None and c < dim) else 0
    for c in range(3):
        if c < dim and c < len(bcs) and bcs[c] is not None:
            dofs, vals = bcs[c]
            s.bc_dofs[c], s.bc_vals[c], s.bc_n[c] = ptr(dofs), ptr(vals), len(dofs)
        else:
            s.bc_dofs[c], s.bc_vals[c], s.bc_n[c] = 0, 0, 0
    s.mat = mat
    return s


def controls_struct(dt, pressure_factor=50.0, tolerance=1e-6, max_iterations=50_000, check_interval=50,
                    iter_max=50_000, max_ph_iterations=1000, rel_drop0=1e-2, freeze_jacobian=None,
                    finite_K=False, assemble_scaling=True, throw_on_failure=True,
                    precision=abi.PRECISION_FP64, cfl_v=0.98, c_fact=0.9, history=None) -> abi.StokesControlsC:
    c = abi.StokesControlsC()
    c.dt, c.pressure_factor, c.tolerance = float(dt), float(pressure_factor), float(tolerance)
    c.max_iterations, c.check_interval, c.iter_max = int(max_iterations), int(check_interval), int(iter_max)
    c.max_ph_iterations, c.rel_drop0 = int(max_ph_iterations), float(rel_drop0)
    c.freeze_jacobian = -1 if freeze_jacobian is None else int(bool(freeze_jacobian))
    c.finite_K, c.assemble_scaling = int(bool(finite_K)), int(bool(assemble_scaling))
    c.throw_on_failure, c.precision = int(bool(throw_on_failure)), int(precision)
    c.cfl_v, c.c_fact = float(cfl_v), float(c_fact)
    if history is not None:
        import ctypes
        c.history = history.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        c.history_capacity = history.shape[0]
    return c


def stats_dict(st: abi.StokesStatsC) -> dict:
    return {name: getattr(st, name) for name, _ in abi.StokesStatsC._fields_}
