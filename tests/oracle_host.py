"""Test-side binding of the CPU oracle (oracle/_build/liboracle.so).

The oracle is test infrastructure: the parity checker of libfemtools_b200. This
module builds host (numpy) problems with the same struct packing the product
uses, so a test can hand one problem to both implementations.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from conftest import fem

abi = fem._abi
problem = fem.problem

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "liboracle.so")

_P = C.POINTER
_vp = C.c_void_p
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            import subprocess
            subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
        L = C.CDLL(ORACLE_SO)
        sig = {
            "orc_last_error": (C.c_char_p, []),
            "orc_num_threads": (C.c_int, []),
            "orc_set_num_threads": (None, [C.c_int]),
            "orc_tables": (C.c_int, [C.c_int, _vp, _vp, _vp, _vp, _vp]),
            "orc_structured_mesh": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp]),
            "orc_geometry": (C.c_int, [C.c_int, C.c_int64, _vp, _vp, _vp, _vp]),
            "orc_strain_rate_stress": (C.c_int, [C.c_int, C.c_int64, _vp, _vp, _vp * 3, _vp * 6, _vp * 14]),
            "orc_lithostatic_residual": (C.c_int, [_P(abi.LithostaticProblemC), C.c_double, _vp, C.c_int32]),
            "orc_solve_lithostatic": (C.c_int, [_P(abi.LithostaticProblemC), _P(abi.LithostaticControlsC),
                                                _P(abi.ThermalStatsC)]),
            "orc_lithostatic_element_custom": (C.c_int, [C.c_int] * 3 + [_vp] * 9 + [C.c_double] + [_vp] * 4),
            "orc_cap_update": (C.c_int, [_P(abi.CapProblemC)]),
            "orc_cap_invariants": (C.c_int, [C.c_int64, _vp, _vp] + [C.c_double] * 4 + [_vp] * 3),
            "orc_cell_pressure_preconditioner": (C.c_int, [_P(abi.CellPressureProblemC)]),
            "orc_cell_pressure_residuals": (C.c_int, [_P(abi.CellPressureProblemC), C.c_int32]),
            "orc_solve_cell_pressure": (C.c_int, [_P(abi.CellPressureProblemC), _P(abi.CellPressureControlsC),
                                                  _P(abi.CellPressureStatsC)]),
            "orc_pressure_residual": (C.c_int, [_P(abi.StokesProblemC), C.c_double, C.c_int32]),
            "orc_momentum_residual": (C.c_int, [_P(abi.StokesProblemC), C.c_double, C.c_int32]),
            "orc_stokes_residuals": (C.c_int, [_P(abi.StokesProblemC), C.c_double, C.c_int32]),
            "orc_jacobian_diagnostics": (C.c_int, [_P(abi.StokesProblemC), C.c_double, C.c_int32]),
            "orc_pressure_scaling": (C.c_int, [_P(abi.StokesProblemC), C.c_double, C.c_double, C.c_int32]),
            "orc_store_stress": (C.c_int, [_P(abi.StokesProblemC), C.c_double]),
            "orc_solve_stokes": (C.c_int, [_P(abi.StokesProblemC), _P(abi.StokesControlsC), _P(abi.StokesStatsC)]),
            "orc_dr_iterations": (C.c_int, [_P(abi.StokesProblemC), C.c_double, C.c_int32, _vp, _vp, C.c_int64,
                                            C.c_int32, _vp]),
            "orc_jacobian_range": (C.c_int, [_P(abi.StokesProblemC), C.c_double, C.c_int32, C.c_int64, C.c_int64]),
            "orc_thermal_residual": (C.c_int, [_P(abi.ThermalProblemC), C.c_double, C.c_double, C.c_int32]),
            "orc_solve_thermal": (C.c_int, [_P(abi.ThermalProblemC), _P(abi.ThermalControlsC), _P(abi.ThermalStatsC)]),
            "orc_transfer_temperature": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int64]),
            "orc_shear_heating": (C.c_int, [_P(abi.StokesProblemC), C.c_double, _vp]),
            "orc_shear_dissipation": (C.c_int, [C.c_int, _vp, _vp, _vp, C.c_double, _vp]),
            "orc_thermal_element_custom": (C.c_int, [C.c_int] * 3 + [_vp] * 8 + [_P(abi.ThermalProblemC), C.c_double,
                                                                                C.c_double, _vp]),
            "orc_stokes_adjoint_residual": (C.c_int, [_P(abi.StokesProblemC), C.c_double, C.c_int32, C.c_int32,
                                                      _vp * 3, _vp, _vp * 3, _vp]),
            "orc_stokes_viscosity_sensitivity": (C.c_int, [_P(abi.StokesProblemC), C.c_double, C.c_int32, C.c_int32,
                                                           _vp * 3, _vp, _vp]),
            "orc_solve_coupled": (C.c_int, [_P(abi.ThermalProblemC), _P(abi.StokesProblemC), _P(abi.StokesControlsC),
                                            C.c_double, C.c_int32, _vp, _P(abi.StokesStatsC)]),
            "orc_element_custom": (C.c_int, [C.c_int] * 4 + [_vp] * 15 + [_P(abi.StokesMaterialC), C.c_double,
                                                                              C.c_int32, _vp, _vp, _vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def ptr(a):
    if a is None:
        return 0
    assert isinstance(a, np.ndarray) and a.flags["C_CONTIGUOUS"], "oracle arrays must be contiguous numpy"
    return a.ctypes.data


def check(rc):
    if rc != 0:
        raise abi.FemB200Error(rc, lib().orc_last_error().decode())


class HostStokes:
    """numpy mirror of a StokesDR state plus its packed problem for the oracle."""

    def __init__(self, mesh, material, plastic=None, phases_v=None, phases_v_layout=abi.PHASE_NODAL,
                 phases_P=None, phases_P_layout=abi.PHASE_NODAL, stress=True, scaling_eta=None):
        self.mesh = mesh
        self.material = material
        self.plastic = plastic
        dim, nn, nP = mesh.dim, mesh.nnodes, mesh.nnodesP
        z = lambda n: np.zeros(n)
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
        self.phases_v = phases_v if phases_v is not None else np.ones(nn, dtype=np.int32)
        self.phases_v_layout = phases_v_layout if phases_v is not None else abi.PHASE_NODAL
        self.phases_P = phases_P if phases_P is not None else np.ones(nP, dtype=np.int32)
        self.phases_P_layout = phases_P_layout if phases_P is not None else abi.PHASE_NODAL
        self.P_old = None
        self.P_old_layout = abi.FIELD_NODAL
        self.viscosity_ip = None
        self.body_force = None
        self.scaling_eta = scaling_eta
        self.mesh_arrays = {
            "dim": dim, "nels": mesh.nels, "nnodes": nn, "nnodesP": nP,
            "el2n": np.ascontiguousarray(mesh.el2n), "dofsP": np.ascontiguousarray(mesh.dofsP),
            "el2nP": np.ascontiguousarray(mesh.el2nP),
            "geo_v": np.ascontiguousarray(mesh.geo_v), "geo_P": np.ascontiguousarray(mesh.geo_P),
        }
        self.bcs = [None] * dim

    def set_bc(self, comps):
        """comps: one (dofs, vals) pair per velocity component."""
        self.bcs = [(np.ascontiguousarray(d, dtype=np.int32), np.ascontiguousarray(v, dtype=np.float64))
                    for d, v in comps]

    def state(self):
        return {
            "v": self.v, "rate": self.rate, "Rv": self.Rv, "Rv0": self.Rv0, "dRdv": self.dRdv, "PC": self.PC,
            "P": self.P, "P0": self.P0, "gammaP": self.gammaP, "T": self.T, "T0": self.T0, "Q": self.Q,
            "Pf": self.Pf, "RP": self.RP, "M_P": self.M_P, "Pnum": self.Pnum,
            "phases_v": self.phases_v, "phases_v_layout": self.phases_v_layout,
            "phases_P": self.phases_P, "phases_P_layout": self.phases_P_layout,
            "tau_old": self.tau_old, "tau": self.tau,
            "tau_old_layout": abi.FIELD_IP if self.tau_old is not None else abi.FIELD_NONE,
            "P_old": self.P_old, "P_old_layout": self.P_old_layout,
            "viscosity_ip": self.viscosity_ip, "body_force": self.body_force,
        }

    def struct(self):
        s = abi.StokesProblemC()
        mat = problem.material_struct(self.material, self.plastic, self.scaling_eta)
        problem.fill_stokes_problem(s, self.mesh_arrays, self.state(), mat, self.bcs, ptr)
        self._s = s
        return s

    # ---- oracle calls ----
    def pressure_scaling(self, gamma_fact, dt, finite_K=False):
        check(lib().orc_pressure_scaling(C.byref(self.struct()), gamma_fact, dt, int(finite_K)))

    def pressure_residual(self, dt, finite_K=False):
        check(lib().orc_pressure_residual(C.byref(self.struct()), dt, int(finite_K)))

    def momentum_residual(self, dt, with_pnum=False):
        check(lib().orc_momentum_residual(C.byref(self.struct()), dt, int(with_pnum)))

    def stokes_residuals(self, dt, finite_K=False):
        check(lib().orc_stokes_residuals(C.byref(self.struct()), dt, int(finite_K)))

    def jacobian_diagnostics(self, dt, finite_K=False):
        check(lib().orc_jacobian_diagnostics(C.byref(self.struct()), dt, int(finite_K)))

    def jacobian_range(self, dt, e0, e1, finite_K=False):
        """The Jacobian diagnostics of elements [e0, e1) into the full-size arrays."""
        check(lib().orc_jacobian_range(C.byref(self.struct()), dt, int(finite_K), int(e0), int(e1)))

    def dr_iterations(self, dt, alpha, beta, iterations, check_norms=False, finite_K=False):
        """`iterations` inner DR iterations of the solve's loop with fixed Chebyshev steps
        (the preconditioner already in PC), plus one check's norms and λmin when asked;
        returns the check's velocity error."""
        a = np.ascontiguousarray(alpha, dtype=np.float64)
        b = np.ascontiguousarray(beta, dtype=np.float64)
        ev = C.c_double(0.0)
        check(lib().orc_dr_iterations(C.byref(self.struct()), dt, int(finite_K), ptr(a), ptr(b), int(iterations),
                                      int(check_norms), C.byref(ev)))
        return ev.value

    def store_stress(self, dt):
        check(lib().orc_store_stress(C.byref(self.struct()), dt))

    def shear_heating(self, dt):
        phi = np.zeros(self.mesh.nq * self.mesh.nels)
        check(lib().orc_shear_heating(C.byref(self.struct()), dt, ptr(phi)))
        return phi

    def adjoint_residual(self, dt, lam_v, lam_P, finite_K=False, with_pnum=True):
        """(dR/du)ᵀλ at the current state (R the augmented residual: Pnum = γP·RP/M_P
        inline): returns (dv per component, dP)."""
        lam_v = [np.ascontiguousarray(x, dtype=np.float64) for x in lam_v]
        lam_P = np.ascontiguousarray(lam_P, dtype=np.float64)
        dv = [np.zeros(self.mesh.nnodes) for _ in range(3)]
        dP = np.zeros(self.mesh.nnodesP)
        lv = (_vp * 3)(*[ptr(x) for x in lam_v])
        ov = (_vp * 3)(*[ptr(x) for x in dv])
        check(lib().orc_stokes_adjoint_residual(C.byref(self.struct()), dt, int(finite_K), int(with_pnum), lv,
                                                 ptr(lam_P), ov, ptr(dP)))
        return dv, dP

    def viscosity_sensitivity(self, dt, lam_v, lam_P, finite_K=False, with_pnum=True):
        """λ·∂R/∂η at every integration point (nq × nels)."""
        lam_v = [np.ascontiguousarray(x, dtype=np.float64) for x in lam_v]
        lam_P = np.ascontiguousarray(lam_P, dtype=np.float64)
        out = np.zeros(self.mesh.nq * self.mesh.nels)
        lv = (_vp * 3)(*[ptr(x) for x in lam_v])
        check(lib().orc_stokes_viscosity_sensitivity(C.byref(self.struct()), dt, int(finite_K), int(with_pnum), lv,
                                                      ptr(lam_P), ptr(out)))
        return out

    def solve(self, history_capacity=0, **kw):
        hist = np.zeros((history_capacity, 4 + self.mesh.dim)) if history_capacity else None
        c = problem.controls_struct(history=hist, **kw)
        st = abi.StokesStatsC()
        rc = lib().orc_solve_stokes(C.byref(self.struct()), C.byref(c), C.byref(st))
        check(rc)
        out = problem.stats_dict(st)
        if hist is not None:
            out["history"] = hist[: st.history_len]
        return out


def element_custom(dim, N, dNdx, dOmega, NP, v, P, material, dt=1.0, P0=None, T=None, T0=None, Q=None,
                   Pnum=None, phv=None, php=None, tau_old=None, P0_ip=None, plastic=None, finite_K=False):
    """One synthetic element through the oracle (the reference's element unit-test setup)."""
    N = np.ascontiguousarray(N, dtype=np.float64)
    nq, nv = N.shape
    NP = np.ascontiguousarray(NP, dtype=np.float64)
    npd = NP.shape[1]
    arr = lambda x: None if x is None else np.ascontiguousarray(x, dtype=np.float64)
    iarr = lambda x: None if x is None else np.ascontiguousarray(x, dtype=np.int32)
    m = problem.material_struct(material, plastic)
    R = np.zeros(dim * nv)
    RP = np.zeros(npd)
    ntau = 6 if dim == 3 else 3
    tau = np.zeros(nq * ntau)
    args = [arr(dNdx), arr(dOmega), NP, arr(v), arr(P), arr(P0), arr(T), arr(T0), arr(Q), arr(Pnum),
            iarr(phv), iarr(php), arr(tau_old), arr(P0_ip)]
    keep = [N] + args
    rc = lib().orc_element_custom(dim, nv, npd, nq, ptr(N), *[ptr(a) for a in args], C.byref(m), dt,
                                  int(finite_K), ptr(R), ptr(RP), ptr(tau))
    del keep
    check(rc)
    return R.reshape(dim, nv), RP, tau.reshape(nq, ntau)


class HostThermal:
    """numpy mirror of a ThermalDiffusionDR state (heat_diffusion_types.jl:90-132)."""

    def __init__(self, mesh, k=(1.0,), Cp=(1.0,), rho0=(1.0,), alpha=(0.0,), K=(np.inf,), phases=None,
                 cfl=0.98, c_fact=0.9, eps=1e-6):
        self.mesh = mesh
        nn = mesh.nnodes
        for name in ("T", "T0", "rate", "R", "R0", "dRdT", "PC", "P", "source"):
            setattr(self, name, np.zeros(nn))
        self.phases = np.ones(nn, dtype=np.int32) if phases is None else phases
        self.mat = dict(k=k, Cp=Cp, rho0=rho0, alpha=alpha, K=K)
        self.cfl, self.c_fact, self.eps = cfl, c_fact, eps
        self.source_ip = None
        self.bc = (np.zeros(0, dtype=np.int32), np.zeros(0))
        self.el2n = np.ascontiguousarray(mesh.el2n)
        self.geo = np.ascontiguousarray(mesh.geo_v)

    def set_bc(self, dofs, vals):
        self.bc = (np.ascontiguousarray(dofs, dtype=np.int32), np.ascontiguousarray(vals, dtype=np.float64))

    def struct(self):
        t = abi.ThermalProblemC()
        t.dim, t.dtype, t.geo_dtype = self.mesh.dim, abi.F64, abi.F64
        t.nv, t.nq = (27, 27) if self.mesh.dim == 3 else (9, 9)
        t.nels, t.nnodes = self.mesh.nels, self.mesh.nnodes
        t.el2n, t.geo = ptr(self.el2n), ptr(self.geo)
        for name in ("T", "T0", "rate", "R", "R0", "dRdT", "PC", "P", "source"):
            setattr(t, name, ptr(getattr(self, name)))
        t.source_ip = ptr(self.source_ip)
        t.phases, t.phases_layout = ptr(self.phases), abi.PHASE_NODAL
        t.bc_dofs, t.bc_vals, t.bc_n = ptr(self.bc[0]), ptr(self.bc[1]), len(self.bc[0])
        n = len(self.mat["k"])
        t.nphases = n
        for name, fill in (("k", 1.0), ("Cp", 1.0), ("rho0", 1.0), ("alpha", 0.0), ("K", np.inf)):
            arr = getattr(t, name)
            vals = self.mat[name]
            for i in range(abi.MAX_PHASES):
                arr[i] = vals[i] if i < n else fill
        t.cfl, t.c_fact, t.eps = self.cfl, self.c_fact, self.eps
        self._t = t
        return t

    def residual(self, dt, Tref, jac=False):
        check(lib().orc_thermal_residual(C.byref(self.struct()), dt, Tref, int(jac)))

    def solve(self, dt, Tref=273.0, tolerance=None, max_iterations=10_000, check_interval=100, throw_on_failure=True):
        c = abi.ThermalControlsC()
        c.dt, c.Tref = dt, Tref
        c.tolerance = self.eps if tolerance is None else tolerance
        c.max_iterations, c.check_interval, c.throw_on_failure = max_iterations, check_interval, int(throw_on_failure)
        st = abi.ThermalStatsC()
        check(lib().orc_solve_thermal(C.byref(self.struct()), C.byref(c), C.byref(st)))
        return {"converged": bool(st.converged), "iterations": st.iterations, "residual": st.residual}


def solve_coupled(thermal: HostThermal, stokes: HostStokes, Tref=273.0, shear_heating=False, history_capacity=0, **kw):
    phi = np.zeros(stokes.mesh.nq * stokes.mesh.nels) if shear_heating else None
    c = problem.controls_struct(**kw)
    st = abi.StokesStatsC()
    t = thermal.struct()
    rc = lib().orc_solve_coupled(C.byref(t), C.byref(stokes.struct()), C.byref(c), Tref, int(shear_heating),
                                 ptr(phi), C.byref(st))
    check(rc)
    return problem.stats_dict(st), phi


def strain_rate_stress(dim, el2n, geo_v, v, tau):
    """Oracle element-averaged diagnostics: list of 14 (3-D) / 10 (2-D) arrays of nels."""
    el2n = np.ascontiguousarray(el2n, dtype=np.int32)
    geo_v = np.ascontiguousarray(geo_v, dtype=np.float64)
    nels = el2n.shape[0]
    vs = [np.ascontiguousarray(x, dtype=np.float64) for x in v]
    ts = [np.ascontiguousarray(x, dtype=np.float64) for x in tau]
    nf = 14 if dim == 3 else 10
    out = [np.zeros(nels) for _ in range(nf)]
    vp = (C.c_void_p * 3)(*([ptr(x) for x in vs] + [0] * (3 - len(vs))))
    tp = (C.c_void_p * 6)(*([ptr(x) for x in ts] + [0] * (6 - len(ts))))
    op = (C.c_void_p * 14)(*([ptr(x) for x in out] + [0] * (14 - nf)))
    check(lib().orc_strain_rate_stress(dim, nels, ptr(el2n), ptr(geo_v), vp, tp, op))
    return out


class HostCellPressure:
    """Oracle state of the cell-pressure Hex27 Stokes problem (host numpy arrays)."""

    def __init__(self, mesh, eta, rho, g, phases, v=None, P=None):
        self.mesh = mesh
        nn, ne = mesh.nnodes, mesh.nels
        self.el2n = np.ascontiguousarray(mesh.el2n, dtype=np.int32)
        self.geo_v = np.ascontiguousarray(mesh.geo_v, dtype=np.float64)
        self.phases = np.ascontiguousarray(phases, dtype=np.int32)
        self.eta, self.rho, self.g = tuple(eta), tuple(rho), tuple(g)
        self.v = [np.ascontiguousarray(x, dtype=np.float64).copy() for x in v] if v is not None else \
            [np.zeros(nn) for _ in range(3)]
        self.P = np.ascontiguousarray(P, dtype=np.float64).copy() if P is not None else np.zeros(4 * ne)
        self.Rv = [np.zeros(nn) for _ in range(3)]
        self.RP = np.zeros(4 * ne)
        self.diagonal = [np.zeros(nn) for _ in range(3)]
        self.pressure_mass = np.zeros(4 * ne)
        self._keep = []

    def struct(self, bc=None, load=None):
        p = abi.CellPressureProblemC()
        p.nels, p.nnodes = self.mesh.nels, self.mesh.nnodes
        p.el2n, p.geo_v, p.phases = ptr(self.el2n), ptr(self.geo_v), ptr(self.phases)
        p.nphases = len(self.eta)
        for i in range(len(self.eta)):
            p.eta[i], p.rho[i] = self.eta[i], self.rho[i]
        keep = []
        for c in range(3):
            p.g[c] = self.g[c]
            p.v[c], p.Rv[c], p.diagonal[c] = ptr(self.v[c]), ptr(self.Rv[c]), ptr(self.diagonal[c])
            if load is not None:
                ld = np.ascontiguousarray(load[c], dtype=np.float64)
                keep.append(ld)
                p.load[c] = ptr(ld)
            if bc is not None and bc[c] is not None:
                d = np.ascontiguousarray(bc[c][0], dtype=np.int32)
                vv = np.ascontiguousarray(np.broadcast_to(np.asarray(bc[c][1], dtype=np.float64), d.shape))
                keep += [d, vv]
                p.bc_dofs[c], p.bc_vals[c], p.bc_n[c] = ptr(d), ptr(vv), len(d)
        p.P, p.RP, p.pressure_mass = ptr(self.P), ptr(self.RP), ptr(self.pressure_mass)
        self._keep = keep
        return p

    def preconditioner(self):
        check(lib().orc_cell_pressure_preconditioner(C.byref(self.struct())))

    def residuals(self, which=3):
        check(lib().orc_cell_pressure_residuals(C.byref(self.struct()), which))

    def solve(self, bc, tolerance=1e-5, max_iterations=3000, check_interval=100, velocity_step=0.6,
              pressure_step=0.2, throw_on_failure=True, load=None):
        p = self.struct(bc, load)
        c = abi.CellPressureControlsC()
        c.tolerance, c.max_iterations, c.check_interval = tolerance, max_iterations, check_interval
        c.velocity_step, c.pressure_step, c.throw_on_failure = velocity_step, pressure_step, int(throw_on_failure)
        st = abi.CellPressureStatsC()
        check(lib().orc_solve_cell_pressure(C.byref(p), C.byref(c), C.byref(st)))
        return st


class HostLithostatic:
    """Oracle state of the lithostatic-pressure problem (host numpy arrays)."""

    def __init__(self, mesh, rho0=(1.0,), alpha=(0.0,), K=(float("inf"),), phases=None, T=None, P=None,
                 cfl=0.98, c_fact=0.9, eps=1e-6):
        nn = mesh.nnodes
        self.mesh = mesh
        self.el2n = np.ascontiguousarray(mesh.el2n, dtype=np.int32)
        self.geo = np.ascontiguousarray(mesh.geo_v, dtype=np.float64)
        self.phases = np.ascontiguousarray(np.ones(nn) if phases is None else phases, dtype=np.int32)
        self.T = np.ascontiguousarray(np.zeros(nn) if T is None else T, dtype=np.float64)
        self.P = np.ascontiguousarray(np.zeros(nn) if P is None else P, dtype=np.float64).copy()
        for name in ("rate", "R", "R0", "dRdP", "PC"):
            setattr(self, name, np.zeros(nn))
        self.rho0, self.alpha, self.K = rho0, alpha, K
        self.cfl, self.c_fact, self.eps = cfl, c_fact, eps
        self._keep = []

    def struct(self, bc=None):
        p = abi.LithostaticProblemC()
        d = self.mesh.dim
        p.dim, p.nv, p.nq = (3, 27, 27) if d == 3 else (2, 9, 9)
        p.nels, p.nnodes = self.mesh.nels, self.mesh.nnodes
        p.el2n, p.geo = ptr(self.el2n), ptr(self.geo)
        for name in ("P", "rate", "R", "R0", "dRdP", "PC", "T"):
            setattr(p, name, ptr(getattr(self, name)))
        p.phases, p.phases_layout, p.nphases = ptr(self.phases), abi.PHASE_NODAL, len(self.rho0)
        for i in range(abi.MAX_PHASES):
            p.rho0[i] = self.rho0[i] if i < len(self.rho0) else 1.0
            p.alpha[i] = self.alpha[i] if i < len(self.alpha) else 0.0
            p.K[i] = self.K[i] if i < len(self.K) else float("inf")
        self._keep = []
        if bc is not None:
            dd = np.ascontiguousarray(bc[0], dtype=np.int32)
            vv = np.ascontiguousarray(bc[1], dtype=np.float64)
            self._keep = [dd, vv]
            p.bc_dofs, p.bc_vals, p.bc_n = ptr(dd), ptr(vv), len(dd)
        p.cfl, p.c_fact, p.eps = self.cfl, self.c_fact, self.eps
        return p

    def residual(self, Tref, g, jac=False):
        gg = np.zeros(3)
        gg[:len(g)] = g
        check(lib().orc_lithostatic_residual(C.byref(self.struct()), Tref, ptr(gg), int(jac)))

    def solve(self, bc, Tref, g, tolerance=None, max_iterations=10_000, check_interval=100, throw_on_failure=True):
        p = self.struct(bc)
        c = abi.LithostaticControlsC()
        c.Tref = Tref
        for k, x in enumerate(g):
            c.g[k] = x
        c.tolerance = self.eps if tolerance is None else tolerance
        c.max_iterations, c.check_interval, c.throw_on_failure = max_iterations, check_interval, int(throw_on_failure)
        st = abi.ThermalStatsC()
        check(lib().orc_solve_lithostatic(C.byref(p), C.byref(c), C.byref(st)))
        return st


def lithostatic_element(N, dNdx, dO, P, T, phases, rho0, alpha, K, Tref, g):
    """Oracle element residual, Jacobian row sums and |diagonal| for given N (nq × nv),
    physical gradients dNdx (nq × nv × dim) and weights dO (nq)."""
    N = np.ascontiguousarray(N, dtype=np.float64)
    dNdx = np.ascontiguousarray(dNdx, dtype=np.float64)
    nq, nv, dim = dNdx.shape
    arr = lambda x, t=np.float64: np.ascontiguousarray(x, dtype=t)
    dO, P, T = arr(dO), arr(P), arr(T)
    ph = arr(phases, np.int32)
    pad = lambda x, fill: arr(list(x) + [fill] * (abi.MAX_PHASES - len(x)))
    r0, al, KK = pad(rho0, 1.0), pad(alpha, 0.0), pad(K, float("inf"))
    gg = arr(list(g) + [0.0] * (3 - len(g)))
    R, rows, diag = np.zeros(nv), np.zeros(nv), np.zeros(nv)
    check(lib().orc_lithostatic_element_custom(dim, nv, nq, ptr(N), ptr(dNdx), ptr(dO), ptr(P), ptr(T), ptr(ph),
                                               ptr(r0), ptr(al), ptr(KK), Tref, ptr(gg), ptr(R), ptr(rows),
                                               ptr(diag)))
    return R, rows, diag


def cap_update(ncomp, trial, P_trial, eta_ve, K_dt, k, kq, c, pT, eta_reg, maxiter=40):
    """orc_cap_update on host arrays broadcast to one length: cap_return_map (ncomp 0,
    trial = s_trial) or cap_local_update (ncomp 3 or 6, trial = n × ncomp stresses).
    Returns a dict of numpy arrays named like femb200_cap_problem's outputs."""
    if ncomp:
        trial = np.ascontiguousarray(trial, dtype=np.float64).reshape(-1, ncomp)
        n = trial.shape[0]
        arrs = [np.ascontiguousarray(np.broadcast_to(np.asarray(a, dtype=np.float64), (n,)))
                for a in (P_trial, eta_ve, K_dt, k, kq, c, pT, eta_reg)]
    else:
        arrs = np.broadcast_arrays(*[np.asarray(a, dtype=np.float64)
                                     for a in (trial, P_trial, eta_ve, K_dt, k, kq, c, pT, eta_reg)])
        arrs = [np.ascontiguousarray(a).reshape(-1) for a in arrs]
        trial, arrs = arrs[0], arrs[1:]
        n = trial.shape[0]
    out = {name: np.empty(n) for name in ("tau_II", "P", "lambda", "A_tau", "A_p", "gamma_dot", "theta_dot")}
    out["converged"] = np.empty(n, dtype=np.int32)
    if ncomp:
        out["tau"] = np.empty((n, ncomp))
    pr = abi.CapProblemC()
    pr.n, pr.ncomp, pr.maxiter = n, ncomp, maxiter
    if ncomp:
        pr.tau_trial = ptr(trial)
    else:
        pr.s_trial = ptr(trial)
    pr.P_trial, pr.eta_ve, pr.K_dt, pr.k, pr.kq, pr.c, pr.pT, pr.eta_reg = [ptr(a) for a in arrs]
    pr.tau = ptr(out.get("tau"))
    pr.tau_II, pr.P, pr.lambda_ = ptr(out["tau_II"]), ptr(out["P"]), ptr(out["lambda"])
    pr.A_tau, pr.A_p = ptr(out["A_tau"]), ptr(out["A_p"])
    pr.gamma_dot, pr.theta_dot, pr.converged = ptr(out["gamma_dot"]), ptr(out["theta_dot"]), ptr(out["converged"])
    assert lib().orc_cap_update(C.byref(pr)) == 0
    out["converged"] = out["converged"].astype(bool)
    out["_keep"] = (trial, arrs)
    return out


def cap_invariants(s, p, k, kq, c, pT):
    """orc_cap_invariants at the points (s, p) of one material: (F, Aτ, Ap) arrays."""
    s, p = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in np.broadcast_arrays(s, p)]
    F, At, Ap = np.empty(len(s)), np.empty(len(s)), np.empty(len(s))
    assert lib().orc_cap_invariants(len(s), ptr(s), ptr(p), k, kq, c, pT, ptr(F), ptr(At), ptr(Ap)) == 0
    return F, At, Ap


def shear_dissipation(dim, tau, tau_old, grad, inv2Gdt):
    """orc_shear_dissipation: stress power less elastic power at one point."""
    t, o, g = (np.ascontiguousarray(x, dtype=np.float64).ravel() for x in (tau, tau_old, grad))
    out = np.zeros(1)
    check(lib().orc_shear_dissipation(dim, ptr(t), ptr(o), ptr(g), inv2Gdt, ptr(out)))
    return float(out[0])


def thermal_element_custom(dim, N, dNdx, dOmega, T, T0, src, P, phases, k, Cp, rho0, alpha, K, dt=1.0, Tref=0.0):
    """One synthetic thermal element through the oracle (integrate_residual's unit-test setup)."""
    N = np.ascontiguousarray(N, dtype=np.float64)
    nq, nv = N.shape
    arr = lambda x: np.ascontiguousarray(x, dtype=np.float64)
    tp = abi.ThermalProblemC()
    for name, vals in (("k", k), ("Cp", Cp), ("rho0", rho0), ("alpha", alpha), ("K", K)):
        field = getattr(tp, name)
        for i, v in enumerate(vals):
            field[i] = v
    tp.nphases = len(k)
    args = [arr(dNdx), arr(dOmega), arr(T), arr(T0), arr(src), arr(P)]
    ph = np.ascontiguousarray(phases, dtype=np.int32)
    R = np.zeros(nv)
    check(lib().orc_thermal_element_custom(dim, nv, nq, ptr(N), *[ptr(a) for a in args], ptr(ph), C.byref(tp),
                                           dt, Tref, ptr(R)))
    return R
