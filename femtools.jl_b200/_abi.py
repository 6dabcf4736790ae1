"""ctypes mirror of include/femtools_b200.h and the loader of libfemtools_b200.

The structs below must match the C header field for field; test_abi checks the
sizes against the compiled library. Loading the CUDA library never falls back
to anything: a missing or unloadable library raises at import of the solver.
"""
from __future__ import annotations

import ctypes as C
import os

MAX_PHASES = 16

# status codes
OK, EINVAL, ECUDA, ENOMEM, ENOTCONV, ENAN, EKABOOM, ELAMBDA, EUNSUPPORTED, ENONFINITE = range(10)
F64, F32 = 0, 1
PHASE_NODAL, PHASE_CELL, PHASE_ELEMENT_NODE = 0, 1, 2
FIELD_NONE, FIELD_IP, FIELD_NODAL = 0, 1, 2
PRECISION_FP64, PRECISION_MIXED = 0, 1

_dvec = C.c_double * MAX_PHASES


class StokesMaterialC(C.Structure):
    _fields_ = [
        ("nphases", C.c_int32),
        ("eta", _dvec), ("eta_b", _dvec), ("G", _dvec), ("alpha", _dvec),
        ("rho0", _dvec), ("K", _dvec),
        ("g", C.c_double * 3), ("Tref", C.c_double),
        ("plastic", C.c_int32),
        ("cos_phi", _dvec), ("sin_phi", _dvec), ("sin_psi", _dvec),
        ("C", _dvec), ("eta_reg", _dvec), ("Kb", _dvec),
        ("use_scaling_eta", C.c_int32),
        ("scaling_eta", _dvec),
    ]


_vp = C.c_void_p
_ip = C.POINTER(C.c_int32)


class StokesProblemC(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("nv", C.c_int32), ("np", C.c_int32), ("nq", C.c_int32),
        ("dtype", C.c_int32), ("geo_dtype", C.c_int32),
        ("nels", C.c_int64), ("nnodes", C.c_int64), ("nnodesP", C.c_int64),
        ("el2n", _vp), ("dofsP", _vp), ("el2nP", _vp), ("geo_v", _vp), ("geo_P", _vp),
        ("v", _vp * 3), ("rate", _vp * 3), ("Rv", _vp * 3), ("Rv0", _vp * 3),
        ("dRdv", _vp * 3), ("PC", _vp * 3),
        ("P", _vp), ("P0", _vp), ("gammaP", _vp), ("T", _vp), ("T0", _vp), ("Q", _vp),
        ("Pf", _vp), ("RP", _vp), ("M_P", _vp), ("Pnum", _vp),
        ("phases_v", _vp), ("phases_v_layout", C.c_int32),
        ("phases_P", _vp), ("phases_P_layout", C.c_int32),
        ("tau_old", _vp * 6), ("tau_old_layout", C.c_int32),
        ("tau", _vp * 6),
        ("P_old", _vp), ("P_old_layout", C.c_int32),
        ("viscosity_ip", _vp),
        ("body_force", _vp * 3),
        ("bc_dofs", _vp * 3), ("bc_vals", _vp * 3), ("bc_n", C.c_int64 * 3),
        ("mat", StokesMaterialC),
    ]


class StokesControlsC(C.Structure):
    _fields_ = [
        ("dt", C.c_double), ("pressure_factor", C.c_double), ("tolerance", C.c_double),
        ("max_iterations", C.c_int64), ("check_interval", C.c_int64), ("iter_max", C.c_int64),
        ("max_ph_iterations", C.c_int64), ("rel_drop0", C.c_double),
        ("freeze_jacobian", C.c_int32), ("finite_K", C.c_int32),
        ("assemble_scaling", C.c_int32), ("throw_on_failure", C.c_int32),
        ("precision", C.c_int32),
        ("cfl_v", C.c_double), ("c_fact", C.c_double),
        ("history", C.POINTER(C.c_double)), ("history_capacity", C.c_int64),
    ]


class StokesStatsC(C.Structure):
    _fields_ = [
        ("itPH", C.c_int64), ("iter", C.c_int64),
        ("err", C.c_double), ("err_abs", C.c_double), ("err_rel", C.c_double),
        ("err_v", C.c_double), ("err_P", C.c_double),
        ("converged", C.c_int32), ("reached_total_iter", C.c_int32),
        ("lambda_max", C.c_double), ("lambda_max_gershgorin", C.c_double),
        ("jacobian_assemblies", C.c_int64), ("history_len", C.c_int64),
        ("err_T", C.c_double), ("thermal_iterations", C.c_int64),
        ("defect_corrections", C.c_int64),
    ]


class ThermalProblemC(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("nv", C.c_int32), ("nq", C.c_int32), ("dtype", C.c_int32),
        ("geo_dtype", C.c_int32),
        ("nels", C.c_int64), ("nnodes", C.c_int64),
        ("el2n", _vp), ("geo", _vp),
        ("T", _vp), ("T0", _vp), ("rate", _vp), ("R", _vp), ("R0", _vp), ("dRdT", _vp), ("PC", _vp),
        ("P", _vp), ("source", _vp), ("source_ip", _vp),
        ("phases", _vp), ("phases_layout", C.c_int32),
        ("bc_dofs", _vp), ("bc_vals", _vp), ("bc_n", C.c_int64),
        ("nphases", C.c_int32),
        ("k", _dvec), ("Cp", _dvec), ("rho0", _dvec), ("alpha", _dvec), ("K", _dvec),
        ("cfl", C.c_double), ("c_fact", C.c_double), ("eps", C.c_double),
    ]


class ThermalControlsC(C.Structure):
    _fields_ = [
        ("dt", C.c_double), ("Tref", C.c_double), ("tolerance", C.c_double),
        ("max_iterations", C.c_int64), ("check_interval", C.c_int64),
        ("throw_on_failure", C.c_int32),
    ]


class ThermalStatsC(C.Structure):
    _fields_ = [("converged", C.c_int32), ("iterations", C.c_int64), ("residual", C.c_double)]


class LithostaticProblemC(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("nv", C.c_int32), ("nq", C.c_int32),
        ("nels", C.c_int64), ("nnodes", C.c_int64),
        ("el2n", _vp), ("geo", _vp),
        ("P", _vp), ("rate", _vp), ("R", _vp), ("R0", _vp), ("dRdP", _vp), ("PC", _vp),
        ("T", _vp), ("phases", _vp), ("phases_layout", C.c_int32),
        ("nphases", C.c_int32), ("rho0", _dvec), ("alpha", _dvec), ("K", _dvec),
        ("bc_dofs", _vp), ("bc_vals", _vp), ("bc_n", C.c_int64),
        ("cfl", C.c_double), ("c_fact", C.c_double), ("eps", C.c_double),
    ]


class LithostaticControlsC(C.Structure):
    _fields_ = [
        ("Tref", C.c_double), ("g", C.c_double * 3), ("tolerance", C.c_double),
        ("max_iterations", C.c_int64), ("check_interval", C.c_int64), ("throw_on_failure", C.c_int32),
    ]


class CellPressureProblemC(C.Structure):
    _fields_ = [
        ("nels", C.c_int64), ("nnodes", C.c_int64),
        ("el2n", _vp), ("geo_v", _vp), ("phases", _vp), ("nphases", C.c_int32),
        ("eta", _dvec), ("rho", _dvec), ("g", C.c_double * 3),
        ("v", _vp * 3), ("P", _vp), ("Rv", _vp * 3), ("RP", _vp), ("diagonal", _vp * 3), ("pressure_mass", _vp),
        ("load", _vp * 3), ("bc_dofs", _vp * 3), ("bc_vals", _vp * 3), ("bc_n", C.c_int64 * 3),
    ]


class CellPressureControlsC(C.Structure):
    _fields_ = [
        ("tolerance", C.c_double), ("max_iterations", C.c_int64), ("check_interval", C.c_int64),
        ("velocity_step", C.c_double), ("pressure_step", C.c_double), ("throw_on_failure", C.c_int32),
        ("history", C.POINTER(C.c_double)), ("history_capacity", C.c_int64),
    ]


class CellPressureStatsC(C.Structure):
    _fields_ = [
        ("converged", C.c_int32), ("reached_total_iter", C.c_int32), ("iterations", C.c_int64),
        ("residual", C.c_double), ("err_v", C.c_double), ("err_P", C.c_double), ("history_len", C.c_int64),
    ]


class CapProblemC(C.Structure):
    _fields_ = [
        ("n", C.c_int64), ("ncomp", C.c_int32), ("maxiter", C.c_int32),
        ("tau_trial", _vp), ("s_trial", _vp), ("P_trial", _vp), ("eta_ve", _vp), ("K_dt", _vp),
        ("k", _vp), ("kq", _vp), ("c", _vp), ("pT", _vp), ("eta_reg", _vp),
        ("tau", _vp), ("tau_II", _vp), ("P", _vp), ("lambda_", _vp), ("A_tau", _vp), ("A_p", _vp),
        ("gamma_dot", _vp), ("theta_dot", _vp), ("converged", _vp),
    ]


PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libfemtools_b200.so")

# Every exported entry point of include/femtools_b200.h, with its ctypes signature.
_P = C.POINTER
SIGNATURES = {
    "femb200_create": (C.c_int, [_P(_vp)]),
    "femb200_destroy": (C.c_int, [_vp]),
    "femb200_set_stream": (C.c_int, [_vp, _vp]),
    "femb200_set_ordered_scatter": (C.c_int, [_vp, C.c_int32]),
    "femb200_last_error": (C.c_char_p, [_vp]),
    "femb200_version": (C.c_char_p, []),
    "femb200_pressure_residual": (C.c_int, [_vp, _P(StokesProblemC), C.c_double, C.c_int32]),
    "femb200_momentum_residual": (C.c_int, [_vp, _P(StokesProblemC), C.c_double, C.c_int32]),
    "femb200_stokes_residuals": (C.c_int, [_vp, _P(StokesProblemC), C.c_double, C.c_int32]),
    "femb200_velocity_update": (C.c_int, [_vp, _P(StokesProblemC), _P(C.c_double), _P(C.c_double)]),
    "femb200_apply_dirichlet": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int64, C.c_int32]),
    "femb200_jacobian_diagnostics": (C.c_int, [_vp, _P(StokesProblemC), C.c_double, C.c_int32]),
    "femb200_pressure_scaling": (C.c_int, [_vp, _P(StokesProblemC), C.c_double, C.c_double, C.c_int32]),
    "femb200_store_stress": (C.c_int, [_vp, _P(StokesProblemC), C.c_double]),
    "femb200_solve_stokes": (C.c_int, [_vp, _P(StokesProblemC), _P(StokesControlsC), _P(StokesStatsC)]),
    "femb200_stokes_adjoint_residual": (C.c_int, [_vp, _P(StokesProblemC), C.c_double, C.c_int32, C.c_int32,
                                                  _vp * 3, _vp, _vp * 3, _vp]),
    "femb200_stokes_viscosity_sensitivity": (C.c_int, [_vp, _P(StokesProblemC), C.c_double, C.c_int32, C.c_int32,
                                                       _vp * 3, _vp, _vp]),
    "femb200_solve_stokes_adjoint": (C.c_int, [_vp, _P(StokesProblemC), _P(StokesControlsC), _vp * 3, _vp * 3, _vp,
                                               _P(StokesStatsC)]),
    "femb200_conv3x3_forward": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                          C.c_int32, C.c_int32]),
    "femb200_conv3x3_weight_grad": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                              C.c_int32]),
    "femb200_conv3x3_flip_weights": (C.c_int, [_vp, _vp, _vp, C.c_int32, C.c_int32]),
    "femb200_mse_loss_grad": (C.c_int, [_vp, _vp, _vp, C.c_int32, C.c_int32, C.c_double, _vp, C.c_int64,
                                        _P(C.c_double)]),
    "femb200_adam_step": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, C.c_int64, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_int64]),
    "femb200_f32_to_bf16": (C.c_int, [_vp, _vp, _vp, C.c_int64]),
    "femb200_q9_grid_fields": (C.c_int, [_vp, _P(StokesProblemC), _vp, _vp, _vp, C.c_int32, C.c_int32, C.c_double,
                                         C.c_double, _vp]),
    "femb200_net_input": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int64]),
    "femb200_net_target": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, C.c_int64]),
    "femb200_apply_warm_start": (C.c_int, [_vp, _P(StokesProblemC), _vp * 2, _vp * 2, _vp, _vp, _vp, C.c_int32,
                                           _P(C.c_float)]),
    "femb200_extrapolate_state": (C.c_int, [_vp, _P(StokesProblemC), _vp * 3, _vp * 3, _vp, _vp]),
    "femb200_precompute_geometry": (C.c_int, [_vp, C.c_int32, C.c_int64, C.c_int64, _vp, _vp, _vp, _vp, C.c_int32]),
    "femb200_strain_rate_stress": (C.c_int, [_vp, _P(StokesProblemC), _vp * 6, _vp * 14]),
    "femb200_lithostatic_residual": (C.c_int, [_vp, _P(LithostaticProblemC), C.c_double, C.c_double * 3,
                                               C.c_int32]),
    "femb200_solve_lithostatic": (C.c_int, [_vp, _P(LithostaticProblemC), _P(LithostaticControlsC),
                                            _P(ThermalStatsC)]),
    "femb200_cell_pressure_preconditioner": (C.c_int, [_vp, _P(CellPressureProblemC)]),
    "femb200_cell_pressure_residuals": (C.c_int, [_vp, _P(CellPressureProblemC), C.c_int32]),
    "femb200_solve_cell_pressure": (C.c_int, [_vp, _P(CellPressureProblemC), _P(CellPressureControlsC),
                                              _P(CellPressureStatsC)]),
    "femb200_cap_update": (C.c_int, [_vp, _P(CapProblemC)]),
    "femb200_thermal_residual": (C.c_int, [_vp, _P(ThermalProblemC), C.c_double, C.c_double, C.c_int32]),
    "femb200_solve_thermal": (C.c_int, [_vp, _P(ThermalProblemC), _P(ThermalControlsC), _P(ThermalStatsC)]),
    "femb200_transfer_temperature": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int64, C.c_int32]),
    "femb200_shear_heating": (C.c_int, [_vp, _P(StokesProblemC), C.c_double, _vp]),
    "femb200_solve_coupled": (C.c_int, [_vp, _P(ThermalProblemC), _P(StokesProblemC),
                                        _P(StokesControlsC), C.c_double, C.c_int32, _vp,
                                        _P(StokesStatsC)]),
    "femb200_profile": (C.c_int, [_vp, C.c_int32]),
    "femb200_profile_read": (C.c_int, [_vp, _P(C.c_double), _P(C.c_int64)]),
    "femb200_profile_counters": (C.c_int, [_vp, _P(C.c_int64), C.c_int32]),
    "femb200_color_mesh": (C.c_int, [_vp, C.c_int32, C.c_int64, C.c_int64, _vp, _P(C.c_int32)]),
    "femb200_color_groups": (C.c_int, [_vp, C.c_int64, C.c_int32, _vp, _vp]),
    "femb200_thermal_residual_colored": (C.c_int, [_vp, _P(ThermalProblemC), C.c_double, C.c_double, C.c_int32,
                                                   _vp, _vp, C.c_int32]),
    "femb200_solve_thermal_noalloc": (C.c_int, [_vp, _P(ThermalProblemC), _P(ThermalControlsC), _P(ThermalStatsC)]),
}
NOALLOC_MAX_NODES = 8388608   # FEMB200_NOALLOC_MAX_NODES
PROF_RESIDUAL, PROF_JACOBIAN, PROF_NODE, PROF_ALL, PROF_OUTER, PROF_COUNT = range(6)
COUNTER_STRESS_READS, COUNTER_SHARED_JACOBIANS, COUNTER_COUNT = 0, 1, 4

_lib = None


def load_library(path: str = LIB_PATH):
    """Load libfemtools_b200 and attach signatures. Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"libfemtools_b200 not built at {path}; run __graft_entry__.build() "
            "(the CUDA extension is required: there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class FemB200Error(RuntimeError):
    """Raised when a libfemtools_b200 call returns a non-OK status."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code
