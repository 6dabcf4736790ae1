"""Drucker–Prager tensile cap (DruckerPragerCap, src/stokes/types/stokes_types.jl:426-545;
src/stokes/assemblers/rheology.jl:510-724), after Popov, Berlie & Kaus (2025), "A dilatant
visco-elasto-viscoplasticity model with globally continuous tensile cap", GMD 18, 7035-7058.

`DruckerPragerCap` holds the per-phase parameters with the reference's checks. The batched
local return — `cap_return_map` on (s_trial, p_trial) and `cap_local_update` on a plane-strain
or 3-D trial stress — runs on the device through femb200_cap_update, one thread per point.
`cap_geometry`, `cap_yield_function`, `cap_invariants` and `softened_cohesion` are the
scalar formulas of the cap surface on the host, for parameter checks and plots of the
surface; they take no part in the device return.

Pressure is compression-positive, so the tensile strength pT is ≤ 0.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import NamedTuple

import numpy as np
import torch

from . import _abi as abi
from .problem import _tuple
from .solver import _Handle, _check, _ptr

EPS = np.finfo(np.float64).eps


class DruckerPragerCap:
    """DruckerPragerCap(ϕ, Ψ, C, pT, η_reg, Kb; C_min=C, H_C=0) with angles in radians
    (stokes_types.jl:492-545). Stores cosϕ, sinϕ, sinΨ and the tuples as given; raises
    ValueError for the parameter sets the reference rejects."""

    def __init__(self, phi, psi, C, pT, eta_reg, Kb, C_min=None, H_C=None):
        phi, psi, C, pT, eta_reg, Kb = map(_tuple, (phi, psi, C, pT, eta_reg, Kb))
        n = len(phi)
        if not all(len(t) == n for t in (psi, C, pT, eta_reg, Kb)):
            raise ValueError("every tensile-cap parameter needs one value per phase")
        C_min = C if C_min is None else _tuple(C_min, n)
        H_C = (0.0,) * n if H_C is None else _tuple(H_C, n)
        if len(C_min) != n or len(H_C) != n:
            raise ValueError("every tensile-cap parameter needs one value per phase")
        for i in range(n):
            ph = i + 1
            vals = (phi[i], psi[i], C[i], pT[i], eta_reg[i], Kb[i], C_min[i], H_C[i])
            if not all(math.isfinite(v) for v in vals):
                raise ValueError(f"phase {ph}: tensile-cap parameters must all be finite")
            if pT[i] > 0:
                raise ValueError(f"phase {ph}: tensile strength pT must be ≤ 0 with compression-positive "
                                 f"pressure, got {pT[i]}")
            r = C[i] * math.cos(phi[i]) + math.sin(phi[i]) * pT[i]
            if not r > 0:
                raise ValueError(f"phase {ph}: cap radius is not positive; need C·cos(ϕ) + sin(ϕ)·pT > 0, "
                                 f"got {r}. Cohesion must exceed sin(ϕ)·|pT|.")
            if not Kb[i] > 0:
                raise ValueError(f"phase {ph}: dilatant plasticity requires a positive finite bulk modulus, "
                                 f"got {Kb[i]}")
            if not eta_reg[i] >= 0:
                raise ValueError(f"phase {ph}: η_reg must be ≥ 0, got {eta_reg[i]}")
            if not C_min[i] >= 0:
                raise ValueError(f"phase {ph}: C_min must be ≥ 0, got {C_min[i]}")
            if not C_min[i] <= C[i]:
                raise ValueError(f"phase {ph}: C_min must be ≤ C, got C_min={C_min[i]}, C={C[i]}")
            if not H_C[i] <= 0:
                raise ValueError(f"phase {ph}: H_C must be ≤ 0 for softening, got {H_C[i]}")
            if not C_min[i] * math.cos(phi[i]) + math.sin(phi[i]) * pT[i] > 0:
                raise ValueError(f"phase {ph}: softened cap radius must remain positive; "
                                 "need C_min·cos(ϕ) + sin(ϕ)·pT > 0")
        self.cos_phi = tuple(math.cos(x) for x in phi)
        self.sin_phi = tuple(math.sin(x) for x in phi)
        self.sin_psi = tuple(math.sin(x) for x in psi)
        self.C, self.pT, self.eta_reg, self.Kb, self.C_min, self.H_C = C, pT, eta_reg, Kb, C_min, H_C

    @property
    def nphases(self):
        return len(self.C)


class CapGeometry(NamedTuple):
    a: float
    b: float
    p_y: float
    R_y: float
    p_d: float
    tau_d: float
    p_q: float


def cap_geometry(k, kq, c, pT) -> CapGeometry:
    """Cap centre p_y and radius R_y (the circle through pT tangent to τII = k·P + c),
    the delimiter (p_d, τ_d), the potential centre p_q and the scalings a = √(1 + k²),
    b = √(1 + kq²) (rheology.jl:556-567; Popov et al. Eqs. 13-17)."""
    a = math.sqrt(1.0 + k * k)
    b = math.sqrt(1.0 + kq * kq)
    p_y = (a * pT + c) / (a - k)
    R_y = p_y - pT
    p_d = p_y - R_y * k / a
    tau_d = R_y / a
    return CapGeometry(a, b, p_y, R_y, p_d, tau_d, p_d + kq * tau_d)


def cap_yield_function(tII, P, k, c, geom: CapGeometry):
    """Composite yield function (rheology.jl:596-603; Eq. 18): the shear line where
    P + k·τII ≥ p_y, else a·(√(τII² + (P − p_y)² + eps²) − R_y)."""
    if P + k * tII >= geom.p_y:
        return tII - k * P - c
    return geom.a * (math.sqrt(tII * tII + (P - geom.p_y) ** 2 + EPS * EPS) - geom.R_y)


def softened_cohesion(C, C_min, H_C, gamma):
    """Linear cohesion softening clamp(C + H_C·γ, C_min, C) (rheology.jl:569-572)."""
    if gamma is None:
        return C
    return min(max(C + H_C * gamma, C_min), C)


def cap_invariants(s, p, k, kq, c, pT):
    """(F, Aτ, Ap) with Aτ = ½ ∂Q/∂s and Ap = −∂Q/∂p (rheology.jl:614-622); the yield and
    potential branches are chosen independently."""
    g = cap_geometry(k, kq, c, pT)
    F = cap_yield_function(s, p, k, c, g)
    if p + kq * s >= g.p_q:
        return F, 0.5, kq
    Rq = math.hypot(s, p - g.p_q)
    if Rq == 0.0:
        return F, 0.0, 0.0
    return F, g.b * s / (2 * Rq), -g.b * (p - g.p_q) / Rq


def cap_invariants_phase(plastic: DruckerPragerCap, phase, s, p, gamma=None):
    """cap_invariants(plastic, phase, s, p, γ) (rheology.jl:624-631): the phase's
    parameters (1-based phase) with cohesion softened by the accepted history γ."""
    i = phase - 1
    Cs = softened_cohesion(plastic.C[i], plastic.C_min[i], plastic.H_C[i], gamma)
    return cap_invariants(s, p, plastic.sin_phi[i], plastic.sin_psi[i], Cs * plastic.cos_phi[i], plastic.pT[i])


def _points(*args, shape=None):
    """Broadcast scalars / arrays / tensors to contiguous float64 CUDA tensors of one shape."""
    ts = [torch.as_tensor(a, dtype=torch.float64, device="cuda") for a in args]
    if shape is None:
        shape = torch.broadcast_shapes(*[t.shape for t in ts])
    try:
        return [t.expand(shape).reshape(-1).contiguous() for t in ts], torch.Size(shape)
    except RuntimeError:
        raise ValueError("the trial stresses and the point arrays differ in length") from None


def _run(ncomp, trial, P_trial, eta_ve, K_dt, k, kq, c, pT, eta_reg, maxiter):
    lib, h = _Handle.get()
    if ncomp == 0:
        (trial, Pt, eve, Kdt, k, kq, c, pT, er), shape = _points(trial, P_trial, eta_ve, K_dt, k, kq, c, pT, eta_reg)
    else:
        (Pt, eve, Kdt, k, kq, c, pT, er), shape = _points(P_trial, eta_ve, K_dt, k, kq, c, pT, eta_reg,
                                                          shape=(trial.shape[0],))
    n = Pt.numel()
    out = {name: torch.empty(n, dtype=torch.float64, device="cuda")
           for name in ("tau_II", "P", "lambda", "A_tau", "A_p", "gamma_dot", "theta_dot")}
    out["converged"] = torch.empty(n, dtype=torch.int32, device="cuda")
    if ncomp:
        out["tau"] = torch.empty(n, ncomp, dtype=torch.float64, device="cuda")
    prob = abi.CapProblemC()
    prob.n, prob.ncomp, prob.maxiter = n, ncomp, int(maxiter)
    if ncomp:
        prob.tau_trial = _ptr(trial)
    else:
        prob.s_trial = _ptr(trial)
    prob.P_trial, prob.eta_ve, prob.K_dt = _ptr(Pt), _ptr(eve), _ptr(Kdt)
    prob.k, prob.kq, prob.c, prob.pT, prob.eta_reg = _ptr(k), _ptr(kq), _ptr(c), _ptr(pT), _ptr(er)
    prob.tau = _ptr(out.get("tau"))
    prob.tau_II, prob.P, prob.lambda_ = _ptr(out["tau_II"]), _ptr(out["P"]), _ptr(out["lambda"])
    prob.A_tau, prob.A_p = _ptr(out["A_tau"]), _ptr(out["A_p"])
    prob.gamma_dot, prob.theta_dot, prob.converged = _ptr(out["gamma_dot"]), _ptr(out["theta_dot"]), _ptr(out["converged"])
    _check(lib, h, lib.femb200_cap_update(h, C.byref(prob)))
    out["converged"] = out["converged"].bool()
    return out, shape


def cap_return_map(s_trial, p_trial, eta_ve, K_dt, k, kq, c, pT, eta_reg, maxiter=40):
    """cap_return_map(s_trial, p_trial, ηve, KΔt, k, kq, c, pT, η_reg; maxiter=40)
    (rheology.jl:640-698) at every point of the broadcast inputs, on the device. Returns a
    dict of tensors: tau_II, P, lambda, A_tau, A_p, converged (and the rates λ·Aτ, λ·Ap
    as gamma_dot, theta_dot, NaN where the solve failed); a failed point keeps its trial
    state with converged False."""
    out, shape = _run(0, s_trial, p_trial, eta_ve, K_dt, k, kq, c, pT, eta_reg, maxiter)
    return {key: v.reshape(shape) for key, v in out.items()}


def cap_local_update(tau_trial, P_trial, eta_ve, K_dt, k, kq, c, pT, eta_reg, maxiter=40):
    """cap_local_update(τ_trial, P_trial, ηve, KΔt, k, kq, c, pT, η_reg) (rheology.jl:700-724)
    on the device: tau_trial is (n, 3) plane-strain (xx, yy, xy) or (n, 6) 3-D
    (xx, yy, zz, xy, xz, yz) stresses. Returns tau (radially corrected), P = P_trial +
    KΔt·θdot, gamma_dot, theta_dot (NaN everywhere for a failed local solve) and the return
    map's tau_II, lambda, A_tau, A_p, converged."""
    t = torch.as_tensor(tau_trial, dtype=torch.float64, device="cuda")
    if t.dim() == 1:
        t = t.unsqueeze(0)
    if t.shape[-1] not in (3, 6):
        raise ValueError("trial stresses need 3 (plane strain) or 6 (3-D) components")
    out, _ = _run(t.shape[-1], t.contiguous(), P_trial, eta_ve, K_dt, k, kq, c, pT, eta_reg, maxiter)
    return out
