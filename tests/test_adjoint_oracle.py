"""The oracle's adjoint operator, pinned against finite differences of its own
forward residual (the reference's FD checks of the adjoint, test/test_stokes_adjoint_api.jl:47-130
and test/test_stokes_3d_reference.jl:190-209, restated on element states).

Φ(u) = λv·Rv(u) + λP·RP(u), with Rv carrying Pnum = γP·RP/M_P formed inline (the
residual the DR loop drives to zero): its gradient in v and P is (dR/du)ᵀλ, and its
derivative in the viscosity of one integration point is λ·∂R/∂η_q.
"""
import numpy as np
import pytest

import oracle_host as oh
from cases import random_state_case, vep_layers_case


def phi(hs, dt, lam_v, lam_P, finite_K):
    hs.stokes_residuals(dt, finite_K=finite_K)
    return sum(float(np.dot(lam_v[c], hs.Rv[c])) for c in range(3)) + float(np.dot(lam_P, hs.RP))


def host_with_state(case):
    hs = case.host_state(oh)
    if case.gammaP is None:
        rng = np.random.default_rng(11)
        hs.gammaP[:] = rng.uniform(1, 5, hs.mesh.nnodesP)
        hs.M_P[:] = rng.uniform(0.01, 0.1, hs.mesh.nnodesP)
    return hs


@pytest.mark.parametrize("plastic,finite_K", [(False, False), (True, False), (True, True)])
def test_oracle_adjoint_matches_finite_differences(plastic, finite_K):
    case = random_state_case(dim=3, n=2, seed=21, phases="nodal", plastic=plastic, distort=True)
    hs = host_with_state(case)
    dt = case.dt
    rng = np.random.default_rng(5)
    lam_v = [rng.standard_normal(hs.mesh.nnodes) for _ in range(3)]
    lam_P = rng.standard_normal(hs.mesh.nnodesP)
    dv, dP = hs.adjoint_residual(dt, lam_v, lam_P, finite_K=finite_K)
    h = 1e-6
    for c, idx in [(0, 7), (1, 30), (2, 62), (0, 124)]:
        x0 = hs.v[c][idx]
        hs.v[c][idx] = x0 + h; fp = phi(hs, dt, lam_v, lam_P, finite_K)
        hs.v[c][idx] = x0 - h; fm = phi(hs, dt, lam_v, lam_P, finite_K)
        hs.v[c][idx] = x0
        fd = (fp - fm) / (2 * h)
        assert abs(fd - dv[c][idx]) <= 1e-6 * max(1.0, abs(fd)), (c, idx, fd, dv[c][idx])
    for k in (0, 5, 17, 31):
        x0 = hs.P[k]
        hs.P[k] = x0 + h; fp = phi(hs, dt, lam_v, lam_P, finite_K)
        hs.P[k] = x0 - h; fm = phi(hs, dt, lam_v, lam_P, finite_K)
        hs.P[k] = x0
        fd = (fp - fm) / (2 * h)
        assert abs(fd - dP[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, dP[k])


def test_oracle_viscosity_sensitivity_matches_finite_differences():
    case = random_state_case(dim=3, n=2, seed=22, phases="cell", plastic=True, distort=True)
    hs = host_with_state(case)
    dt = case.dt
    rng = np.random.default_rng(6)
    hs.viscosity_ip = 10 ** rng.uniform(0, 1, hs.mesh.nq * hs.mesh.nels)
    lam_v = [rng.standard_normal(hs.mesh.nnodes) for _ in range(3)]
    lam_P = rng.standard_normal(hs.mesh.nnodesP)
    sens = hs.viscosity_sensitivity(dt, lam_v, lam_P)
    h = 1e-6
    for q in (0, 13, 40, 150, 215):
        x0 = hs.viscosity_ip[q]
        hs.viscosity_ip[q] = x0 + h; fp = phi(hs, dt, lam_v, lam_P, False)
        hs.viscosity_ip[q] = x0 - h; fm = phi(hs, dt, lam_v, lam_P, False)
        hs.viscosity_ip[q] = x0
        fd = (fp - fm) / (2 * h)
        assert abs(fd - sens[q]) <= 1e-6 * max(1.0, abs(fd)), (q, fd, sens[q])


def dense_adjoint(hs, dt, obj, bc):
    """λ from the transposed Jacobian assembled column by column through the oracle's
    adjoint operator, restricted to the unconstrained DoFs (λ = 0 on Dirichlet DoFs)."""
    nn, nP = hs.mesh.nnodes, hs.mesh.nnodesP
    n = 3 * nn + nP
    fixed = np.zeros(n, dtype=bool)
    for c, (dofs, _) in enumerate(bc):
        fixed[c * nn + np.asarray(dofs) - 1] = True
    free = np.nonzero(~fixed)[0]
    A = np.zeros((len(free), len(free)))
    for k, j in enumerate(free):
        e = np.zeros(n)
        e[j] = 1.0
        dv, dP = hs.adjoint_residual(dt, [e[c * nn:(c + 1) * nn] for c in range(3)], e[3 * nn:])
        col = np.concatenate(dv + [dP])
        A[:, k] = col[free]
    rhs = -np.concatenate(obj + [np.zeros(nP)])[free]
    lam = np.zeros(n)
    lam[free] = np.linalg.solve(A, rhs)
    return [lam[c * nn:(c + 1) * nn] for c in range(3)], lam[3 * nn:]


def forward_J(ac, delta, tol=1e-13):
    hs = ac.case.host_state(oh)
    hs.viscosity_ip = ac.eta_ip(delta)
    st = hs.solve(dt=ac.case.dt, tolerance=tol, check_interval=50, max_iterations=400000, iter_max=400000,
                  throw_on_failure=False)
    assert st["converged"]
    return ac.objective(hs.v)[0], hs


def test_oracle_adjoint_gradient_matches_fd():
    # dJ/dδ_e = Σ_q η_q λ·∂R/∂η_q with λ from the transposed augmented Jacobian
    # (the reference checks its adjoint gradient against central differences,
    # test/test_stokes_adjoint_api.jl:47-130).
    from cases import fem
    ac = fem.configs.adjoint_case(n=2, seed=1)
    J0, hs = forward_J(ac, ac.delta)
    _, obj = ac.objective(hs.v)
    lam_v, lam_P = dense_adjoint(hs, ac.case.dt, obj, ac.case.bc)
    sens = hs.viscosity_sensitivity(ac.case.dt, lam_v, lam_P)
    eta = ac.eta_ip()
    grad = (eta * sens).reshape(hs.mesh.nels, hs.mesh.nq).sum(axis=1)
    h = 1e-4
    for k in range(hs.mesh.nels):
        d = ac.delta.copy(); d[k] += h
        Jp, _ = forward_J(ac, d)
        d[k] -= 2 * h
        Jm, _ = forward_J(ac, d)
        fd = (Jp - Jm) / (2 * h)
        assert abs(fd - grad[k]) <= 1e-5 * np.abs(grad).max() + 1e-6 * abs(fd), (k, fd, grad[k])
