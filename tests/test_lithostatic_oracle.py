"""The oracle's lithostatic-pressure path (LithostaticPressureDR), pinned to the known
answers of the reference's test/test_lithostatic_pressure.jl (element residual,
parameters, stiffness term, EOS Jacobian, multi-phase density, the finite incompressible
limit) and to the exact
hydrostatic solution P = ρ|g|(1 − height) that Q2 elements reproduce."""
import math

import numpy as np
import pytest

import oracle_host as oh
from conftest import fem

# one integration point with identity J⁻¹: physical gradients [0 1; 0 −1], N = (½, ½), dΩ = 1
N1 = [[0.5, 0.5]]
G1 = [[[0.0, 1.0], [0.0, -1.0]]]


def el(P, T=(300.0, 300.0), phases=(1, 1), rho0=(2.0,), alpha=(0.1,), K=(100.0,), Tref=300.0, g=(0.0, -1.0)):
    return oh.lithostatic_element(N1, G1, [1.0], P, T, phases, rho0, alpha, K, Tref, g)


def test_residual_parameters():
    r1, _, _ = el([0.0, 0.0])
    r2, _, _ = el([0.0, 0.0], g=(0.0, -2.0))
    r3, _, _ = el([0.0, 0.0], Tref=290.0)
    np.testing.assert_allclose(r1, [-2.0, 2.0], rtol=1e-14)
    np.testing.assert_allclose(r2, 2 * r1, rtol=1e-14)
    np.testing.assert_allclose(r3, [0.0, 0.0], atol=1e-14)


def test_stiffness_term():
    r, _, _ = el([2.0, 0.0])
    np.testing.assert_allclose(r, [-4.02, 4.02], rtol=1e-14)


def test_jacobian_includes_the_eos_pressure_term():
    _, rows, diag = el([2.0, 0.0])
    np.testing.assert_allclose(rows, [2.0, 2.0], rtol=1e-14)
    np.testing.assert_allclose(diag, [1.01, 0.99], rtol=1e-14)


def test_multi_phase_density():
    r, _, _ = el([0.0, 0.0], phases=(1, 2), rho0=(2.0, 4.0), alpha=(0.1, 0.1), K=(100.0, 100.0))
    np.testing.assert_allclose(r, [-3.0, 3.0], rtol=1e-14)


@pytest.mark.parametrize("dim", [2, 3])
def test_hydrostatic_solution_is_reproduced(dim):
    mesh = fem.structured_mixed_mesh(dim, (4,) * dim if dim == 2 else (2,) * dim)
    rho = 1.3
    h = mesh.coords[:, dim - 1]
    top = (np.nonzero(np.abs(h - 1.0) < 1e-12)[0] + 1).astype(np.int32)
    g = (0.0, -1.0) if dim == 2 else (0.0, 0.0, -1.0)
    hs = oh.HostLithostatic(mesh, rho0=(rho,), alpha=(0.0,), K=(math.inf,))
    st = hs.solve((top, np.zeros(len(top))), Tref=0.0, g=g, tolerance=1e-11, max_iterations=200_000)
    assert st.converged
    np.testing.assert_allclose(hs.P, rho * (1.0 - h), atol=1e-8)


def test_non_convergence_message():
    mesh = fem.structured_mixed_mesh(2, (4, 4))
    top = (np.nonzero(np.abs(mesh.coords[:, 1] - 1.0) < 1e-12)[0] + 1).astype(np.int32)
    hs = oh.HostLithostatic(mesh)
    with pytest.raises(fem._abi.FemB200Error, match="Lithostatic pressure DR solver did not converge after 1 "):
        hs.solve((top, np.zeros(len(top))), Tref=0.0, g=(0.0, -1.0), tolerance=0.0, max_iterations=1,
                 check_interval=1)


def test_incompressible_limit_stays_finite():
    # test/test_lithostatic_pressure.jl:186-206: with a negative shape value, K = ∞ stays finite
    # (1/K is interpolated) and a stiff finite K approaches it
    N, P, g = [[-0.25, 1.25]], [1.0e6, 1.0e6], (0.0, -9.81)
    inc, _, _ = oh.lithostatic_element(N, G1, [1.0], P, (300.0, 300.0), (1, 1), (2.0,), (0.1,), (math.inf,), 300.0, g)
    assert np.isfinite(inc).all()
    stiff, _, _ = oh.lithostatic_element(N, G1, [1.0], P, (300.0, 300.0), (1, 1), (2.0,), (0.1,), (1.0e30,), 300.0, g)
    np.testing.assert_allclose(stiff, inc, rtol=1e-12)
