"""Lithostatic pressure (LithostaticPressureDR) through the C ABI against the CPU
oracle (itself pinned to the reference's known answers in test_lithostatic_oracle.py).
FP64 assemblies agree to 1e-12 of their largest entry (atomic scatter order); full
relaxations take the same number of iterations and agree to 1e-9 relative."""
import math

import numpy as np
import pytest

import oracle_host as oh
from cases import random_state_case
from conftest import fem

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
abi = fem._abi


def host(x):
    return x.detach().cpu().numpy()


def close(got, want, rel):
    np.testing.assert_allclose(host(got), want, rtol=0, atol=rel * max(np.abs(want).max(), 1e-300))


MAT = dict(rho0=(3.3, 2.9), alpha=(3e-2, 1e-2), K=(50.0, math.inf))


def states(dim, seed):
    mesh = random_state_case(dim=dim, n=3, seed=seed, distort=True).mesh
    rng = np.random.default_rng(seed)
    ph = rng.integers(1, 3, mesh.nnodes).astype(np.int32)
    T = rng.uniform(0.0, 2.0, mesh.nnodes)
    P = rng.standard_normal(mesh.nnodes)
    dr = fem.LithostaticPressureDR(mesh, phases=ph, **MAT)
    dr.T.copy_(torch.as_tensor(T, device="cuda"))
    dr.P.copy_(torch.as_tensor(P, device="cuda"))
    hs = oh.HostLithostatic(mesh, phases=ph, T=T, P=P, **MAT)
    return mesh, dr, hs


@pytest.mark.parametrize("dim", [2, 3])
def test_residual_and_jacobian_match_oracle(dim):
    mesh, dr, hs = states(dim, seed=5 + dim)
    g = (0.2, -1.0) if dim == 2 else (0.1, 0.2, -1.0)
    fem.assemble_lithostatic_pressure(dr, Tref=0.5, g=g, compute_jacobian=True)
    hs.residual(0.5, g, jac=True)
    close(dr.R, hs.R, 1e-12)
    close(dr.dRdP, hs.dRdP, 1e-12)
    close(dr.PC, hs.PC, 1e-12)


@pytest.mark.parametrize("dim", [2, 3])
def test_solve_matches_oracle(dim):
    mesh, dr, hs = states(dim, seed=11 + dim)
    h = mesh.coords[:, dim - 1]
    top = (np.nonzero(np.abs(h - 1.0) < 1e-12)[0] + 1).astype(np.int32)
    bc = (top, np.zeros(len(top)))
    g = (0.0, -1.0) if dim == 2 else (0.0, 0.0, -1.0)
    st = fem.solve_lithostatic(dr, bc, Tref=0.5, g=g, tolerance=1e-9, max_iterations=100_000)
    ref = hs.solve(bc, Tref=0.5, g=g, tolerance=1e-9, max_iterations=100_000)
    assert st["converged"] and ref.converged
    assert st["iterations"] == ref.iterations
    close(dr.P, hs.P, 1e-9)


def test_hydrostatic_and_errors():
    mesh = fem.structured_mixed_mesh(3, (3, 3, 3))
    z = mesh.coords[:, 2]
    top = (np.nonzero(np.abs(z - 1.0) < 1e-12)[0] + 1).astype(np.int32)
    dr = fem.LithostaticPressureDR(mesh, rho0=(2.0,))
    st = fem.solve_lithostatic(dr, (top, np.zeros(len(top))), Tref=0.0, g=(0.0, 0.0, -1.0), tolerance=1e-11,
                               max_iterations=200_000)
    assert st["converged"]
    np.testing.assert_allclose(host(dr.P), 2.0 * (1.0 - z), atol=1e-8)
    with pytest.raises(ValueError, match="needs g"):
        fem.solve_lithostatic(dr, (top, np.zeros(len(top))))
    with pytest.raises(abi.FemB200Error, match="Lithostatic pressure DR solver did not converge after 1 "):
        fem.solve_lithostatic(dr, (top, np.zeros(len(top))), g=(0.0, 0.0, -1.0), tolerance=0.0, max_iterations=1,
                              check_interval=1)
