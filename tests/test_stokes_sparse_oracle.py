"""The oracle's StokesDR Hex27/P1-disc residuals, pinned the way the reference pins its
matrix-free Stokes residuals (test/test_stokes_3d_reference.jl:34-97, 155): they must
equal A·x − b of the sparse saddle-point system assembled directly from the element
integrals (tests/sparse_stokes.py), to rtol 1e-11, on distorted and affinely sheared
meshes, for every phase layout; and the oracle's DR solve must converge to the sparse
direct solution of that system.

The case is visco-elastic (finite G with a random stress history, finite bulk
viscosity, thermal expansion and a pressure-dependent density): every linear term
of the element residual is exercised; plasticity, the only non-affine term, is off."""
import numpy as np
import pytest

import oracle_host as oh
import sparse_stokes as ss


def _blocks(case, hs):
    return ss.assemble(case, case.dt, hs.gammaP, hs.M_P, hs.P0, hs.T, hs.T0, hs.tau_old)


def _close(got, want, rtol, what):
    np.testing.assert_allclose(got, want, rtol=rtol, atol=rtol * np.abs(want).max(), err_msg=what)


@pytest.mark.parametrize("distort", [True, False])
@pytest.mark.parametrize("phases", ["nodal", "cell", "element"])
def test_residuals_equal_the_sparse_system(distort, phases):
    case = ss.linear_vep_case(n=2, seed=5, distort=distort, phases=phases)
    hs = case.host_state(oh)
    blk = _blocks(case, hs)
    x = np.concatenate([np.concatenate(hs.v), hs.P])
    nv = 3 * case.mesh.nnodes
    # Pnum off: the pressure residual and the momentum residual with P alone
    A, b = ss.augmented_system(blk, with_pnum=False)
    ref = A @ x - b
    hs.pressure_residual(case.dt)
    hs.momentum_residual(case.dt, with_pnum=False)
    _close(np.concatenate(hs.Rv), ref[:nv], 1e-11, "Rv without Pnum")
    _close(hs.RP, ref[nv:], 1e-11, "RP")
    # the fused sweep: RP, Pnum = γP·RP/M_P, Rv with P + Pnum
    A, b = ss.augmented_system(blk, with_pnum=True)
    ref = A @ x - b
    hs.stokes_residuals(case.dt)
    _close(np.concatenate(hs.Rv), ref[:nv], 1e-11, "Rv with Pnum")
    _close(hs.RP, ref[nv:], 1e-11, "RP (fused)")
    _close(hs.Pnum, blk["D"] @ ref[nv:], 1e-11, "Pnum")


def test_solve_converges_to_the_sparse_solution():
    case = ss.layered_solve_case(n=2, seed=3)
    hs = case.host_state(oh)
    v_ref, P_ref = ss.sparse_solution(case, _blocks(case, hs))
    st = hs.solve(dt=case.dt, tolerance=1e-11, check_interval=50, max_iterations=200_000, iter_max=200_000)
    assert st["converged"]
    v = np.concatenate(hs.v)
    assert np.linalg.norm(v - v_ref) <= 1e-7 * np.linalg.norm(v_ref)
    assert np.linalg.norm(hs.P - P_ref) <= 1e-7 * np.linalg.norm(P_ref)
