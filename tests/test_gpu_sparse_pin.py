"""libfemtools_b200's StokesDR residual sweeps and DR solves against the sparse
Q2/P1-disc saddle-point system assembled from the element integrals
(tests/sparse_stokes.py; the reference's own pin, test/test_stokes_3d_reference.jl:
34-97, 155), through the C ABI.

FP64 sweeps must equal A·x − b to 1e-10 of the largest entry: the distorted mesh
takes the general sweep (per-point geometry), the sheared mesh the pipelined sweep
(one J⁻¹ per element); the FP32 sweeps to 2e-5. The FP64 and mixed-precision solves
(FP32 increments on the thread-per-element sweep inside FP64 Powell–Hestenes steps)
must converge to the sparse direct solution of the same system (the mixed solve on
affine cells, which it requires)."""
import numpy as np
import pytest

import oracle_host as oh
import sparse_stokes as ss
from conftest import fem

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _close(got, want, rtol, what):
    g = got.detach().cpu().double().numpy() if hasattr(got, "detach") else np.asarray(got)
    np.testing.assert_allclose(g, want, rtol=rtol, atol=rtol * np.abs(want).max(), err_msg=what)


@pytest.mark.parametrize("dtype", ["fp64", "fp32"])
@pytest.mark.parametrize("distort", [True, False])
@pytest.mark.parametrize("phases", ["nodal", "cell"])
def test_device_residuals_equal_the_sparse_system(dtype, distort, phases):
    case = ss.linear_vep_case(n=3, seed=8, distort=distort, phases=phases)
    hs = case.host_state(oh)
    blk = ss.assemble(case, case.dt, hs.gammaP, hs.M_P, hs.P0, hs.T, hs.T0, hs.tau_old)
    nv = 3 * case.mesh.nnodes
    tdt = torch.float64 if dtype == "fp64" else torch.float32
    dr = case.device_state(fem, dtype=tdt, geometry_dtype=tdt)
    # the state vector the device holds (FP32: the FP64 state rounded once)
    x = np.concatenate([np.concatenate([t.double().cpu().numpy() for t in dr.v]), dr.P.double().cpu().numpy()])
    rtol = 1e-10 if dtype == "fp64" else 2e-5
    A, b = ss.augmented_system(blk, with_pnum=False)
    ref = A @ x - b
    fem.assemble_pressure_residual(dr, case.dt)
    fem.assemble_momentum_residual(dr, case.dt, with_pnum=False)
    _close(torch.cat(list(dr.Rv)), ref[:nv], rtol, "Rv without Pnum")
    _close(dr.RP, ref[nv:], rtol, "RP")
    A, b = ss.augmented_system(blk, with_pnum=True)
    ref = A @ x - b
    fem.assemble_stokes_residuals(dr, case.dt)
    _close(torch.cat(list(dr.Rv)), ref[:nv], rtol, "Rv with Pnum (fused sweep)")
    _close(dr.RP, ref[nv:], rtol, "RP (fused sweep)")
    _close(dr.Pnum, blk["D"] @ ref[nv:], rtol, "Pnum (fused sweep)")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_solve_converges_to_the_sparse_solution(precision):
    # the mixed-precision solve needs affine cells: it runs on the undistorted box
    case = ss.layered_solve_case(n=2, seed=3, distort=precision == "fp64")
    hs = case.host_state(oh)
    blk = ss.assemble(case, case.dt, hs.gammaP, hs.M_P, hs.P0, hs.T, hs.T0, hs.tau_old)
    v_ref, P_ref = ss.sparse_solution(case, blk)
    dr = case.device_state(fem)
    st = fem.solve(dr, case.bc_device(), dt=case.dt, tolerance=1e-11, check_interval=50, max_iterations=200_000,
                   iter_max=200_000, precision=precision)
    assert st["converged"]
    v = torch.cat(list(dr.v)).cpu().numpy()
    bound = 1e-7 if precision == "fp64" else 1e-6
    assert np.linalg.norm(v - v_ref) <= bound * np.linalg.norm(v_ref)
    assert np.linalg.norm(dr.P.cpu().numpy() - P_ref) <= bound * np.linalg.norm(P_ref)
