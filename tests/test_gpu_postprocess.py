"""Device strain-rate / stress diagnostics (compute_strain_rate_stress_postprocess,
src/postprocess/postprocess.jl) through the C ABI against the CPU oracle, plus the
reference's known answers. FP64 bound: 1e-12 of the largest value of each field (the
gradient is contracted in a different order than the oracle's)."""
import math

import numpy as np
import pytest

import oracle_host as oh
from cases import random_state_case
from conftest import fem

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def host(x):
    return x.detach().cpu().numpy()


@pytest.mark.parametrize("dim", [3, 2])
def test_diagnostics_match_oracle_on_distorted_mesh(dim):
    case = random_state_case(dim=dim, n=3, seed=21, distort=True)
    dr = case.device_state(fem)
    nt = 6 if dim == 3 else 3
    rng = np.random.default_rng(4)
    tau = [rng.standard_normal(case.mesh.nq * case.mesh.nels) for _ in range(nt)]
    post = fem.compute_strain_rate_stress_postprocess(dr, tau)
    ref = oh.strain_rate_stress(dim, case.mesh.el2n, case.mesh.geo_v, case.v, tau)
    assert len(post) == len(ref)
    for name, got, want in zip(post._fields, post, ref):
        np.testing.assert_allclose(host(got), want, rtol=0, atol=1e-12 * max(np.abs(want).max(), 1e-300),
                                   err_msg=name)


def test_constant_plane_stress_known_answer():
    # τ = (2, −1, 0.5) at every point, v = 0: τII = √3.25 (τzz = −(τxx + τyy)), ε = 0
    case = random_state_case(dim=2, n=2, seed=1, distort=True)
    dr = case.device_state(fem)
    for c in range(2):
        dr.v[c].zero_()
    n = case.mesh.nq * case.mesh.nels
    post = fem.compute_strain_rate_stress_postprocess(dr, [np.full(n, 2.0), np.full(n, -1.0), np.full(n, 0.5)])
    np.testing.assert_allclose(host(post.tauII), math.sqrt(3.25), rtol=1e-14)
    np.testing.assert_allclose(host(post.τzz), -1.0, rtol=1e-14)
    assert np.all(host(post.εII) == 0.0)


def test_linear_velocity_gives_its_constant_strain_rate():
    # Q2 elements reproduce v = A·x exactly, distorted or not: every cell average is sym(A)
    case = random_state_case(dim=3, n=3, seed=2, distort=True)
    A = np.array([[0.3, -0.2, 0.5], [0.1, 0.7, -0.4], [0.2, 0.6, -1.0]])
    dr = case.device_state(fem)
    x = case.mesh.coords
    for c in range(3):
        dr.v[c].copy_(torch.as_tensor(x @ A[c], device="cuda"))
    n = case.mesh.nq * case.mesh.nels
    post = fem.compute_strain_rate_stress_postprocess(dr, [np.zeros(n)] * 6)
    S = 0.5 * (A + A.T)
    want = {"εxx": S[0, 0], "εyy": S[1, 1], "εzz": S[2, 2], "εxy": S[0, 1], "εxz": S[0, 2], "εyz": S[1, 2]}
    for name, val in want.items():
        np.testing.assert_allclose(host(getattr(post, name)), val, rtol=0, atol=1e-12)
    dev = S - np.trace(S) / 3 * np.eye(3)
    eII = math.sqrt(0.5 * (dev[0, 0] ** 2 + dev[1, 1] ** 2 + dev[2, 2] ** 2) + dev[0, 1] ** 2 + dev[0, 2] ** 2
                    + dev[1, 2] ** 2 + np.finfo(float).eps ** 2)
    np.testing.assert_allclose(host(post.εII), eII, rtol=1e-12)


def test_fp32_state_keeps_fp32():
    case = random_state_case(dim=3, n=2, seed=3, distort=True)
    dr = case.device_state(fem, dtype=torch.float32, geometry_dtype=torch.float32)
    n = case.mesh.nq * case.mesh.nels
    post = fem.compute_strain_rate_stress_postprocess(dr, [np.ones(n)] * 6)
    assert post.tauII.dtype == torch.float32
    ref = oh.strain_rate_stress(3, case.mesh.el2n, case.mesh.geo_v, case.v, [np.ones(n)] * 6)
    np.testing.assert_allclose(host(post.εxx), ref[0], rtol=0, atol=2e-5 * np.abs(ref[0]).max())


def test_solve_then_write_vtk(tmp_path):
    # the current stress of a state after update_stokes_current_stress, diagnosed on the
    # device, projected to nodes and written out
    case = random_state_case(dim=3, n=2, seed=6, distort=False)
    dr = case.device_state(fem)
    fem.update_stokes_current_stress(dr, case.dt)
    post = fem.compute_strain_rate_stress_postprocess(dr)
    tau_nodal = [np.zeros(case.mesh.nnodes) for _ in range(6)]
    fem.update_old_stress_from_cells(tau_nodal, post, case.mesh.el2n, case.mesh.nnodes)
    path = tmp_path / "stokes.vtk"
    fem.write_stokes_vtk(str(path), case.mesh, case.mesh.coords, case.mesh.el2nP, case.mesh.dofsP,
                         host(dr.P), [host(v) for v in dr.v], post)
    text = path.read_text()
    assert f"CELL_DATA {case.mesh.nels}" in text and "TENSORS tau float" in text
    assert np.all(np.isfinite(tau_nodal[0]))
