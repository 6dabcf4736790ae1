"""Cell-pressure Hex27 Stokes (CellPressureStokesDR) through the C ABI against the CPU
oracle (itself pinned to the sparse saddle-point system in test_cellpressure_oracle.py).
Element sums run in a different order on the device (warp reductions, FP64 atomics),
so assemblies agree to 1e-12 of their largest entry; full relaxations take the same
number of iterations and agree to 1e-9 relative."""
import ctypes as C

import numpy as np
import pytest

import oracle_host as oh
from conftest import fem

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
abi = fem._abi


def host(x):
    return x.detach().cpu().numpy()


def close(got, want, rel):
    np.testing.assert_allclose(host(got), want, rtol=0, atol=rel * max(np.abs(want).max(), 1e-300))


def states(n=3, seed=4, distort=True, random=True):
    case = fem.configs.cell_pressure_case(n=n, seed=seed, distort=distort)
    rng = np.random.default_rng(seed + 10)
    v = [rng.standard_normal(case.mesh.nnodes) for _ in range(3)] if random else None
    P = rng.standard_normal(4 * case.mesh.nels) if random else None
    dr = fem.CellPressureStokesDR(case.mesh, case.material, phases=case.phases)
    if random:
        for c in range(3):
            dr.v[c].copy_(torch.as_tensor(v[c], device="cuda"))
        dr.P.copy_(torch.as_tensor(P, device="cuda"))
    hs = oh.HostCellPressure(case.mesh, case.material.eta, case.material.rho0, case.material.g, case.phases, v, P)
    return case, dr, hs


@pytest.mark.parametrize("distort", [False, True])
def test_assemblies_match_oracle(distort):
    case, dr, hs = states(distort=distort)
    fem.stokes_preconditioner_3d(dr)
    fem.assemble_stokes_pressure_residual_3d(dr)
    fem.assemble_stokes_momentum_residual_3d(dr)
    hs.preconditioner()
    hs.residuals(3)
    for c in range(3):
        close(dr.diagonal[c], hs.diagonal[c], 1e-12)
        close(dr.Rv[c], hs.Rv[c], 1e-12)
    close(dr.pressure_mass, hs.pressure_mass, 1e-12)
    close(dr.RP, hs.RP, 1e-12)


@pytest.mark.parametrize("distort", [True, False])
def test_solve_matches_oracle(distort):
    # an undistorted box has affine cells: the device solve then reads one J⁻¹ and
    # |det J| per cell, the oracle still every quadrature point
    case, dr, hs = states(n=3, seed=2, distort=distort, random=False)
    kw = dict(tolerance=1e-8, max_iterations=100000, check_interval=100)
    st = fem.solve_cell_pressure(dr, case.bc, collect_history=True, **kw)
    ref = hs.solve(case.bc, **kw)
    assert st["converged"] and ref.converged
    assert st["iterations"] == ref.iterations
    assert len(st["history"]) == ref.iterations // 100
    for c in range(3):
        close(dr.v[c], hs.v[c], 1e-9)
    close(dr.P, hs.P, 1e-9)
    # boundary velocities pinned, the mean of the constant mode removed
    for c in range(3):
        assert torch.all(dr.v[c][torch.as_tensor(case.bc[c][0] - 1, device="cuda").long()] == 0)
    M0 = host(dr.pressure_mass)[0::4]
    assert abs((host(dr.P)[0::4] * M0).sum()) <= 1e-12 * np.abs(host(dr.P)).max() * M0.sum()


def test_load_stands_in_for_gravity():
    # the same block driven by a momentum load instead of gravity reaches the same state
    case, dr, _ = states(n=2, seed=3, random=False)
    fem.assemble_stokes_momentum_residual_3d(dr)                  # v = 0, P = 0: Rv = −∫ N ρ g
    load = [(-r).clone() for r in dr.Rv]
    kw = dict(tolerance=1e-9, max_iterations=100000, check_interval=100)
    fem.solve_cell_pressure(dr, case.bc, **kw)
    mat0 = fem.StokesMaterial(eta=case.material.eta, rho0=case.material.rho0, g=(0.0, 0.0, 0.0))
    dr0 = fem.CellPressureStokesDR(case.mesh, mat0, phases=case.phases)
    fem.solve_cell_pressure(dr0, case.bc, load=load, **kw)
    for c in range(3):
        close(dr0.v[c], host(dr.v[c]), 1e-6)


def test_non_convergence_and_validation():
    case, dr, _ = states(n=2, seed=1, random=False)
    with pytest.raises(abi.FemB200Error, match="3-D Stokes solve did not converge after 200 iterations"):
        fem.solve_cell_pressure(dr, case.bc, tolerance=1e-14, max_iterations=200)
    st = fem.solve_cell_pressure(dr, case.bc, tolerance=1e-14, max_iterations=150, throw_on_failure=False)
    assert not st["converged"] and st["reached_total_iter"] and st["iterations"] == 150
    with pytest.raises(ValueError, match="phases must lie in 1:2"):
        fem.CellPressureStokesDR(case.mesh, case.material, phases=np.full(case.mesh.nels, 3))
    with pytest.raises(ValueError, match="purely viscous"):
        fem.CellPressureStokesDR(case.mesh, fem.StokesMaterial(eta=(1.0,), G=(1.0,), g=(0.0, 0.0, -1.0)))
    # the library checks phases and connectivity on the device before any gather by them
    lib, h = fem.solver._Handle.get()
    dr.phases.fill_(5)
    with pytest.raises(abi.FemB200Error, match="phases must lie in 1:nphases"):
        fem.solver._check(lib, h, lib.femb200_cell_pressure_residuals(h, C.byref(dr.problem()), 3))
    dr.phases.fill_(1)
    dr.el2n[0, 3] = case.mesh.nnodes + 7
    with pytest.raises(abi.FemB200Error, match="connectivity entry outside"):
        fem.solve_cell_pressure(dr, case.bc)


def _sparse_solution(case, objective=None):
    import dataclasses  # noqa: F401
    import scipy.sparse.linalg as spla
    from test_cellpressure_oracle import sparse_stokes_reference
    A, rhs, free = sparse_stokes_reference(case)
    x = np.zeros(len(rhs))
    Af = A[free][:, free].tocsc()
    x[free] = spla.spsolve(Af, rhs[free])
    lam = None
    if objective is not None:
        lam = np.zeros(len(rhs))
        lam[free] = spla.spsolve(Af.T.tocsc(), objective[free])
    return x, lam


def test_adjoint_and_material_gradients_match_the_sparse_system():
    # solve_adjoint! and stokes_material_gradient_3d (DR_adjoint.jl:446-531) against the
    # transposed sparse system and central differences of its solutions
    import dataclasses
    case = fem.configs.cell_pressure_case(n=2, seed=5, distort=True)
    mesh = case.mesh
    nn, nv = mesh.nnodes, 3 * mesh.nnodes
    rng = np.random.default_rng(12)
    obj = [rng.standard_normal(nn) for _ in range(3)]
    for c in range(3):
        obj[c][case.bc[c][0] - 1] = 0.0
    objective = np.concatenate([np.stack(obj, axis=1).ravel(), np.zeros(4 * mesh.nels)])
    x, lam = _sparse_solution(case, objective)
    dr = fem.CellPressureStokesDR(mesh, case.material, phases=case.phases)
    fem.solve_cell_pressure(dr, case.bc, tolerance=1e-11, max_iterations=400_000)
    lv, lP, st = fem.solve_adjoint_cell_pressure(dr, case.bc, obj, tolerance=1e-11, max_iterations=400_000)
    assert st["converged"]
    lam_v = lam[:nv].reshape(-1, 3)
    got = np.stack([host(t) for t in lv], axis=1)
    assert np.linalg.norm(got - lam_v) <= 1e-6 * np.linalg.norm(lam_v)
    assert np.allclose(host(dr.v[2]), x[:nv].reshape(-1, 3)[:, 2], atol=1e-6 * np.abs(x[:nv]).max())
    grads = fem.stokes_material_gradient_3d(dr, lv)
    J = lambda cs: float(objective @ _sparse_solution(cs)[0])
    h = 1e-5
    for p in range(len(case.material.eta)):
        rho = list(case.material.rho0)
        rp, rm = list(rho), list(rho)
        rp[p] += h
        rm[p] -= h
        mat = lambda r=None, e=None: fem.StokesMaterial(eta=e or case.material.eta, rho0=r or rho, g=case.material.g)
        fd_rho = (J(dataclasses.replace(case, material=mat(r=rp))) - J(dataclasses.replace(case, material=mat(r=rm)))) / (2 * h)
        eta = list(case.material.eta)
        ep, em = list(eta), list(eta)
        ep[p] *= 1 + h
        em[p] *= 1 - h
        fd_eta = (J(dataclasses.replace(case, material=mat(e=ep))) - J(dataclasses.replace(case, material=mat(e=em)))) / (2 * h * eta[p])
        assert abs(grads["density_gradient"][p] - fd_rho) <= 1e-4 * max(abs(fd_rho), 1e-12)
        assert abs(grads["viscosity_gradient"][p] - fd_eta) <= 1e-4 * max(abs(fd_eta), 1e-12)
    # the forward state is untouched by the adjoint solve
    assert np.allclose(host(dr.v[2]), x[:nv].reshape(-1, 3)[:, 2], atol=1e-6 * np.abs(x[:nv]).max())


def test_nan_velocity_raises_the_non_finite_exit():
    # src/stokes/solvers/DR.jl:1041-1044: max(maximum(norm, Rv), norm(RP)) carries a NaN
    # into isfinite(err); the oracle stops with the same message
    case, dr, hs = states(n=2, seed=1, random=False)
    node = int(np.setdiff1d(np.arange(1, case.mesh.nnodes + 1), case.mesh.boundary_nodes)[0]) - 1
    dr.v[1][node] = float("nan")
    hs.v[1][node] = np.nan
    with pytest.raises(abi.FemB200Error) as ref:
        hs.solve(case.bc, tolerance=1e-8, max_iterations=1000, check_interval=100)
    with pytest.raises(abi.FemB200Error) as got:
        fem.solve_cell_pressure(dr, case.bc, tolerance=1e-8, max_iterations=1000, check_interval=100)
    assert got.value.code == ref.value.code == abi.ENONFINITE
    assert str(got.value) == str(ref.value) == "non-finite residual in 3-D Stokes solve"
