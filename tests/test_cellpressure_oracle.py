"""The oracle's cell-pressure Hex27 Stokes path (CellPressureStokesDR), pinned the way
the reference pins its own (test/test_stokes_3d_reference.jl:24-97, :147-155): the
matrix-free momentum and continuity residuals must equal A·x − rhs of the sparse
Q2/P1-disc saddle-point system assembled directly from the element integrals, and the
relaxation must converge to the sparse direct solution (velocity; the pressure is
fixed only up to the constant mode). The sparse assembly below is restated from that
test's text."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import oracle_host as oh
from conftest import fem


def sparse_stokes_reference(case):
    mesh = case.mesh
    t = fem.element_tables(3)
    eta, rho, g = case.material.eta, case.material.rho0, case.material.g
    nn, ne = mesh.nnodes, mesh.nels
    nv, npr = 3 * nn, 4 * ne
    rows, cols, vals = [], [], []
    rhs = np.zeros(nv + npr)
    I3 = np.eye(3)
    modes = np.column_stack([np.ones(27), t.NP[:, 1], t.NP[:, 2], t.NP[:, 3]])   # (1, ξ, η, ζ) at q
    for cell in range(ne):
        nodes = mesh.el2n[cell] - 1
        ph = case.phases[cell] - 1
        vd = (3 * nodes[:, None] + np.arange(3)[None, :]).ravel()            # vdof(node, i), node-major
        pd = nv + 4 * cell + np.arange(4)
        Ke = np.zeros((81, 81))
        Be = np.zeros((81, 4))
        fe = np.zeros(81)
        for q in range(27):
            geo = mesh.geo_v[cell, q]
            Jinv = geo[:9].reshape(3, 3, order="F")                           # J⁻¹[j, k] = geo[j + 3k]
            dO = geo[9]
            G = t.dN[q] @ Jinv                                                # ∂N_a/∂x_k
            K = (np.einsum("ab,ij->aibj", G @ G.T, I3) + np.einsum("aj,bi->aibj", G, G)
                 - (2.0 / 3.0) * np.einsum("ai,bj->aibj", G, G))
            Ke += eta[ph] * dO * K.reshape(81, 81)
            Be += -dO * np.einsum("ai,p->aip", G, modes[q]).reshape(81, 4)
            fe += dO * np.einsum("a,i->ai", t.N[q], rho[ph] * np.asarray(g)).ravel()
        rr, cc = np.meshgrid(vd, vd, indexing="ij")
        rows += [rr.ravel()]; cols += [cc.ravel()]; vals += [Ke.ravel()]
        rb, cb = np.meshgrid(vd, pd, indexing="ij")
        rows += [rb.ravel(), cb.ravel()]; cols += [cb.ravel(), rb.ravel()]; vals += [Be.ravel(), Be.ravel()]
        np.add.at(rhs, vd, fe)
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(nv + npr, nv + npr))
    fixed = set()
    for c in range(3):
        fixed.update((3 * (case.bc[c][0] - 1) + c).tolist())
    fixed.add(nv)                                                             # pressure gauge
    free = np.array(sorted(set(range(nv + npr)) - fixed))
    return A, rhs, free


@pytest.mark.parametrize("distort", [False, True])
def test_matrix_free_residuals_equal_the_sparse_system(distort):
    case = fem.configs.cell_pressure_case(n=2, seed=7, distort=distort)
    rng = np.random.default_rng(3)
    v = [rng.standard_normal(case.mesh.nnodes) for _ in range(3)]
    P = rng.standard_normal(4 * case.mesh.nels)
    hs = oh.HostCellPressure(case.mesh, case.material.eta, case.material.rho0, case.material.g, case.phases, v, P)
    hs.residuals(3)
    A, rhs, _ = sparse_stokes_reference(case)
    x = np.concatenate([np.stack(v, axis=1).ravel(), P])
    ref = A @ x - rhs
    got = np.concatenate([np.stack(hs.Rv, axis=1).ravel(), hs.RP])
    np.testing.assert_allclose(got, ref, rtol=1e-11, atol=1e-11 * np.abs(ref).max())


def test_preconditioner_is_the_viscous_diagonal_and_mode_mass():
    case = fem.configs.cell_pressure_case(n=2, seed=2, distort=True)
    hs = oh.HostCellPressure(case.mesh, case.material.eta, case.material.rho0, case.material.g, case.phases)
    hs.preconditioner()
    # the diagonal of the sparse viscous block (its rows carry η (|∇N|² + (∂_c N)²/3))
    A, _, _ = sparse_stokes_reference(case)
    d = A.diagonal()[: 3 * case.mesh.nnodes].reshape(-1, 3)
    for c in range(3):
        np.testing.assert_allclose(hs.diagonal[c], d[:, c], rtol=1e-12)
    # mode 1 mass is the cell volume: the cells fill the unit cube
    assert abs(hs.pressure_mass[0::4].sum() - 1.0) < 1e-12


def test_relaxation_converges_to_the_sparse_solution():
    case = fem.configs.cell_pressure_case(n=2, seed=1, distort=True)
    hs = oh.HostCellPressure(case.mesh, case.material.eta, case.material.rho0, case.material.g, case.phases)
    st = hs.solve(case.bc, tolerance=1e-9, max_iterations=60000, check_interval=100)
    assert st.converged and st.iterations % 100 == 0 and st.residual < 1e-9
    A, rhs, free = sparse_stokes_reference(case)
    x = np.zeros(len(rhs))
    x[free] = spla.spsolve(A[free][:, free].tocsc(), rhs[free])
    nv = 3 * case.mesh.nnodes
    v_ref = x[:nv].reshape(-1, 3)
    v = np.stack(hs.v, axis=1)
    assert np.linalg.norm(v - v_ref) <= 1e-5 * np.linalg.norm(v_ref)
    # pressure agrees up to the constant mode
    P, P_ref = hs.P.reshape(-1, 4), x[nv:].reshape(-1, 4)
    np.testing.assert_allclose(P[:, 1:], P_ref[:, 1:], atol=1e-5 * np.abs(P_ref).max())
    d0 = P[:, 0] - P_ref[:, 0]
    assert np.ptp(d0) <= 1e-5 * np.abs(P_ref).max()


def test_non_convergence_is_reported():
    case = fem.configs.cell_pressure_case(n=2, seed=1)
    hs = oh.HostCellPressure(case.mesh, case.material.eta, case.material.rho0, case.material.g, case.phases)
    with pytest.raises(fem._abi.FemB200Error, match="did not converge after 200 iterations"):
        hs.solve(case.bc, tolerance=1e-12, max_iterations=200, check_interval=100)
    st = hs.solve(case.bc, tolerance=1e-12, max_iterations=150, check_interval=100, throw_on_failure=False)
    assert not st.converged and st.reached_total_iter and st.iterations == 150


def test_oracle_adjoint_is_the_transposed_sparse_solve():
    # the adjoint of the symmetric operator is the forward relaxation with the objective
    # as load, no gravity and homogeneous conditions (DR_adjoint.jl:446-484)
    import scipy.sparse.linalg as spla
    case = fem.configs.cell_pressure_case(n=2, seed=4, distort=True)
    nn = case.mesh.nnodes
    rng = np.random.default_rng(2)
    obj = [rng.standard_normal(nn) for _ in range(3)]
    for c in range(3):
        obj[c][case.bc[c][0] - 1] = 0.0
    hs = oh.HostCellPressure(case.mesh, case.material.eta, (0.0,) * len(case.material.eta), (0.0, 0.0, 0.0),
                             case.phases)
    st = hs.solve([(b[0], np.zeros(len(b[0]))) for b in case.bc], tolerance=1e-11, max_iterations=400_000,
                  load=obj)
    assert st.converged
    A, rhs, free = sparse_stokes_reference(case)
    objective = np.concatenate([np.stack(obj, axis=1).ravel(), np.zeros(4 * case.mesh.nels)])
    lam = np.zeros(len(rhs))
    lam[free] = spla.spsolve(A[free][:, free].T.tocsc(), objective[free])
    lv = lam[: 3 * nn].reshape(-1, 3)
    assert np.linalg.norm(np.stack(hs.v, axis=1) - lv) <= 1e-6 * np.linalg.norm(lv)


def test_prescribed_velocities_enter_the_first_residual():
    # test/test_stokes_3d_boundary_values.jl: one Hex27 cell, every boundary node prescribed
    # (vx = x, vy = vz = 0), no gravity; one iteration with a check must not report
    # convergence from the all-zero start, and a start that already carries the prescribed
    # values gives the same first iteration
    mesh = fem.structured_mixed_mesh(3, (1, 1, 1))
    x = mesh.coords
    gamma = np.nonzero(np.any((np.abs(x) < 1e-12) | (np.abs(x - 1.0) < 1e-12), axis=1))[0]
    dofs = (gamma + 1).astype(np.int32)
    vals = [x[gamma, 0].copy(), np.zeros(len(gamma)), np.zeros(len(gamma))]
    bc = [(dofs, vals[c]) for c in range(3)]
    ph = np.ones(1, dtype=np.int32)
    kw = dict(check_interval=1, max_iterations=1)
    hs = oh.HostCellPressure(mesh, (1.0,), (1.0,), (0.0, 0.0, 0.0), ph)
    with pytest.raises(fem._abi.FemB200Error, match="3-D Stokes solve did not converge"):
        hs.solve(bc, **kw)
    hs = oh.HostCellPressure(mesh, (1.0,), (1.0,), (0.0, 0.0, 0.0), ph)
    st = hs.solve(bc, throw_on_failure=False, **kw)
    assert not st.converged and st.reached_total_iter and st.err_P > 1e-5
    for c in range(3):
        assert (hs.v[c][gamma] == vals[c]).all()
    v0 = [np.zeros(mesh.nnodes) for _ in range(3)]
    for c in range(3):
        v0[c][gamma] = vals[c]
    hc = oh.HostCellPressure(mesh, (1.0,), (1.0,), (0.0, 0.0, 0.0), ph, v=v0)
    stc = hc.solve(bc, throw_on_failure=False, **kw)
    assert stc.err_P == pytest.approx(st.err_P, rel=1e-14)
    np.testing.assert_allclose(hc.P, hs.P, rtol=1e-14, atol=1e-300)
    for c in range(3):
        np.testing.assert_allclose(hc.v[c], hs.v[c], rtol=1e-14, atol=1e-300)
