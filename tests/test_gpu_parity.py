"""Parity of libfemtools_b200 (through its C ABI) against the CPU oracle.

Element sweeps are compared entry by entry; in FP64 the only differences are
summation order (atomic scatter, sum-factorised contractions), so the bound is
|gpu − oracle| ≤ 1e-10·|oracle| + 1e-11·max|oracle|. Full DR solves must take the
same number of iterations and agree to 1e-8 relative on v, P and τ.
"""
import math

import numpy as np
import pytest

import oracle_host as oh
from cases import inclusion_2d_case, random_state_case, vep_layers_case
from conftest import fem

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
abi = fem._abi


def close(gpu, ref, rtol=1e-10, atol_rel=1e-11, what=""):
    g = gpu.detach().cpu().numpy() if hasattr(gpu, "detach") else np.asarray(gpu)
    scale = max(np.abs(ref).max(), 1e-300)
    np.testing.assert_allclose(g, ref, rtol=rtol, atol=atol_rel * scale, err_msg=what)


LAYOUTS = ["nodal", "cell", "element"]


@pytest.mark.parametrize("dim", [3, 2])
@pytest.mark.parametrize("phases", LAYOUTS)
def test_pressure_residual(dim, phases):
    case = random_state_case(dim=dim, n=3, seed=11, phases=phases)
    dr, hs = case.device_state(fem), case.host_state(oh)
    for finite_K in (False, True):
        fem.assemble_pressure_residual(dr, case.dt, finite_K=finite_K)
        hs.pressure_residual(case.dt, finite_K=finite_K)
        close(dr.RP, hs.RP, what=f"RP finite_K={finite_K}")


@pytest.mark.parametrize("dim", [3, 2])
@pytest.mark.parametrize("phases", LAYOUTS)
@pytest.mark.parametrize("plastic", [False, True])
def test_momentum_residual(dim, phases, plastic):
    case = random_state_case(dim=dim, n=3, seed=5, phases=phases, plastic=plastic)
    dr, hs = case.device_state(fem), case.host_state(oh)
    for with_pnum in (False, True):
        fem.assemble_momentum_residual(dr, case.dt, with_pnum=with_pnum)
        hs.momentum_residual(case.dt, with_pnum=with_pnum)
        for c in range(dim):
            close(dr.Rv[c], hs.Rv[c], what=f"Rv[{c}] pnum={with_pnum}")


@pytest.mark.parametrize("phases", LAYOUTS)
@pytest.mark.parametrize("plastic", [False, True])
def test_pipelined_sweep_on_affine_mesh(phases, plastic):
    # Affine cells take the pipelined sweep with one J⁻¹ per element.
    case = random_state_case(dim=3, n=4, seed=13, phases=phases, plastic=plastic, distort=False)
    dr, hs = case.device_state(fem), case.host_state(oh)
    fem.assemble_stokes_residuals(dr, case.dt)
    hs.stokes_residuals(case.dt)
    close(dr.RP, hs.RP, what="RP")
    close(dr.Pnum, hs.Pnum, what="Pnum")
    for c in range(3):
        close(dr.Rv[c], hs.Rv[c], what=f"Rv[{c}]")
    fem.update_stokes_current_stress(dr, case.dt)
    hs.store_stress(case.dt)
    for c in range(6):
        close(dr.tau[c], hs.tau[c], what=f"τ[{c}]")


@pytest.mark.parametrize("dim", [3, 2])
def test_fused_residual_sweep(dim):
    case = random_state_case(dim=dim, n=4, seed=2, phases="cell")
    dr, hs = case.device_state(fem), case.host_state(oh)
    fem.assemble_stokes_residuals(dr, case.dt)
    hs.stokes_residuals(case.dt)
    close(dr.RP, hs.RP, what="RP")
    close(dr.Pnum, hs.Pnum, what="Pnum")
    for c in range(dim):
        close(dr.Rv[c], hs.Rv[c], what=f"Rv[{c}]")


@pytest.mark.parametrize("dim", [3, 2])
@pytest.mark.parametrize("plastic", [False, True])
@pytest.mark.parametrize("phases", ["nodal", "cell"])
def test_jacobian_diagnostics(dim, plastic, phases):
    case = random_state_case(dim=dim, n=2, seed=8, phases=phases, plastic=plastic)
    dr, hs = case.device_state(fem), case.host_state(oh)
    fem.assemble_augmented_momentum_jacobian(dr, case.dt)
    hs.jacobian_diagnostics(case.dt)
    for c in range(dim):
        close(dr.dRdv[c], hs.dRdv[c], rtol=1e-9, what=f"dRdv[{c}]")
        close(dr.PC[c], hs.PC[c], rtol=1e-9, what=f"PC[{c}]")


@pytest.mark.parametrize("plastic", [False, True])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_jacobian_diagnostics_on_axis_aligned_cells(plastic, precision):
    # a box mesh: every J⁻¹ is diagonal and the library takes its diagonal-geometry kernel
    case = random_state_case(dim=3, n=3, seed=9, phases="cell", plastic=plastic, distort=False)
    straight = fem.structured_mixed_mesh(3, (3, 3, 3), hi=(1.0, 2.0, 0.5))
    case.mesh.coords, case.mesh.geo_v, case.mesh.geo_P = straight.coords, straight.geo_v, straight.geo_P
    dt_ = torch.float64 if precision == "fp64" else torch.float32
    dr, hs = case.device_state(fem, dtype=dt_, geometry_dtype=dt_), case.host_state(oh)
    fem.assemble_augmented_momentum_jacobian(dr, case.dt)
    hs.jacobian_diagnostics(case.dt)
    tol = 1e-9 if precision == "fp64" else 2e-5
    for c in range(3):
        close(dr.dRdv[c], hs.dRdv[c], rtol=tol, atol_rel=tol, what=f"dRdv[{c}]")
        close(dr.PC[c], hs.PC[c], rtol=tol, atol_rel=tol, what=f"PC[{c}]")


@pytest.mark.parametrize("dim", [3, 2])
@pytest.mark.parametrize("finite_K", [False, True])
def test_pressure_scaling(dim, finite_K):
    case = random_state_case(dim=dim, n=3, seed=4, phases="nodal")
    dr, hs = case.device_state(fem), case.host_state(oh)
    fem.assemble_viscosity_weighted_pressure_scaling(dr, 50.0, case.dt, finite_K=finite_K)
    hs.pressure_scaling(50.0, case.dt, finite_K=finite_K)
    close(dr.M_P, hs.M_P, what="M_P")
    close(dr.gammaP, hs.gammaP, what="γP")


@pytest.mark.parametrize("dim", [3, 2])
def test_stress_store_and_shear_heating(dim):
    case = random_state_case(dim=dim, n=3, seed=9, phases="element")
    dr, hs = case.device_state(fem), case.host_state(oh)
    fem.update_stokes_current_stress(dr, case.dt)
    hs.store_stress(case.dt)
    for c in range(len(hs.tau)):
        close(dr.tau[c], hs.tau[c], what=f"τ[{c}]")
    phi = fem.assemble_shear_heating(dr, case.dt)
    close(phi, hs.shear_heating(case.dt), what="Φ")


def test_vep_solve_matches_oracle_step_by_step():
    # Three time steps of the 3-D visco-elasto-plastic layered problem, each to 1e-8,
    # with P0 ← P and τ_old ← τ between steps (the time-step driver of the examples).
    case = vep_layers_case(n=3, seed=1)
    dr, hs = case.device_state(fem), case.host_state(oh)
    bc = case.bc_device()
    for step in range(3):
        st = fem.solve(dr, bc, dt=case.dt, tolerance=1e-8, check_interval=50, throw_on_failure=False)
        ref = hs.solve(dt=case.dt, tolerance=1e-8, check_interval=50, throw_on_failure=False)
        assert st["converged"] and ref["converged"]
        assert st["iter"] == ref["iter"], (step, st["iter"], ref["iter"])
        assert st["itPH"] == ref["itPH"]
        for c in range(3):
            close(dr.v[c], hs.v[c], rtol=1e-8, atol_rel=1e-9, what=f"step {step} v[{c}]")
        close(dr.P, hs.P, rtol=1e-8, atol_rel=1e-9, what=f"step {step} P")
        fem.update_stokes_current_stress(dr, case.dt)
        hs.store_stress(case.dt)
        for c in range(6):
            close(dr.tau[c], hs.tau[c], rtol=1e-8, atol_rel=1e-9, what=f"step {step} τ[{c}]")
            dr.tau_old[c].copy_(dr.tau[c])
            hs.tau_old[c][:] = hs.tau[c]
        dr.P0.copy_(dr.P)
        hs.P0[:] = hs.P


def test_2d_inclusion_solve_matches_oracle():
    # The incompressible 1e3-contrast inclusion needs ~1e5 DR iterations at 8² cells.
    case = inclusion_2d_case(n=8)
    dr, hs = case.device_state(fem), case.host_state(oh)
    kw = dict(tolerance=1e-8, check_interval=50, max_iterations=200_000, iter_max=200_000)
    st = fem.solve(dr, case.bc_device(), dt=case.dt, **kw)
    ref = hs.solve(dt=case.dt, **kw)
    # Over ~1e5 iterations the atomic summation order shifts the trajectory by a few
    # checks; both runs converge to the same solution within the solve tolerance.
    assert st["converged"] and ref["converged"]
    assert abs(st["iter"] - ref["iter"]) <= 0.05 * ref["iter"]
    for c in range(2):
        close(dr.v[c], hs.v[c], rtol=1e-5, atol_rel=1e-6)
    close(dr.P, hs.P, rtol=1e-5, atol_rel=1e-6)


def test_q9_hydrostatic_known_answer_on_gpu():
    # test/test_stokes_quadrature_viscosity.jl:89-116, through the device solver.
    mesh = fem.structured_mixed_mesh(2, (2, 2))
    mat = fem.StokesMaterial(eta=(2.0,), eta_b=(math.inf,), G=(math.inf,), alpha=(0.0,), g=(0.0, 1.0))
    dr = fem.StokesDR(mesh, mat, stress=False)
    fem.assemble_viscosity_weighted_pressure_scaling(dr, 50.0, 1.0)
    np.testing.assert_allclose(dr.gammaP.cpu().numpy(), 50.0, rtol=1e-12)
    nodes = mesh.boundary_nodes
    bc = [fem.DirichletBoundaryCondition(nodes, np.zeros(len(nodes)))] * 2
    st = fem.solve_stokes_dyrel(dr, bc, 1.0, ncheck=10, eps_tol=1e-11, history_capacity=10000)
    assert st["converged"]
    assert st["history"][0, 0] == 0 and st["history"][-1, 0] == st["iter"]
    y = mesh.coords[mesh.el2nP.ravel() - 1, 1]
    diff = dr.P.cpu().numpy() - y
    assert diff.max() - diff.min() < 1e-7
    assert torch.linalg.norm(dr.v[0]).item() + torch.linalg.norm(dr.v[1]).item() < 1e-7


def test_solver_error_paths():
    # A budget too small to converge raises with the reference's message; a zero
    # preconditioner is reported as an invalid λmax (utils.jl:152-158).
    case = vep_layers_case(n=2, seed=0)
    dr = case.device_state(fem)
    with pytest.raises(abi.FemB200Error, match="Stokes solve did not converge"):
        fem.solve(dr, case.bc_device(), dt=case.dt, tolerance=1e-12, max_iterations=2, check_interval=1)
    dr = case.device_state(fem)
    st = fem.solve(dr, case.bc_device(), dt=case.dt, tolerance=1e-12, max_iterations=2, check_interval=1,
                   throw_on_failure=False)
    assert not st["converged"] and st["reached_total_iter"]
    bad = vep_layers_case(n=2, seed=0)
    bad.material = fem.StokesMaterial(eta=(0.0,) * 3, G=(1.0,) * 3, g=(0.0, 0.0, -1.0))
    dr = bad.device_state(fem)
    with pytest.raises(abi.FemB200Error, match="invalid λmax"):
        fem.solve(dr, bad.bc_device(), dt=bad.dt)


@pytest.mark.parametrize("dim", [3, 2])
def test_thermal_solve_matches_oracle(dim):
    mesh = fem.structured_mixed_mesh(dim, (3,) * dim)
    rng = np.random.default_rng(3)
    kw = dict(k=(1.0, 2.5), Cp=(1.0, 1.3), rho0=(1.0, 1.2), alpha=(0.05, 0.02), K=(50.0, 80.0))
    ph = rng.integers(1, 3, mesh.nnodes).astype(np.int32)
    th = fem.ThermalDiffusionDR(mesh, phases=ph, eps=1e-9, **kw)
    ht = oh.HostThermal(mesh, phases=ph, eps=1e-9, **kw)
    T0 = rng.uniform(0, 1, mesh.nnodes)
    th.T0.copy_(torch.as_tensor(T0)); ht.T0[:] = T0
    th.T.copy_(torch.as_tensor(T0)); ht.T[:] = T0
    src = rng.uniform(0, 1, mesh.nnodes)
    th.source.copy_(torch.as_tensor(src)); ht.source[:] = src
    b = mesh.boundary_nodes
    bc = fem.DirichletBoundaryCondition(b, np.zeros(len(b)))
    ht.set_bc(b, np.zeros(len(b)))
    fem.assemble_thermal_residual(th, 0.1, 0.3, compute_jacobian=True)
    ht.residual(0.1, 0.3, jac=True)
    close(th.R, ht.R, what="R")
    close(th.dRdT, ht.dRdT, rtol=1e-9, what="∂R∂T")
    close(th.PC, ht.PC, rtol=1e-9, what="PC")
    st = fem.solve_thermal(th, bc, 0.1, Tref=0.3, check_interval=20)
    ref = ht.solve(0.1, Tref=0.3, check_interval=20)
    assert st["iterations"] == ref["iterations"]
    close(th.T, ht.T, rtol=1e-9)


def test_coupled_shear_heating_closed_form_on_gpu():
    # test/test_coupled_solver.jl:67-120 on a Hex27 mesh: T = Δt(ηve γ̇)²/η.
    dt, eta, G, gd = 0.5, 2.0, 1.0, 1.0
    etave = 1 / (1 / eta + 1 / (G * dt))
    T_expected = dt * (etave * gd) ** 2 / eta
    mesh = fem.structured_mixed_mesh(3, (2, 2, 2))
    c = mesh.coords
    nodes = mesh.boundary_nodes
    th = fem.ThermalDiffusionDR(mesh, eps=1e-10)
    sk = fem.StokesDR(mesh, fem.StokesMaterial(eta=(eta,), eta_b=(1.0,), G=(G,), alpha=(0.0,), g=(0.0, 0.0, 0.0)))
    sk.v[0].copy_(torch.as_tensor(gd * c[:, 1] + 0.1 * np.sin(np.pi * c[:, 0]) * np.sin(np.pi * c[:, 1])))
    bc_v = [fem.DirichletBoundaryCondition(nodes, gd * c[nodes - 1, 1])] + \
           [fem.DirichletBoundaryCondition(nodes, np.zeros(len(nodes)))] * 2
    bc_T = fem.DirichletBoundaryCondition(nodes, np.full(len(nodes), T_expected))
    st, _ = fem.solve_coupled(th, sk, bc_T, bc_v, dt, shear_heating=True, pressure_factor=1.0, check_interval=10,
                              iter_max=20_000, max_iterations=20_000, tolerance=1e-10)
    assert st["converged"]
    np.testing.assert_allclose(th.T.cpu().numpy(), T_expected, atol=1e-8)
    # and the coupled trajectory equals the oracle's
    ht = oh.HostThermal(mesh, eps=1e-10)
    hs = oh.HostStokes(mesh, fem.StokesMaterial(eta=(eta,), eta_b=(1.0,), G=(G,), alpha=(0.0,), g=(0.0, 0.0, 0.0)))
    hs.v[0][:] = gd * c[:, 1] + 0.1 * np.sin(np.pi * c[:, 0]) * np.sin(np.pi * c[:, 1])
    hs.set_bc([(nodes, gd * c[nodes - 1, 1]), (nodes, np.zeros(len(nodes))), (nodes, np.zeros(len(nodes)))])
    ht.set_bc(nodes, np.full(len(nodes), T_expected))
    ref, _ = oh.solve_coupled(ht, hs, shear_heating=True, dt=dt, pressure_factor=1.0, check_interval=10,
                              iter_max=20_000, max_iterations=20_000, tolerance=1e-10)
    assert st["iter"] == ref["iter"]
    assert st["thermal_iterations"] == ref["thermal_iterations"]


def test_fp32_state_tracks_fp64_oracle():
    # The reference's whole-solve Float32 states (stokes_types.jl:109): FP32 sweeps on
    # FP32 state, compared with the FP64 oracle at FP32 tolerance.
    case = random_state_case(dim=3, n=3, seed=21, phases="cell")
    dr = case.device_state(fem, dtype=torch.float32)
    hs = case.host_state(oh)
    fem.assemble_stokes_residuals(dr, case.dt)
    hs.stokes_residuals(case.dt)
    for c in range(3):
        close(dr.Rv[c].double(), hs.Rv[c], rtol=5e-4, atol_rel=5e-5, what=f"FP32 Rv[{c}]")
    close(dr.RP.double(), hs.RP, rtol=5e-4, atol_rel=5e-5, what="FP32 RP")


@pytest.mark.parametrize("dim", [3, 2])
def test_colored_thermal_assembly_matches_atomic(dim):
    # assemble_diffusion_matrices_colored! vs the atomic assembler (test/test_assembler_api.jl:8-60),
    # on a mesh with mixed phases, and against the oracle.
    mesh = fem.structured_mixed_mesh(dim, (4,) * dim)
    rng = np.random.default_rng(9)
    kw = dict(k=(1.0, 2.5), Cp=(1.0, 1.3), rho0=(1.0, 1.2), alpha=(0.05, 0.02), K=(50.0, 80.0))
    ph = rng.integers(1, 3, mesh.nnodes).astype(np.int32)
    th = fem.ThermalDiffusionDR(mesh, phases=ph, **kw)
    ht = oh.HostThermal(mesh, phases=ph, **kw)
    for name in ("T", "T0", "source"):
        x = rng.uniform(0, 1, mesh.nnodes)
        getattr(th, name).copy_(torch.as_tensor(x))
        getattr(ht, name)[:] = x
    groups = fem.generate_element_groups(fem.color_mesh(mesh))
    fem.assemble_thermal_residual(th, 0.1, 0.3, compute_jacobian=True)
    atomic = [x.clone() for x in (th.R, th.dRdT, th.PC)]
    fem.assemble_diffusion_matrices_colored(th, groups, 0.1, 0.3, compute_jacobian=True)
    ht.residual(0.1, 0.3, jac=True)
    for got, ref, host, what in zip((th.R, th.dRdT, th.PC), atomic, (ht.R, ht.dRdT, ht.PC), ("R", "∂R∂T", "PC")):
        close(got, ref.cpu().numpy(), rtol=1e-12, atol_rel=1e-14, what=what + " colored vs atomic")
        close(got, host, rtol=1e-9, what=what + " colored vs oracle")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("where", ["tau_old", "vy"])
def test_nan_input_raises_the_reference_nan_exit(precision, where):
    # src/stokes/solvers/DR.jl:570-575: Julia's max / min carry a NaN residual into
    # isnan(err); a NaN in one velocity component or one stress-history point must not
    # be hidden by the max over components. The oracle raises the same message.
    case = vep_layers_case(n=2, seed=0)
    dr, hs = case.device_state(fem), case.host_state(oh)
    if where == "tau_old":
        dr.tau_old[0][5] = float("nan")
        hs.tau_old[0][5] = np.nan
    else:
        interior = np.setdiff1d(np.arange(1, case.mesh.nnodes + 1), case.mesh.boundary_nodes)
        dr.v[1][int(interior[0]) - 1] = float("nan")
        hs.v[1][interior[0] - 1] = np.nan
    kw = dict(dt=case.dt, tolerance=1e-8, check_interval=50, throw_on_failure=False)
    with pytest.raises(abi.FemB200Error) as ref:
        hs.solve(**kw)
    with pytest.raises(abi.FemB200Error) as got:
        fem.solve(dr, case.bc_device(), precision=precision, **kw)
    assert got.value.code == ref.value.code == abi.ENAN
    assert str(got.value) == str(ref.value) == "NaN detected in outer loop at PH=1"


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_unstable_pseudo_time_step_raises_kaboom(precision):
    # DR.jl:711-712: a CFL far above the stability limit grows the velocity error past
    # 1e10 by the first check; the oracle stops at the same check with the same message.
    case = vep_layers_case(n=2, seed=0)
    dr, hs = case.device_state(fem), case.host_state(oh)
    kw = dict(dt=case.dt, tolerance=1e-8, check_interval=50, throw_on_failure=False, cfl_v=4.0)
    with pytest.raises(abi.FemB200Error) as ref:
        hs.solve(**kw)
    with pytest.raises(abi.FemB200Error) as got:
        fem.solve(dr, case.bc_device(), precision=precision, **kw)
    assert got.value.code == ref.value.code == abi.EKABOOM
    assert str(ref.value) == "Kaboom! Error > 1e10 in inner loop PH=1 PT=50"
    if precision == "fp64":
        assert str(got.value) == str(ref.value)
    else:
        assert str(got.value).startswith("Kaboom! Error > 1e10 in inner loop PH=1 PT=")
