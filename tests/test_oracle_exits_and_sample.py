"""The oracle's failure exits and the CPU-sample entry points the benchmark times.

Failure exits (src/stokes/solvers/DR.jl:570-575, :700-712, :1041-1044): the reference
forms its errors with Julia's max / min / maximum, which return NaN when any
argument is NaN, so a NaN anywhere in the residual reaches `isnan(err)` and raises
"NaN detected in outer loop at PH=…"; a pseudo-time step above the stability limit
grows the error past 1e10 and raises "Kaboom! Error > 1e10 in inner loop PH=… PT=…".

CPU sample: `orc_dr_iterations` must run exactly the solve's own inner iteration
and `orc_jacobian_range` the solve's Jacobian assembly restricted to a block of
elements, so that the timed reference figure prices the solve's real work.
"""
import math

import numpy as np
import pytest

import oracle_host as oh
from cases import vep_layers_case
from conftest import fem

abi = fem._abi


def _solve(hs, case, **kw):
    return hs.solve(dt=case.dt, tolerance=1e-8, check_interval=50, throw_on_failure=False, **kw)


def test_nan_in_the_stress_history_raises_the_reference_nan_exit():
    case = vep_layers_case(n=2, seed=0)
    hs = case.host_state(oh)
    hs.tau_old[0][5] = np.nan
    with pytest.raises(abi.FemB200Error) as e:
        _solve(hs, case)
    assert e.value.code == abi.ENAN
    assert str(e.value) == "NaN detected in outer loop at PH=1"


def test_nan_in_one_velocity_component_is_not_hidden_by_the_max_over_components():
    # maximum(norm, Rv) over (vx, vy, vz): a NaN in vy alone must still raise
    case = vep_layers_case(n=2, seed=0)
    hs = case.host_state(oh)
    interior = np.setdiff1d(np.arange(1, case.mesh.nnodes + 1), case.mesh.boundary_nodes)
    hs.v[1][interior[0] - 1] = np.nan
    with pytest.raises(abi.FemB200Error) as e:
        _solve(hs, case)
    assert e.value.code == abi.ENAN
    assert str(e.value) == "NaN detected in outer loop at PH=1"


def test_unstable_pseudo_time_step_raises_kaboom():
    case = vep_layers_case(n=2, seed=0)
    hs = case.host_state(oh)
    with pytest.raises(abi.FemB200Error) as e:
        _solve(hs, case, cfl_v=4.0)
    assert e.value.code == abi.EKABOOM
    assert str(e.value) == "Kaboom! Error > 1e10 in inner loop PH=1 PT=50"


def test_cell_pressure_nan_velocity_raises_the_non_finite_exit():
    case = fem.configs.cell_pressure_case(n=2, seed=1)
    hs = oh.HostCellPressure(case.mesh, case.material.eta, case.material.rho0, case.material.g, case.phases)
    node = int(np.setdiff1d(np.arange(1, case.mesh.nnodes + 1), case.mesh.boundary_nodes)[0]) - 1
    hs.v[1][node] = np.nan
    with pytest.raises(abi.FemB200Error) as e:
        hs.solve(case.bc, tolerance=1e-8, max_iterations=1000, check_interval=100)
    assert e.value.code == abi.ENONFINITE
    assert str(e.value) == "non-finite residual in 3-D Stokes solve"


def test_sample_iteration_is_the_solves_first_iteration():
    # the solve with max_iterations = 0 runs M_P/γP, the Jacobian, the outer residual,
    # one inner iteration (Chebyshev steps from λmax with λmin = 0) and the PH update
    case = vep_layers_case(n=3, seed=2)
    a, b = case.host_state(oh), case.host_state(oh)
    _solve(a, case, max_iterations=0)
    b.pressure_scaling(50.0, case.dt)
    b.jacobian_diagnostics(case.dt)
    lmax = [float(np.max(b.dRdv[c] / b.PC[c])) for c in range(3)]
    dtau = [2.0 / math.sqrt(x) * 0.98 for x in lmax]
    b.dr_iterations(case.dt, [d * d for d in dtau], [1.0] * 3, 1)
    for c in range(3):
        np.testing.assert_array_equal(a.v[c], b.v[c])
        np.testing.assert_array_equal(a.Rv[c], b.Rv[c])


def test_sample_check_gives_the_solves_velocity_error():
    case = vep_layers_case(n=2, seed=1)
    hs = case.host_state(oh)
    hs.pressure_scaling(50.0, case.dt)
    hs.jacobian_diagnostics(case.dt)
    ev = hs.dr_iterations(case.dt, [1e-3] * 3, [0.9] * 3, 3, check_norms=True)
    want = max(np.linalg.norm(hs.Rv[c]) for c in range(3)) / (2 * math.sqrt(case.mesh.nnodes))
    assert ev == pytest.approx(want, rel=1e-14)


def test_jacobian_by_blocks_sums_to_the_full_assembly():
    case = vep_layers_case(n=3, seed=4)
    hs = case.host_state(oh)
    hs.pressure_scaling(50.0, case.dt)
    hs.jacobian_diagnostics(case.dt)
    full = [(hs.dRdv[c].copy(), hs.PC[c].copy()) for c in range(3)]
    acc = [(np.zeros_like(x), np.zeros_like(y)) for x, y in full]
    cuts = [0, 7, 20, case.mesh.nels]
    for e0, e1 in zip(cuts[:-1], cuts[1:]):
        hs.jacobian_range(case.dt, e0, e1)
        for c in range(3):
            acc[c][0][:] += hs.dRdv[c]
            acc[c][1][:] += hs.PC[c]
    for c in range(3):
        np.testing.assert_allclose(acc[c][0], full[c][0], rtol=1e-13, atol=0)
        np.testing.assert_allclose(acc[c][1], full[c][1], rtol=1e-13, atol=0)
    with pytest.raises(abi.FemB200Error, match="element range"):
        hs.jacobian_range(case.dt, 0, case.mesh.nels + 1)
