"""femb200_solve_thermal_noalloc, the allocation-free thermal DR solve, against
femb200_solve_thermal on the same inputs, through the C ABI.

This file is collected last on purpose: it must pass in a fresh process (its
first call then does the per-device set-up of the fixed scratch array) and after
every other test (the array then holds whatever earlier calls left in it).
"""
import ctypes as C

import numpy as np
import pytest

from conftest import fem

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
abi = fem._abi

# tolerance of the thermal parity tests: FP64, atomic scatter order only
RTOL, ATOL_REL = 1e-9, 1e-11


def _state(mesh, seed):
    rng = np.random.default_rng(seed)
    kw = dict(k=(1.0, 2.5), Cp=(1.0, 1.3), rho0=(1.0, 1.2), alpha=(0.05, 0.02), K=(50.0, 80.0))
    ph = rng.integers(1, 3, mesh.nnodes).astype(np.int32)
    th = fem.ThermalDiffusionDR(mesh, phases=ph, eps=1e-9, **kw)
    T0 = torch.as_tensor(rng.uniform(0, 1, mesh.nnodes))
    th.T0.copy_(T0)
    th.T.copy_(T0)
    th.source.copy_(torch.as_tensor(rng.uniform(0, 1, mesh.nnodes)))
    return th


def _solve_noalloc(th, bc, dt, Tref, check_interval):
    lib, h = fem.solver._Handle.get()
    th.set_bc(bc)
    c = abi.ThermalControlsC()
    c.dt, c.Tref, c.tolerance = dt, Tref, th.eps
    c.max_iterations, c.check_interval, c.throw_on_failure = 10_000, check_interval, 1
    st = abi.ThermalStatsC()
    rc = lib.femb200_solve_thermal_noalloc(h, C.byref(th.problem()), C.byref(c), C.byref(st))
    if rc != abi.OK:
        raise abi.FemB200Error(rc, lib.femb200_last_error(h).decode())
    return {"converged": bool(st.converged), "iterations": st.iterations, "residual": st.residual}


def _close(a, b, what):
    a, b = a.cpu().numpy(), b.cpu().numpy()
    np.testing.assert_allclose(a, b, rtol=RTOL, atol=ATOL_REL * np.abs(b).max(), err_msg=what)


@pytest.mark.parametrize("dim", [3, 2])
def test_noalloc_matches_solve_thermal_on_two_calls(dim):
    mesh = fem.structured_mixed_mesh(dim, (4,) * dim)
    all_walls = mesh.boundary_nodes
    # second call: fewer constrained nodes, so mask bits left by the first call would show
    z = mesh.coords[:, dim - 1]
    floor_roof = np.flatnonzero((np.abs(z - z.min()) < 1e-12) | (np.abs(z - z.max()) < 1e-12)) + 1
    bcs = [fem.DirichletBoundaryCondition(all_walls, np.zeros(len(all_walls))),
           fem.DirichletBoundaryCondition(floor_roof, np.full(len(floor_roof), 0.25))]
    th = _state(mesh, seed=5)
    th_ref = _state(mesh, seed=5)
    for call, bc in enumerate(bcs):
        th.T.copy_(th.T0)
        th_ref.T.copy_(th_ref.T0)
        got = _solve_noalloc(th, bc, 0.1, 0.3, 20)
        ref = fem.solve_thermal(th_ref, bc, 0.1, Tref=0.3, check_interval=20)
        torch.cuda.synchronize()
        assert got["converged"] and ref["converged"], (call, got, ref)
        assert got["iterations"] == ref["iterations"], (call, got, ref)
        assert abs(got["residual"] - ref["residual"]) <= 1e-6 * ref["residual"] + 1e-15, (call, got, ref)
        _close(th.T, th_ref.T, f"T, call {call + 1}")


def test_noalloc_rejects_meshes_above_the_scratch_size():
    lib, h = fem.solver._Handle.get()
    t = abi.ThermalProblemC()
    t.dim, t.dtype, t.geo_dtype = 3, abi.F64, abi.F64
    t.nnodes = abi.NOALLOC_MAX_NODES + 1
    c = abi.ThermalControlsC()
    c.max_iterations, c.check_interval = 1, 1
    st = abi.ThermalStatsC()
    rc = lib.femb200_solve_thermal_noalloc(h, C.byref(t), C.byref(c), C.byref(st))
    assert rc == abi.EINVAL
    assert str(abi.NOALLOC_MAX_NODES) in lib.femb200_last_error(h).decode()
