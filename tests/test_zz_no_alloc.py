"""femb200_solve_thermal_noalloc, the allocation-free thermal DR solve, against
femb200_solve_thermal on the same inputs, through the C ABI.

The entry point exists for hosts whose device memory belongs to their own pool
(Julia's CUDA.jl pool, PyTorch's caching allocator) or that cannot take the
device-wide synchronisation of cudaFree: it must produce the regular solve's
answer without allocating. The parity test therefore runs it on a handle of its
own, made for the test, and checks that the device's free memory is the same
before and after two calls in a row (cudaMalloc takes memory in steps of at least
2 MB, so any allocation would show).

This file is collected last on purpose: it must pass in a fresh process (the
first call on a handle then looks up the fixed scratch array) and after every
other test (the array then holds whatever earlier calls left in it).
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


def _state(mesh, seed, bc):
    rng = np.random.default_rng(seed)
    kw = dict(k=(1.0, 2.5), Cp=(1.0, 1.3), rho0=(1.0, 1.2), alpha=(0.05, 0.02), K=(50.0, 80.0))
    ph = rng.integers(1, 3, mesh.nnodes).astype(np.int32)
    th = fem.ThermalDiffusionDR(mesh, phases=ph, eps=1e-9, **kw)
    T0 = torch.as_tensor(rng.uniform(0, 1, mesh.nnodes))
    th.T0.copy_(T0)
    th.T.copy_(T0)
    th.source.copy_(torch.as_tensor(rng.uniform(0, 1, mesh.nnodes)))
    th.set_bc(bc)
    return th


def _controls(th, dt, Tref, check_interval):
    c = abi.ThermalControlsC()
    c.dt, c.Tref, c.tolerance = dt, Tref, th.eps
    c.max_iterations, c.check_interval, c.throw_on_failure = 10_000, check_interval, 1
    return c


def _solve_noalloc(lib, h, problem, controls):
    st = abi.ThermalStatsC()
    rc = lib.femb200_solve_thermal_noalloc(h, C.byref(problem), C.byref(controls), C.byref(st))
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
    dt, Tref, ncheck = 0.1, 0.3, 20

    # the regular solve, on the shared handle
    refs, ref_T = [], []
    for bc in bcs:
        th_ref = _state(mesh, 5, bc)
        refs.append(fem.solve_thermal(th_ref, bc, dt, Tref=Tref, check_interval=ncheck))
        ref_T.append(th_ref.T.clone())
    # every device array of the two calls exists before the memory is read
    states = [_state(mesh, 5, bc) for bc in bcs]
    problems = [th.problem() for th in states]
    controls = [_controls(th, dt, Tref, ncheck) for th in states]

    # one call on the shared handle first: under CUDA's lazy loading a kernel's
    # first launch may load its code into device memory, which is the driver's
    # doing, not the entry point's
    lib, shared = fem.solver._Handle.get()
    warm = _solve_noalloc(lib, shared, problems[0], controls[0])
    assert warm["iterations"] == refs[0]["iterations"], (warm, refs[0])
    states[0].T.copy_(states[0].T0)

    h = C.c_void_p()
    assert lib.femb200_create(C.byref(h)) == abi.OK
    try:
        assert lib.femb200_set_stream(h, C.c_void_p(torch.cuda.current_stream().cuda_stream)) == abi.OK
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        got = [_solve_noalloc(lib, h, problems[k], controls[k]) for k in range(2)]
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
    finally:
        lib.femb200_destroy(h)
    assert free_after == free_before, (free_before, free_after)
    for call in range(2):
        g, r = got[call], refs[call]
        assert g["converged"] and r["converged"], (call, g, r)
        assert g["iterations"] == r["iterations"], (call, g, r)
        assert abs(g["residual"] - r["residual"]) <= 1e-6 * r["residual"] + 1e-15, (call, g, r)
        _close(states[call].T, ref_T[call], f"T, call {call + 1}")


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
