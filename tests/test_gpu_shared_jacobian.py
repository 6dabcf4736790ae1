"""Shared elastic element Jacobians in the Hex27 Jacobian diagnostics
(assemble_augmented_momentum_jacobian_matrices_atomix!, momentum_residuals.jl:998-1117).

In the FP32 diagnostics of the mixed-precision solve, with one phase per cell, the
library computes the diagnostics of one element per phase from its elastic
linearisation and lets every element that is elastic at the current state and has the
same inputs within 4e-7 relative (geometry, γP, M_P, η_pc, phase) take that element's
rows instead of its own 81 columns. The assembly must then equal the one without
sharing (a handle created with FEMB200_JAC_SHARED=0) to FP32 rounding, and the oracle
within the FP32 parity tolerance. FP64 diagnostics never share."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle_host as oh
from cases import vep_layers_case
from conftest import fem

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
abi = fem._abi


def _full_handle():
    lib = abi.load_library()
    os.environ["FEMB200_JAC_SHARED"] = "0"
    try:
        h = C.c_void_p()
        assert lib.femb200_create(C.byref(h)) == abi.OK
    finally:
        del os.environ["FEMB200_JAC_SHARED"]
    assert lib.femb200_set_stream(h, C.c_void_p(torch.cuda.current_stream().cuda_stream)) == abi.OK
    return lib, h


def _case(seed, copy_geometry):
    case = vep_layers_case(n=4, seed=seed)
    if copy_geometry:
        # every cell carries the first cell's geometry bit for bit (what a generator that
        # forms J from coordinate differences gives a uniform box)
        m = case.mesh
        m.geo_v = np.ascontiguousarray(np.broadcast_to(m.geo_v[:1], m.geo_v.shape))
        m.geo_P = np.ascontiguousarray(np.broadcast_to(m.geo_P[:1], m.geo_P.shape))
    return case


@pytest.mark.parametrize("precision,copy_geometry", [("fp64", False), ("fp32", False), ("fp32", True)])
@pytest.mark.parametrize("seed", [0, 4])
def test_shared_jacobians_equal_the_full_assembly(precision, copy_geometry, seed):
    case = _case(seed, copy_geometry)
    tdt = torch.float64 if precision == "fp64" else torch.float32
    dr = case.device_state(fem, dtype=tdt, geometry_dtype=tdt)
    fem.assemble_viscosity_weighted_pressure_scaling(dr, 50.0, case.dt)
    lib, h = fem.solver._Handle.get()
    lib.femb200_profile(h, 1)
    fem.assemble_augmented_momentum_jacobian(dr, case.dt)
    cnt = (C.c_int64 * abi.COUNTER_COUNT)()
    lib.femb200_profile_counters(h, cnt, abi.COUNTER_COUNT)
    lib.femb200_profile(h, 0)
    shared = cnt[abi.COUNTER_SHARED_JACOBIANS]
    got = [x.double().cpu().numpy() for x in list(dr.dRdv) + list(dr.PC)]
    lib2, h2 = _full_handle()
    try:
        assert lib2.femb200_jacobian_diagnostics(h2, C.byref(dr.problem()), float(case.dt), 0) == abi.OK
        torch.cuda.synchronize()
    finally:
        lib2.femb200_destroy(h2)
    full = [x.double().cpu().numpy() for x in list(dr.dRdv) + list(dr.PC)]
    print(f"seed {seed} {precision} copied geometry {copy_geometry}: {shared} of {case.mesh.nels} elements took "
          "their phase's shared Jacobian")
    assert (shared > 0) == (precision == "fp32")
    rtol = 1e-13 if precision == "fp64" else 5e-6
    for g, f in zip(got, full):
        np.testing.assert_allclose(g, f, rtol=rtol, atol=rtol * np.abs(f).max())
    hs = case.host_state(oh)
    hs.pressure_scaling(50.0, case.dt)
    hs.jacobian_diagnostics(case.dt)
    tol = 1e-9 if precision == "fp64" else 2e-5
    for g, r in zip(got, hs.dRdv + hs.PC):
        np.testing.assert_allclose(g, r, rtol=tol, atol=tol * np.abs(r).max())
