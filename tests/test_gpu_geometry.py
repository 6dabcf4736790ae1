"""Device element geometry (precompute_geometry / update_geometry!, src/mesh/mesh.jl:592-682,
src/mesh/mixed_mesh.jl:337-392) through the C ABI against the CPU oracle's geometry.

FP64: J, J⁻¹ and |det J| are formed in a different order than the oracle's, so the bound
is 1e-13 of the largest entry. FP32 storage must equal the FP64 result rounded once.
"""
import numpy as np
import pytest

import oracle_host as oh
from cases import random_state_case
from conftest import fem

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
abi = fem._abi


def oracle_geometry(dim, coords, el2n):
    nels = el2n.shape[0]
    nq = 27 if dim == 3 else 9
    geo_v = np.zeros((nels, nq, dim * dim + 1))
    geo_P = np.zeros((nels, nq))
    c = np.ascontiguousarray(coords, dtype=np.float64)
    e = np.ascontiguousarray(el2n, dtype=np.int32)
    oh.check(oh.lib().orc_geometry(dim, nels, oh.ptr(c), oh.ptr(e), oh.ptr(geo_v), oh.ptr(geo_P)))
    return geo_v, geo_P


def distorted(dim, n, seed):
    case = random_state_case(dim=dim, n=n, seed=seed, distort=True)
    return case


@pytest.mark.parametrize("dim", [3, 2])
def test_geometry_matches_oracle_on_distorted_mesh(dim):
    case = distorted(dim, 4 if dim == 3 else 6, seed=3)
    mesh = case.mesh
    geo_v, geo_P = fem.precompute_geometry(mesh.coords, mesh.el2n, dim)
    ref_v, ref_P = oracle_geometry(dim, mesh.coords, mesh.el2n)
    g, gp = geo_v.cpu().numpy(), geo_P.cpu().numpy()
    np.testing.assert_allclose(g, ref_v, rtol=0, atol=1e-13 * np.abs(ref_v).max())
    np.testing.assert_allclose(gp, ref_P, rtol=0, atol=1e-13 * np.abs(ref_P).max())
    # the mesh's own (host) geometry is the same quantity
    np.testing.assert_allclose(g, mesh.geo_v, rtol=0, atol=1e-13 * np.abs(ref_v).max())


def test_fp32_geometry_is_the_fp64_result_rounded_once():
    case = distorted(3, 3, seed=8)
    mesh = case.mesh
    g64, p64 = fem.precompute_geometry(mesh.coords, mesh.el2n, 3, geometry_dtype=torch.float64)
    g32, p32 = fem.precompute_geometry(mesh.coords, mesh.el2n, 3, geometry_dtype=torch.float32)
    assert g32.dtype == torch.float32
    assert torch.equal(g32, g64.to(torch.float32))
    assert torch.equal(p32, p64.to(torch.float32))


def test_update_geometry_in_place_and_residuals_follow():
    # a StokesDR built on the straight mesh, then moved onto the distorted coordinates,
    # must hold the same geometry (same arrays) and give the same residuals as a state
    # built on the distorted mesh directly
    case = distorted(3, 3, seed=5)
    mesh = case.mesh
    straight = fem.structured_mixed_mesh(3, (3, 3, 3))
    moved_case = random_state_case(dim=3, n=3, seed=5, distort=True)
    moved_case.mesh.geo_v = straight.geo_v.copy()
    moved_case.mesh.geo_P = straight.geo_P.copy()
    dr = moved_case.device_state(fem)
    ptr_v = dr._mesh["geo_v"].data_ptr()
    fem.update_geometry(dr, torch.as_tensor(mesh.coords, device="cuda"))
    assert dr._mesh["geo_v"].data_ptr() == ptr_v
    ref_v, ref_P = oracle_geometry(3, mesh.coords, mesh.el2n)
    np.testing.assert_allclose(dr._mesh["geo_v"].cpu().numpy(), ref_v, rtol=0, atol=1e-13 * np.abs(ref_v).max())
    np.testing.assert_allclose(dr._mesh["geo_P"].cpu().numpy(), ref_P, rtol=0, atol=1e-13 * np.abs(ref_P).max())
    direct = case.device_state(fem)
    fem.assemble_stokes_residuals(dr, case.dt)
    fem.assemble_stokes_residuals(direct, case.dt)
    for c in range(3):
        scale = direct.Rv[c].abs().max().item()
        assert (dr.Rv[c] - direct.Rv[c]).abs().max().item() <= 1e-11 * scale
    assert (dr.RP - direct.RP).abs().max().item() <= 1e-11 * direct.RP.abs().max().item()


def test_update_geometry_of_a_thermal_state():
    case = distorted(3, 3, seed=9)
    mesh = case.mesh
    straight = fem.structured_mixed_mesh(3, (3, 3, 3))
    th = fem.ThermalDiffusionDR(straight)
    fem.update_geometry(th, mesh.coords)
    ref_v, _ = oracle_geometry(3, mesh.coords, mesh.el2n)
    np.testing.assert_allclose(th.geo.cpu().numpy(), ref_v, rtol=0, atol=1e-13 * np.abs(ref_v).max())


def test_connectivity_outside_the_node_range_is_rejected():
    mesh = fem.structured_mixed_mesh(2, (2, 2))
    el2n = mesh.el2n.copy()
    el2n[1, 4] = mesh.nnodes + 5           # never dereferenced: the kernel checks before reading
    with pytest.raises(abi.FemB200Error, match="outside 1:nnodes"):
        fem.precompute_geometry(mesh.coords, el2n, 2)
    el2n[1, 4] = 0
    with pytest.raises(abi.FemB200Error, match="outside 1:nnodes"):
        fem.precompute_geometry(mesh.coords, el2n, 2)


def test_empty_mesh_is_a_no_op():
    geo_v, geo_P = fem.precompute_geometry(np.zeros((1, 3)), np.zeros((0, 27), dtype=np.int32), 3)
    assert geo_v.shape == (0, 27, 10) and geo_P.shape == (0, 27)
