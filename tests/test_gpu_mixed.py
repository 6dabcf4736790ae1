"""Mixed-precision DR solve: FP32 Chebyshev iterations on increments inside FP64
Powell–Hestenes steps (controls.precision = MIXED).

The mixed solve stops on the same FP64 outer test as the FP64 solve, so at a
given tolerance it must be as accurate as the FP64 solve: both are compared with
a reference solution converged far below that tolerance (the FP64 path, itself
pinned to the CPU oracle in test_gpu_parity.py), field by field (v, P, τ).
"""
import numpy as np
import pytest

import oracle_host as oh
from cases import random_state_case, vep_layers_case
from conftest import fem

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
abi = fem._abi


def rel_l2(a, b):
    a = a.detach().double().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    b = b.detach().double().cpu().numpy() if hasattr(b, "detach") else np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def fields(dr, dt):
    fem.update_stokes_current_stress(dr, dt)
    return {"v": torch.cat([x.clone() for x in dr.v]), "P": dr.P.clone(), "tau": torch.cat([x.clone() for x in dr.tau])}


def solve_fields(case, tol, precision):
    dr = case.device_state(fem)
    st = fem.solve(dr, case.bc_device(), dt=case.dt, tolerance=tol, check_interval=50, throw_on_failure=False,
                   precision=precision, max_iterations=500_000, iter_max=500_000)
    return st, fields(dr, case.dt)


@pytest.mark.parametrize("seed,plastic", [(1, True), (2, False)])
def test_mixed_solve_as_accurate_as_fp64(seed, plastic):
    case = vep_layers_case(n=4, seed=seed, plastic=plastic)
    st_ref, ref = solve_fields(case, 1e-13, "fp64")
    st64, f64 = solve_fields(case, 1e-8, "fp64")
    stm, fm = solve_fields(case, 1e-8, "mixed")
    assert st_ref["converged"] and st64["converged"] and stm["converged"]
    # the outer test is evaluated in FP64 in both modes
    assert stm["err"] < 1e-8
    # one FP64 base sweep per Powell–Hestenes step that ran Chebyshev iterations
    assert stm["defect_corrections"] == stm["itPH"] - 1
    # same algorithm: the iteration counts stay close
    assert abs(stm["iter"] - st64["iter"]) <= 0.15 * st64["iter"] + 100, (stm["iter"], st64["iter"])
    for k in ("v", "P", "tau"):
        e64, em = rel_l2(f64[k], ref[k]), rel_l2(fm[k], ref[k])
        print(f"seed {seed} plastic {plastic} {k}: fp64 {e64:.3e} mixed {em:.3e} (mixed vs fp64 {rel_l2(fm[k], f64[k]):.3e})")
        assert em <= 3 * e64 + 1e-9, (k, em, e64)


def test_mixed_solve_matches_oracle():
    # The oracle's FP64 solve at the same tolerance, on a VEP problem with plastic points.
    case = vep_layers_case(n=3, seed=4)
    dr, hs = case.device_state(fem), case.host_state(oh)
    st = fem.solve(dr, case.bc_device(), dt=case.dt, tolerance=1e-8, check_interval=50, precision="mixed")
    ref = hs.solve(dt=case.dt, tolerance=1e-8, check_interval=50)
    assert st["converged"] and ref["converged"]
    assert rel_l2(torch.cat(list(dr.v)), np.concatenate(hs.v)) < 1e-6
    assert rel_l2(dr.P, hs.P) < 1e-6


def test_mixed_rejects_unsupported_meshes():
    case = random_state_case(dim=3, n=2, seed=3, phases="cell", distort=True)
    dr = case.device_state(fem)
    with pytest.raises(abi.FemB200Error, match="affine"):
        fem.solve(dr, case.bc_device(), dt=case.dt, precision="mixed")
    case2 = random_state_case(dim=2, n=2, seed=3, phases="cell")
    dr2 = case2.device_state(fem)
    with pytest.raises(abi.FemB200Error, match="3-D"):
        fem.solve(dr2, case2.bc_device(), dt=case2.dt, precision="mixed")


@pytest.mark.parametrize("layout", ["element_node", "nodal"])
def test_mixed_solve_phase_layouts(layout):
    # Element-node phases that repeat the cell phase keep every element in one phase
    # (the thread-per-element incremental sweep); nodal phases put the nodes of the
    # layer interfaces in one phase or the other, so interface elements mix phases
    # (the warp-cooperative sweep). Both must agree with the FP64 solve.
    case = vep_layers_case(n=3, seed=6)
    cell = case.phases_v
    if layout == "element_node":
        case.phases_v = np.repeat(cell[:, None], case.mesh.nv, axis=1).astype(np.int32)
        case.phases_v_layout = abi.PHASE_ELEMENT_NODE
        case.phases_P = np.repeat(cell[:, None], case.mesh.np_, axis=1).astype(np.int32)
        case.phases_P_layout = abi.PHASE_ELEMENT_NODE
    else:
        nodal = np.ones(case.mesh.nnodes, dtype=np.int32)
        nodal[case.mesh.el2n.reshape(-1) - 1] = np.repeat(cell, case.mesh.nv)
        case.phases_v, case.phases_v_layout = nodal, abi.PHASE_NODAL
        case.phases_P = np.repeat(cell, case.mesh.np_).astype(np.int32)
        case.phases_P_layout = abi.PHASE_NODAL
    st64, f64 = solve_fields(case, 1e-8, "fp64")
    stm, fm = solve_fields(case, 1e-8, "mixed")
    assert st64["converged"] and stm["converged"] and stm["err"] < 1e-8
    for k in ("v", "P", "tau"):
        assert rel_l2(fm[k], f64[k]) < 1e-6, (layout, k, rel_l2(fm[k], f64[k]))


def test_mixed_solve_on_sheared_affine_cells():
    # parallelepiped cells (a full J⁻¹): the general-geometry form of the FP32 sweep
    case = random_state_case(dim=3, n=3, seed=8, phases="cell", plastic=False, distort=False)
    st64, f64 = solve_fields(case, 1e-8, "fp64")
    stm, fm = solve_fields(case, 1e-8, "mixed")
    assert st64["converged"] and stm["converged"] and stm["err"] < 1e-8
    for k in ("v", "P"):
        assert rel_l2(fm[k], f64[k]) < 1e-6, (k, rel_l2(fm[k], f64[k]))
