"""Ordered scatter of the mixed-precision solve (femb200_set_ordered_scatter).

With the option on, the FP32 sweep runs once per tile colour and the FP64 sweep and the
Jacobian diagnostics once per colour of warp groups, so every node receives at most one
atomic addition per launch: two solves of the same problem must then be identical bit for
bit, and must reach the answer of the atomic scatter (the two differ only in the order of
additions). Meshes whose tiles do not run along ξ must be refused with the solver's
message.
"""
import numpy as np
import pytest

from cases import vep_layers_case
from conftest import fem

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
abi = fem._abi


def rel_l2(a, b):
    a, b = a.double().cpu().numpy(), b.double().cpu().numpy()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def solve_mixed(case, ordered):
    dr = case.device_state(fem)
    st = fem.solve(dr, case.bc_device(), dt=case.dt, tolerance=1e-8, check_interval=100,
                   throw_on_failure=False, precision="mixed", ordered_scatter=ordered)
    fem.update_stokes_current_stress(dr, case.dt)
    f = {"v": torch.cat([x.clone() for x in dr.v]), "P": dr.P.clone(), "tau": torch.cat([x.clone() for x in dr.tau])}
    return st, f


def test_ordered_scatter_is_reproducible_and_reaches_the_atomic_solution():
    # 32 elements per row: every tile is one row of elements along ξ
    case = vep_layers_case(n=32, seed=0)
    st_a, fa = solve_mixed(case, False)
    st_o, fo = solve_mixed(case, True)
    st_o2, fo2 = solve_mixed(case, True)
    assert st_a["converged"] and st_o["converged"]
    # reproducible: the same path and the same fields, bit for bit
    assert (st_o2["iter"], st_o2["itPH"], st_o2["err"]) == (st_o["iter"], st_o["itPH"], st_o["err"])
    for k in ("v", "P", "tau"):
        assert torch.equal(fo2[k], fo[k]), k
    assert st_o["err"] < 1e-8
    # the same path up to the order of FP32 additions: the stopping check may move by one
    assert abs(st_o["iter"] - st_a["iter"]) <= 100, (st_o["iter"], st_a["iter"])
    assert st_o["itPH"] == pytest.approx(st_a["itPH"], abs=2)
    for k in ("v", "P", "tau"):
        d = rel_l2(fo[k], fa[k])
        print(f"{k}: ordered vs atomic {d:.3e}")
        # both stop at min(err_abs, err_rel) < 1e-8; the mixed solve's fields are within
        # 5e-8 of the FP64 solution at this tolerance
        assert d < 2e-7, (k, d)


def test_ordered_scatter_refuses_tiles_across_rows():
    # 4 elements per row: a tile of 32 elements spans eight rows, whose elements share
    # nodes other than the ξ faces of lane neighbours
    case = vep_layers_case(n=4, seed=1)
    with pytest.raises(abi.FemB200Error, match="ordered scatter needs consecutive elements"):
        solve_mixed(case, True)
    # the handle is usable afterwards, with the option off
    st, _ = solve_mixed(case, False)
    assert st["converged"]
