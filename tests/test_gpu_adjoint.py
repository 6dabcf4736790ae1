"""GPU adjoint (the hand-written reverse-mode element kernel and the frozen-operator
PH/DYREL adjoint solve) against the oracle and against central finite differences.

The oracle's transposed Jacobian is itself pinned by finite differences of its
forward residual (test_adjoint_oracle.py)."""
import numpy as np
import pytest

import oracle_host as oh
from cases import random_state_case
from conftest import fem
from test_adjoint_oracle import dense_adjoint

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.concatenate([np.ravel(x.detach().cpu().numpy() if hasattr(x, "detach") else x) for x in a])
    b = np.concatenate([np.ravel(x) for x in b])
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def device_and_host(case, gammaP=True):
    dr = case.device_state(fem)
    hs = case.host_state(oh)
    if gammaP and case.gammaP is None:
        rng = np.random.default_rng(3)
        g, m = rng.uniform(1, 5, case.mesh.nnodesP), rng.uniform(0.01, 0.1, case.mesh.nnodesP)
        hs.gammaP[:], hs.M_P[:] = g, m
        dr.gammaP.copy_(dr.tensor(g)); dr.M_P.copy_(dr.tensor(m))
    return dr, hs


@pytest.mark.parametrize("phases,plastic,finite_K,with_pnum", [
    ("nodal", True, False, True), ("cell", True, True, True), ("element", False, False, True),
    ("nodal", True, True, False)])
def test_adjoint_residual_matches_oracle(phases, plastic, finite_K, with_pnum):
    case = random_state_case(dim=3, n=3, seed=31, phases=phases, plastic=plastic, distort=True)
    dr, hs = device_and_host(case)
    rng = np.random.default_rng(7)
    lv = [rng.standard_normal(case.mesh.nnodes) for _ in range(3)]
    lP = rng.standard_normal(case.mesh.nnodesP)
    dv, dP = fem.assemble_adjoint_residual(dr, case.dt, [dr.tensor(x) for x in lv], dr.tensor(lP), finite_K=finite_K,
                                           with_pnum=with_pnum)
    torch.cuda.synchronize()
    rv, rP = hs.adjoint_residual(case.dt, lv, lP, finite_K=finite_K, with_pnum=with_pnum)
    assert rel(dv, rv) < 1e-11, rel(dv, rv)
    assert rel([dP], [rP]) < 1e-11, rel([dP], [rP])


def test_viscosity_sensitivity_matches_oracle():
    case = random_state_case(dim=3, n=3, seed=32, phases="nodal", plastic=True, distort=True)
    dr, hs = device_and_host(case)
    rng = np.random.default_rng(8)
    eta = 10 ** rng.uniform(0, 1, case.mesh.nq * case.mesh.nels)
    hs.viscosity_ip = eta
    dr.viscosity_ip = dr.tensor(eta)
    lv = [rng.standard_normal(case.mesh.nnodes) for _ in range(3)]
    lP = rng.standard_normal(case.mesh.nnodesP)
    s = fem.viscosity_sensitivity(dr, case.dt, [dr.tensor(x) for x in lv], dr.tensor(lP))
    ref = hs.viscosity_sensitivity(case.dt, lv, lP)
    assert rel([s], [ref]) < 1e-11


def forward(ac, delta, tol=1e-13):
    dr = ac.case.device_state(fem)
    dr.viscosity_ip = dr.tensor(ac.eta_ip(delta))
    st = fem.solve(dr, ac.case.bc_device(), dt=ac.case.dt, tolerance=tol, check_interval=50,
                   max_iterations=400_000, iter_max=400_000, throw_on_failure=False)
    assert st["converged"]
    return dr


def adjoint_gradient(ac, dr, tol=1e-12):
    J, obj = ac.objective(dr.v)
    lam_v, lam_P, st = fem.solve_adjoint(dr, ac.case.bc_device(), ac.case.dt, [dr.tensor(o) for o in obj],
                                         tolerance=tol, max_iterations=400_000, iter_max=400_000,
                                         max_ph_iterations=400)
    sens = fem.viscosity_sensitivity(dr, ac.case.dt, lam_v, lam_P)
    eta = dr.viscosity_ip
    grad = (eta * sens).reshape(dr.mesh.nels, dr.mesh.nq).sum(dim=1)
    return J, obj, lam_v, lam_P, grad, st


def test_adjoint_solve_matches_dense_oracle_adjoint():
    ac = fem.configs.adjoint_case(n=2, seed=1)
    dr = forward(ac, ac.delta)
    J, obj, lam_v, lam_P, grad, st = adjoint_gradient(ac, dr)
    assert st["converged"], st
    # the oracle's dense transposed Jacobian at the GPU forward state
    hs = ac.case.host_state(oh)
    hs.viscosity_ip = ac.eta_ip()
    for c in range(3):
        hs.v[c][:] = dr.v[c].cpu().numpy()
    hs.P[:] = dr.P.cpu().numpy()
    hs.gammaP[:] = dr.gammaP.cpu().numpy()
    hs.M_P[:] = dr.M_P.cpu().numpy()
    rl_v, rl_P = dense_adjoint(hs, ac.case.dt, obj, ac.case.bc)
    sens = hs.viscosity_sensitivity(ac.case.dt, rl_v, rl_P)
    rgrad = (ac.eta_ip() * sens).reshape(hs.mesh.nels, hs.mesh.nq).sum(axis=1)
    errs = (rel(lam_v, rl_v), rel([lam_P], [rl_P]), rel([grad], [rgrad]))
    print(f"adjoint vs dense oracle adjoint: λv {errs[0]:.2e}, λP {errs[1]:.2e}, gradient {errs[2]:.2e}")
    # the adjoint DR solve runs to 1e-12; its FP64 error against the direct solve is far below 1e-8
    assert max(errs) < 1e-8, errs


def test_adjoint_gradient_matches_central_differences():
    # central differences of J(δ) with the forward solve converged far below h²
    ac = fem.configs.adjoint_case(n=3, seed=2)
    dr = forward(ac, ac.delta)
    J, obj, lam_v, lam_P, grad, st = adjoint_gradient(ac, dr)
    grad = grad.cpu().numpy()
    rng = np.random.default_rng(9)
    h = 1e-4
    for k in rng.choice(dr.mesh.nels, size=6, replace=False):
        d = ac.delta.copy(); d[k] += h
        Jp = ac.objective(forward(ac, d).v)[0]
        d[k] -= 2 * h
        Jm = ac.objective(forward(ac, d).v)[0]
        fd = (Jp - Jm) / (2 * h)
        assert abs(fd - grad[k]) <= 1e-5 * np.abs(grad).max() + 1e-6 * abs(fd), (k, fd, grad[k])


def test_autograd_rule_matches_central_differences_and_reuses_checkpoint():
    # the rrule analogue: torch autograd through the solve, backward by the device adjoint
    ac = fem.configs.adjoint_case(n=2, seed=4)
    dr = ac.case.device_state(fem)
    bc = ac.case.bc_device()
    eta0 = dr.tensor(ac.eta_ip(np.zeros_like(ac.delta)))
    vt = torch.cat([dr.tensor(x) for x in ac.v_target])
    top = torch.zeros(3 * dr.mesh.nnodes, dtype=torch.bool, device=dr.device)
    for c in range(3):
        top[c * dr.mesh.nnodes + torch.as_tensor(ac.top - 1, device=dr.device).long()] = True
    kw = dict(tolerance=1e-13, max_iterations=400_000, iter_max=400_000, throw_on_failure=False, check_interval=50)

    def loss_of(delta):
        v = fem.solve_log_viscosity(delta, dr, bc, ac.case.dt, eta0, solve_kw=kw,
                                    adjoint_kw=dict(tolerance=1e-12, max_iterations=400_000, iter_max=400_000,
                                                    max_ph_iterations=400))
        return (((v - vt) * top) ** 2).sum()

    delta = dr.tensor(ac.delta).requires_grad_(True)
    L = loss_of(delta)
    # clobber the state between forward and backward: the checkpoint must restore it
    for x in dr.v:
        x.zero_()
    L.backward()
    g = delta.grad.cpu().numpy()
    h = 1e-4
    for k in (0, 3, 6):
        d = ac.delta.copy(); d[k] += h
        Lp = float(loss_of(dr.tensor(d)))
        d[k] -= 2 * h
        Lm = float(loss_of(dr.tensor(d)))
        fd = (Lp - Lm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-5 * np.abs(g).max() + 1e-6 * abs(fd), (k, fd, g[k])


def test_checkpoint_host_spill_round_trip():
    case = random_state_case(dim=3, n=2, seed=33, phases="cell", plastic=False, distort=False)
    dr = case.device_state(fem)
    ck = fem.DRCheckpoint(dr, host=True)
    torch.cuda.synchronize()
    ref = [x.clone() for x in dr.v] + [dr.P.clone()]
    for x in dr.v:
        x.add_(1.0)
    dr.P.mul_(3.0)
    ck.restore(dr)
    torch.cuda.synchronize()
    for a, b in zip([*dr.v, dr.P], ref):
        assert torch.equal(a, b)
