"""Tensile-cap local updates (femb200_cap_update) through the C ABI against the JustRelax
fixtures and the CPU oracle (itself pinned in test_cap_oracle.py). The device forms the
Newton Jacobian in closed form and solves it by pivoted elimination, the oracle by dual
numbers and the adjugate, so iterates differ by round-off: converged values agree to
1e-12 of the point's scale max(|s_trial|, |p_trial|), flags and failures exactly."""
import json
import math
import os

import numpy as np
import pytest

import oracle_host as oh
from conftest import fem

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
abi = fem._abi
HERE = os.path.dirname(os.path.abspath(__file__))
K, C0, PT = 0.5, math.cos(math.pi / 6), -0.5


def host(t):
    return t.detach().cpu().numpy()


def test_fixtures_on_the_device():
    with open(os.path.join(HERE, "golden", "cap_justrelax.json")) as f:
        d = json.load(f)
    R = np.array(d["rows"])
    kq = np.sin(np.radians(R[:, 0]))
    o = fem.cap_return_map(R[:, 2], R[:, 3], d["eta_ve"], d["K_dt"], K, kq, C0, d["pT"], R[:, 1])
    assert bool(o["converged"].all())
    got = np.stack([host(o["tau_II"]), host(o["P"]), host(o["lambda"]), host(o["lambda"] * o["A_p"])], axis=1)
    np.testing.assert_allclose(got, R[:, 4:], rtol=d["rtol"], atol=d["atol"])
    np.testing.assert_allclose(host(o["theta_dot"]), R[:, 7], rtol=d["rtol"], atol=d["atol"])


def random_points(n, seed):
    """Trial states around the cap of random materials: elastic, shear, cap and mixed
    branches, including hydrostatic tension (s = 0) and zero regularisation."""
    rng = np.random.default_rng(seed)
    phi = rng.uniform(math.radians(10), math.radians(40), n)
    psi = rng.uniform(0.0, 1.0, n) * phi * (rng.uniform(size=n) < 0.8)
    k, kq = np.sin(phi), np.sin(psi)
    C = rng.uniform(0.5, 3.0, n)
    c = C * np.cos(phi)
    pT = -rng.uniform(0.05, 0.9, n) * c / k
    s = np.abs(rng.normal(0.0, 2.0, n)) * (rng.uniform(size=n) < 0.9)
    p = rng.uniform(-3.0, 4.0, n)
    eve = rng.uniform(0.2, 3.0, n)
    kdt = rng.uniform(0.5, 8.0, n)
    ereg = rng.uniform(0.0, 0.5, n) * (rng.uniform(size=n) < 0.7)
    return s, p, eve, kdt, k, kq, c, pT, ereg


def test_return_map_matches_oracle_on_every_branch():
    s, p, eve, kdt, k, kq, c, pT, ereg = random_points(20000, seed=7)
    dev = fem.cap_return_map(s, p, eve, kdt, k, kq, c, pT, ereg)
    ref = oh.cap_update(0, s, p, eve, kdt, k, kq, c, pT, ereg)
    conv = host(dev["converged"])
    assert (conv == ref["converged"]).all()
    assert conv.mean() > 0.99
    lam = ref["lambda"]
    assert (lam > 0).mean() > 0.3 and (lam == 0).mean() > 0.3      # plastic and elastic points
    scale = np.maximum(np.maximum(np.abs(s), np.abs(p)), 1.0)
    for key in ("tau_II", "P", "lambda", "A_tau", "A_p", "gamma_dot", "theta_dot"):
        d, r = host(dev[key]), ref[key]
        assert (np.isnan(d) == np.isnan(r)).all(), key
        ok = ~np.isnan(r)
        assert (np.abs(d[ok] - r[ok]) / scale[ok]).max() <= 1e-12, key


@pytest.mark.parametrize("ncomp", [3, 6])
def test_local_update_matches_oracle(ncomp):
    n = 5000
    s, p, eve, kdt, k, kq, c, pT, ereg = random_points(n, seed=11 + ncomp)
    rng = np.random.default_rng(ncomp)
    tau = rng.normal(0.0, 1.5, (n, ncomp))
    tau[:50] = 0.0                                  # the invariant floor at zero stress
    dev = fem.cap_local_update(torch.as_tensor(tau, device="cuda"), p, eve, kdt, k, kq, c, pT, ereg)
    ref = oh.cap_update(ncomp, tau, p, eve, kdt, k, kq, c, pT, ereg)
    assert (host(dev["converged"]) == ref["converged"]).all()
    scale = np.maximum(np.maximum(np.abs(tau).max(axis=1), np.abs(p)), 1.0)
    for key in ("P", "gamma_dot", "theta_dot", "tau_II", "lambda"):
        d, r = host(dev[key]), ref[key]
        assert (np.isnan(d) == np.isnan(r)).all(), key
        ok = ~np.isnan(r)
        assert (np.abs(d[ok] - r[ok]) / scale[ok]).max() <= 1e-12, key
    d, r = host(dev["tau"]), ref["tau"]
    ok = ~np.isnan(r).any(axis=1)
    assert (np.abs(d[ok] - r[ok]) / scale[ok, None]).max() <= 1e-12
    assert (host(dev["tau"])[:50] == 0).all()


def test_failures_and_arguments():
    out = fem.cap_return_map([0.0, 0.0, 0.0, 0.0], -1.0, [0.0, 1.0, 1.0, 1.0], [4.0, 0.0, math.inf, 4.0], K, 0.0,
                             C0, PT, 0.1)
    assert not bool(out["converged"][:3].any()) and bool(out["converged"][3])
    assert torch.isnan(out["gamma_dot"][:3]).all() and torch.isnan(out["theta_dot"][:3]).all()
    assert (host(out["tau_II"][:3]) == 0.0).all() and (host(out["P"][:3]) == -1.0).all()
    assert (host(out["lambda"][:3]) == 0.0).all()
    z = fem.cap_return_map(0.0, -1.0, 1.0, 4.0, K, 0.0, C0, PT, 0.1, maxiter=0)
    assert not bool(z["converged"]) and float(z["P"]) == -1.0
    failed = fem.cap_local_update([[0.0, 0.0, 0.0]], -1.0, 0.0, 4.0, K, 0.0, C0, PT, 0.1)
    assert torch.isnan(failed["tau"]).all() and torch.isnan(failed["P"]).all()
    el = fem.cap_return_map(0.2, 0.0, 1.0, 4.0, K, 0.0, C0, PT, 0.1)
    assert bool(el["converged"]) and (float(el["tau_II"]), float(el["P"]), float(el["lambda"])) == (0.2, 0.0, 0.0)
    # the C ABI rejects a bad component count and missing inputs; an empty batch is a no-op
    import ctypes as C
    lib, h = fem.solver._Handle.get()
    pr = abi.CapProblemC()
    pr.n, pr.ncomp = 4, 4
    with pytest.raises(abi.FemB200Error, match="ncomp must be 0"):
        fem.solver._check(lib, h, lib.femb200_cap_update(h, C.byref(pr)))
    pr.ncomp = 0
    with pytest.raises(abi.FemB200Error, match="trial state and every material array are required"):
        fem.solver._check(lib, h, lib.femb200_cap_update(h, C.byref(pr)))
    pr.n = 0
    fem.solver._check(lib, h, lib.femb200_cap_update(h, C.byref(pr)))
