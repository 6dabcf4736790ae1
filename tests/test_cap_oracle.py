"""Pins the tensile-cap oracle (oracle/cap.cpp) and the host cap formulas of
femtools_b200.cap to the reference's own tests (test/test_drucker_prager_cap.jl): the 16
JustRelax return-map rows (tests/golden/cap_justrelax.json, made from that file by
tests/golden/make_cap_fixtures.py) at rtol 1e-12, the closed forms and residual identities
of the coupled return, the geometry identities of the cap surface, and the parameter checks
of DruckerPragerCap, and the Popov 2-D material point (test/test_popov_2d_material_point.jl).
CPU only."""
import json
import math
import os

import numpy as np
import pytest

import oracle_host as oh
from conftest import fem

HERE = os.path.dirname(os.path.abspath(__file__))

# test/test_drucker_prager_cap.jl:9-15 (unit-scale surface) and :281-283 (material point)
CAP_k, CAP_kq = math.sin(math.radians(30.0)), math.sin(math.radians(10.0))
CAP_c, CAP_pT = 10.0 * math.cos(math.radians(30.0)), -5.0
K, C0, PT, ETA_VE, KDT = 0.5, math.cos(math.pi / 6), -0.5, 1.0, 4.0


def fixtures():
    with open(os.path.join(HERE, "golden", "cap_justrelax.json")) as f:
        return json.load(f)


def test_oracle_matches_the_justrelax_fixtures():
    # test/test_drucker_prager_cap.jl:366-403
    d = fixtures()
    R = np.array(d["rows"])
    kq = np.sin(np.radians(R[:, 0]))
    o = oh.cap_update(0, R[:, 2], R[:, 3], d["eta_ve"], d["K_dt"], K, kq, C0, d["pT"], R[:, 1])
    assert o["converged"].all()
    got = np.stack([o["tau_II"], o["P"], o["lambda"], o["lambda"] * o["A_p"]], axis=1)
    np.testing.assert_allclose(got, R[:, 4:], rtol=d["rtol"], atol=d["atol"])


def residual(ret, i, s, p, kq, eta_reg):
    F, At, Ap = fem.cap_invariants(ret["tau_II"][i], ret["P"][i], K, kq, C0, PT)
    lam = ret["lambda"][i]
    return (ret["tau_II"][i] - s + 2 * ETA_VE * lam * At, ret["P"][i] - p - KDT * lam * Ap, F - eta_reg * lam)


@pytest.mark.parametrize("psi", [0.0, math.radians(5.0)])
@pytest.mark.parametrize("eta_reg", [0.1, 0.0])
def test_coupled_return(psi, eta_reg):
    # test/test_drucker_prager_cap.jl:289-312
    kq = math.sin(psi)
    pts = [(0.0, -1.0), (0.0, -0.8), (1.0, -1.0), (1.0, -0.8), (3.0, 2.0)]
    s, p = np.array(pts).T
    ret = oh.cap_update(0, s, p, ETA_VE, KDT, K, kq, C0, PT, eta_reg)
    assert ret["converged"].all() and (ret["lambda"] > 0).all()
    for i, (si, pi) in enumerate(pts):
        assert max(abs(r) for r in residual(ret, i, si, pi, kq, eta_reg)) <= 1e-12
        if pi < 0:
            assert ret["A_p"][i] > 0          # tension opens
    a = math.sqrt(1 + K * K)
    if kq == 0:
        assert ret["lambda"][0] == pytest.approx(a * (PT + 1.0) / (eta_reg + a * KDT), rel=1e-12)
        assert ret["tau_II"][0] == 0
    # radial Drucker–Prager limit on the shear branch
    lam = (3.0 - K * 2.0 - C0) / (ETA_VE + eta_reg + KDT * K * kq)
    assert ret["lambda"][4] == pytest.approx(lam, rel=1e-12)
    assert ret["tau_II"][4] == pytest.approx(3.0 - ETA_VE * lam, rel=1e-12)
    assert ret["P"][4] == pytest.approx(2.0 + KDT * kq * lam, rel=1e-12)


def test_elastic_unloading_and_independent_branches():
    # test/test_drucker_prager_cap.jl:314-332
    ret = oh.cap_update(0, 0.2, 0.0, ETA_VE, KDT, K, 0.0, C0, PT, 0.1)
    assert ret["converged"][0] and (ret["tau_II"][0], ret["P"][0], ret["lambda"][0]) == (0.2, 0.0, 0.0)
    kq = math.sin(math.radians(20.0))
    g = fem.cap_geometry(K, kq, C0, PT)
    for s, p in ((g.tau_d / 2 + 1, g.p_y - K * g.tau_d / 2 + 0.01), (2 * g.tau_d, g.p_y - 2 * K * g.tau_d - 0.01)):
        ret = oh.cap_update(0, s, p, ETA_VE, KDT, K, kq, C0, PT, 0.1)
        assert ret["converged"][0]
        assert max(abs(r) for r in residual(ret, 0, s, p, kq, 0.1)) <= 1e-12


def _rot2(t, th):
    R = np.array([[math.cos(th), -math.sin(th)], [math.sin(th), math.cos(th)]])
    M = R @ np.array([[t[0], t[2]], [t[2], t[1]]]) @ R.T
    return np.array([M[0, 0], M[1, 1], M[0, 1]])


def test_tensor_update_is_radial_and_rotation_invariant():
    # test/test_drucker_prager_cap.jl:334-353, and the same for a 3-D stress
    tau = np.array([1.2, -0.3, 0.4])
    out = oh.cap_update(3, tau, -0.6, ETA_VE, KDT, K, 0.1, C0, PT, 0.1)
    ret = oh.cap_update(0, math.sqrt((1.2 ** 2 + 0.3 ** 2 + 0.9 ** 2) / 2 + 0.4 ** 2), -0.6, ETA_VE, KDT, K, 0.1, C0,
                        PT, 0.1)
    t = out["tau"][0]
    sII = math.sqrt((t[0] ** 2 + t[1] ** 2 + (t[0] + t[1]) ** 2) / 2 + t[2] ** 2)
    assert sII == pytest.approx(ret["tau_II"][0], rel=1e-12)
    assert out["P"][0] == pytest.approx(ret["P"][0], rel=1e-12)
    assert out["gamma_dot"][0] == pytest.approx(ret["lambda"][0] * ret["A_tau"][0], rel=1e-12)
    assert out["theta_dot"][0] == pytest.approx(ret["lambda"][0] * ret["A_p"][0], rel=1e-12)
    rot = oh.cap_update(3, _rot2(tau, 0.7), -0.6, ETA_VE, KDT, K, 0.1, C0, PT, 0.1)
    np.testing.assert_allclose(rot["tau"][0], _rot2(t, 0.7), rtol=1e-12, atol=1e-14)
    assert rot["P"][0] == pytest.approx(out["P"][0], rel=1e-12)
    zero = oh.cap_update(3, np.zeros(3), -1.0, ETA_VE, KDT, K, 0.0, C0, PT, 0.1)
    assert (zero["tau"][0] == 0).all()
    z0 = oh.cap_update(0, 0.0, -1.0, ETA_VE, KDT, K, 0.0, C0, PT, 0.1)
    assert zero["P"][0] == pytest.approx(z0["P"][0], rel=1e-12)
    # 3-D: a rotated stress returns the rotated stress
    rng = np.random.default_rng(3)
    A = rng.standard_normal((3, 3))
    S = A + A.T
    S -= np.trace(S) / 3 * np.eye(3)
    Q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    pack = lambda M: np.array([M[0, 0], M[1, 1], M[2, 2], M[0, 1], M[0, 2], M[1, 2]])
    o3 = oh.cap_update(6, np.stack([pack(S), pack(Q @ S @ Q.T)]), -0.6, ETA_VE, KDT, K, 0.1, C0, PT, 0.1)
    assert o3["converged"].all() and o3["lambda"][0] > 0
    t0 = o3["tau"][0]
    M0 = np.array([[t0[0], t0[3], t0[4]], [t0[3], t0[1], t0[5]], [t0[4], t0[5], t0[2]]])
    np.testing.assert_allclose(o3["tau"][1], pack(Q @ M0 @ Q.T), rtol=1e-11, atol=1e-13)


def test_failures_are_explicit():
    # test/test_drucker_prager_cap.jl:361-368
    for eve, kdt in ((0.0, KDT), (ETA_VE, 0.0), (ETA_VE, math.inf)):
        assert not oh.cap_update(0, 0.0, -1.0, eve, kdt, K, 0.0, C0, PT, 0.1)["converged"][0]
    ret = oh.cap_update(0, 0.0, -1.0, ETA_VE, KDT, K, 0.0, C0, PT, 0.1, maxiter=0)
    assert not ret["converged"][0] and (ret["tau_II"][0], ret["P"][0], ret["lambda"][0]) == (0.0, -1.0, 0.0)
    failed = oh.cap_update(3, np.zeros(3), -1.0, 0.0, KDT, K, 0.0, C0, PT, 0.1)
    assert np.isnan(failed["tau"]).all() and np.isnan(failed["P"][0]) and np.isnan(failed["gamma_dot"][0])


def test_oracle_invariants_match_the_host_formulas():
    # the scalar coefficients of test/test_drucker_prager_cap.jl:26-60 on both branch pairs
    g = fem.cap_geometry(CAP_k, CAP_kq, CAP_c, CAP_pT)
    probes = [(1.0, -6.0), (30.0, 20.0), (g.tau_d / 2, g.p_y - CAP_k * g.tau_d / 2 - 0.1),
              (2 * g.tau_d, g.p_y - 2 * CAP_k * g.tau_d + 0.1), (0.0, -6.0), (0.0, g.p_q)]
    for s, p in probes[2:4]:
        assert (p + CAP_k * s >= g.p_y) != (p + CAP_kq * s >= g.p_q)
    s, p = np.array(probes).T
    F, At, Ap = oh.cap_invariants(s, p, CAP_k, CAP_kq, CAP_c, CAP_pT)
    for i, (si, pi) in enumerate(probes):
        want = fem.cap_invariants(si, pi, CAP_k, CAP_kq, CAP_c, CAP_pT)
        np.testing.assert_allclose((F[i], At[i], Ap[i]), want, rtol=1e-15, atol=1e-15)
        expected_F = si - CAP_k * pi - CAP_c if pi + CAP_k * si >= g.p_y else \
            g.a * (math.hypot(si, pi - g.p_y) - g.R_y)
        assert F[i] == pytest.approx(expected_F, rel=1e-12)
    assert At[4] == 0 and Ap[4] == pytest.approx(g.b, rel=1e-12)
    assert (At[5], Ap[5]) == (0.5, CAP_kq)       # shear branch at the potential centre


def test_cap_geometry_identities():
    # test/test_drucker_prager_cap.jl:101-131, :133-157, :159-173, :214-231
    g = fem.cap_geometry(CAP_k, CAP_kq, CAP_c, CAP_pT)
    ap = lambda a, b, tol=1e-12: abs(a - b) <= tol * max(1.0, abs(b))
    assert ap(g.a, math.sqrt(1 + CAP_k ** 2)) and ap(g.b, math.sqrt(1 + CAP_kq ** 2))
    assert ap(g.R_y, g.p_y - CAP_pT) and ap(g.R_y, (CAP_k * g.p_y + CAP_c) / g.a)
    assert ap(g.tau_d, CAP_k * g.p_d + CAP_c) and ap(g.tau_d, g.R_y / g.a)
    assert ap(math.sqrt(g.tau_d ** 2 + (g.p_d - g.p_y) ** 2), g.R_y)
    assert ap(g.p_q, g.p_d + CAP_kq * g.tau_d)
    assert CAP_c + CAP_k * CAP_pT > 0 and g.R_y > 0 and CAP_pT < g.p_d < g.p_y and g.tau_d > 0
    Fy = lambda t, P: fem.cap_yield_function(t, P, CAP_k, CAP_c, g)
    assert abs(Fy(0.0, CAP_pT)) <= 1e-12
    # on the cap circle between the delimiter and the apex, every point on the cap branch
    th_d = math.atan2(1 / g.a, -CAP_k / g.a)
    for th in np.linspace(th_d, math.pi, 9):
        P, t = g.p_y + g.R_y * math.cos(th), g.R_y * math.sin(th)
        assert abs(Fy(t, P)) <= 1e-10 and P + CAP_k * t <= g.p_y + 1e-10
    for P in np.linspace(g.p_d, g.p_d + 20, 9):
        assert abs(Fy(CAP_k * P + CAP_c, P)) <= 1e-10
    assert Fy(0.0, g.p_y) < 0 and Fy(0.0, CAP_pT - 1.0) > 0 and Fy(2 * g.tau_d, g.p_d + 20) < 0
    # the two branches agree on the switching ray P + k·τII = p_y
    for t in np.linspace(0.0, 3 * g.tau_d, 11):
        P = g.p_y - CAP_k * t
        shear = t - CAP_k * P - CAP_c
        cap = g.a * (math.sqrt(t * t + (P - g.p_y) ** 2) - g.R_y)
        assert abs(shear - cap) <= 1e-10 and abs(Fy(t, P) - shear) <= 1e-10
    # the shear domain is the Drucker–Prager surface for any cap out of reach
    cphi = 10.0 * math.cos(math.radians(30.0))
    for pT in (-5.0, -50.0, -5.0e3):
        gc = fem.cap_geometry(CAP_k, CAP_kq, cphi, pT)
        for t, P in ((5.0, 20.0), (30.0, 100.0), (1.0, 60.0)):
            if P + CAP_k * t >= gc.p_y:
                assert fem.cap_yield_function(t, P, CAP_k, cphi, gc) == pytest.approx(t - cphi - P * CAP_k, abs=1e-14)
    assert 0.0 >= fem.cap_geometry(CAP_k, CAP_kq, CAP_c, -1.0e6).p_y


def test_drucker_prager_cap_parameters():
    # test/test_drucker_prager_cap.jl:62-80 and the constructor checks (stokes_types.jl:492-545)
    phi, psi, C, pT = math.pi / 6, math.pi / 18, 10.0, -5.0
    mat = fem.DruckerPragerCap((phi,), (psi,), (C,), (pT,), (0.1,), (4.0,), C_min=(4.0,), H_C=(-2.0,))
    k, kq, cphi = math.sin(phi), math.sin(psi), math.cos(phi)
    for gam, Cs in ((0.0, C), (2.0, 6.0), (100.0, 4.0)):
        assert fem.cap_invariants_phase(mat, 1, 1.0, -6.0, gam) == fem.cap_invariants(1.0, -6.0, k, kq, Cs * cphi, pT)
        assert fem.cap_geometry(k, kq, Cs * cphi, pT).R_y > 0
    assert fem.cap_invariants_phase(mat, 1, 1.0, -6.0, None) == fem.cap_invariants_phase(mat, 1, 1.0, -6.0, 0.0)
    with pytest.raises(ValueError, match="softened cap radius must remain positive"):
        fem.DruckerPragerCap((phi,), (psi,), (C,), (pT,), (0.1,), (4.0,), C_min=(1.0,), H_C=(-2.0,))
    for Kb in (0.0, -1.0):
        with pytest.raises(ValueError, match="positive finite bulk modulus"):
            fem.DruckerPragerCap((phi,), (psi,), (C,), (pT,), (0.1,), (Kb,))
    for bad in (math.inf, math.nan):
        with pytest.raises(ValueError, match="must all be finite"):
            fem.DruckerPragerCap((phi,), (psi,), (C,), (pT,), (0.1,), (bad,))
        with pytest.raises(ValueError, match="must all be finite"):
            fem.DruckerPragerCap((phi,), (psi,), (bad,), (pT,), (0.1,), (4.0,))
    with pytest.raises(ValueError, match="tensile strength pT must be ≤ 0"):
        fem.DruckerPragerCap((phi,), (psi,), (C,), (1.0,), (0.1,), (4.0,))
    with pytest.raises(ValueError, match="cap radius is not positive"):
        fem.DruckerPragerCap((phi,), (psi,), (1.0,), (-5.0,), (0.1,), (4.0,))


def _grad_F(t, P, g, h=1e-5):
    F = lambda a, b: fem.cap_yield_function(a, b, CAP_k, CAP_c, g)
    return (F(t + h, P) - F(t - h, P)) / (2 * h), (F(t, P + h) - F(t, P - h)) / (2 * h)


def test_yield_gradient_has_magnitude_a_and_is_continuous():
    # test/test_drucker_prager_cap.jl:175-212
    g = fem.cap_geometry(CAP_k, CAP_kq, CAP_c, CAP_pT)
    for t, P in ((2 * g.tau_d, g.p_d + 10.0), (0.2 * g.tau_d, CAP_pT - 0.5), (g.tau_d, g.p_d + 0.05),
                 (g.tau_d, g.p_d - 0.05)):
        dt, dP = _grad_F(t, P, g)
        assert math.hypot(dt, dP) == pytest.approx(g.a, rel=1e-6)
    dt, dP = _grad_F(2 * g.tau_d, g.p_d + 10.0, g)
    assert dt == pytest.approx(1.0, rel=1e-6) and dP == pytest.approx(-CAP_k, rel=1e-6)
    t, P = 0.2 * g.tau_d, CAP_pT - 0.5
    R = math.hypot(t, P - g.p_y)
    dt, dP = _grad_F(t, P, g)
    assert dt == pytest.approx(g.a * t / R, rel=1e-6) and dP == pytest.approx(g.a * (P - g.p_y) / R, rel=1e-6)
    dtp, dPp = _grad_F(g.tau_d, g.p_d + 1e-4, g)
    dtm, dPm = _grad_F(g.tau_d, g.p_d - 1e-4, g)
    assert dtp == pytest.approx(dtm, rel=1e-4) and dPp == pytest.approx(dPm, rel=1e-4)
    assert dtp == pytest.approx(1.0, rel=1e-4) and dPp == pytest.approx(-CAP_k, rel=1e-4)


def test_pa_scale_geometry():
    # test/test_drucker_prager_cap.jl:233-253 (FP64): C = 10 MPa, tensile strength 5 MPa
    k, kq = math.sin(math.radians(30)), math.sin(math.radians(10))
    c, pT = 10.0e6 * math.cos(math.radians(30)), -5.0e6
    g = fem.cap_geometry(k, kq, c, pT)
    tol = math.sqrt(np.finfo(np.float64).eps)
    assert g.R_y == pytest.approx(g.p_y - pT, rel=1e-12)
    assert g.R_y == pytest.approx((k * g.p_y + c) / g.a, rel=tol)
    assert g.tau_d == pytest.approx(k * g.p_d + c, rel=tol)
    assert abs(fem.cap_yield_function(0.0, pT, k, c, g)) <= tol * g.R_y
    # the oracle's return at that scale: a hydrostatic tension beyond pT comes back to the cap
    ret = oh.cap_update(0, 0.0, 2 * pT, 1.0e10, 4.0e10, k, kq, c, pT, 0.0)
    assert ret["converged"][0] and ret["lambda"][0] > 0
    F, _, _ = fem.cap_invariants(ret["tau_II"][0], ret["P"][0], k, kq, c, pT)
    assert abs(F) <= 1e-12 * abs(pT)


def test_popov_2d_material_point():
    # test/test_popov_2d_material_point.jl: ϕ = 30°, ψ = 0, C = 20, pT = −1, ηve = 1, Kb·Δt = 64,
    # η_reg = 0.1
    phi = math.radians(30.0)
    k, kq, c, pT = math.sin(phi), 0.0, 20.0 * math.cos(phi), -1.0
    g = fem.cap_geometry(k, kq, c, pT)
    assert abs(fem.cap_yield_function(0.0, pT, k, c, g)) <= 1e-12
    el = oh.cap_update(0, 0.0, -0.5, 1.0, 64.0, k, kq, c, pT, 0.1)
    assert el["converged"][0] and el["lambda"][0] == 0.0 and el["P"][0] == -0.5
    y = oh.cap_update(0, 0.0, -1.2, 1.0, 64.0, k, kq, c, pT, 0.1)
    assert y["converged"][0] and y["lambda"][0] > 0 and -1.2 < y["P"][0] < pT
    # the plane-strain local update of a zero trial stress (η = G = Δt = 1: ηve = ½) returns
    # the same pressure, with the stress left at zero
    lu = oh.cap_update(3, np.zeros(3), -1.2, 0.5, 64.0, k, kq, c, pT, 0.1)
    assert (lu["tau"][0] == 0).all() and lu["P"][0] == pytest.approx(y["P"][0], rel=1e-12)
    # cohesion softening: C = 20, C_min = 5, H_C = −3
    assert fem.softened_cohesion(20.0, 5.0, -3.0, 0.0) == 20.0
    assert fem.softened_cohesion(20.0, 5.0, -3.0, 2.0) == 14.0
    assert fem.softened_cohesion(20.0, 5.0, -3.0, 10.0) == 5.0
    soft = fem.DruckerPragerCap((phi,), (0.0,), (20.0,), (pT,), (0.1,), (64.0,), C_min=(5.0,), H_C=(-3.0,))
    assert soft.C_min == (5.0,) and soft.H_C == (-3.0,)
    Cs = fem.softened_cohesion(soft.C[0], soft.C_min[0], soft.H_C[0], 2.0)
    ps = oh.cap_update(3, np.zeros(3), -1.2, 0.5, 64.0, k, kq, Cs * soft.cos_phi[0], pT, 0.1)
    ref = oh.cap_update(0, 0.0, -1.2, 1.0, 64.0, k, kq, 14.0 * math.cos(phi), pT, 0.1)
    assert ps["P"][0] == pytest.approx(ref["P"][0], rel=1e-12)
