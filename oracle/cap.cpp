// cap.cpp — TEST INFRASTRUCTURE ONLY: CPU oracle of the Drucker–Prager tensile cap
// (Popov, Berlie & Kaus 2025, GMD 18:7035; src/stokes/assemblers/rheology.jl:510-724),
// the parity checker of femb200_cap_update. The Newton Jacobian of the coupled return
// is taken with forward-mode dual numbers, as the reference's ForwardDiff.jacobian
// does, so it is an independent path to the library's closed-form derivatives.
// Pinned by the JustRelax fixtures and the identities of
// test/test_drucker_prager_cap.jl (tests/test_cap_oracle.py).
#include "oracle_core.hpp"
#include "../include/femtools_b200.h"

#include <algorithm>
#include <cmath>
#include <limits>

using namespace orc;

namespace {

constexpr double EPS = std::numeric_limits<double>::epsilon();
using D3 = Dual<3>;

inline D3 hypot(const D3& a, const D3& b) {
    D3 r;
    r.v = std::hypot(a.v, b.v);
    for (int i = 0; i < 3; ++i) r.d[i] = (a.v * a.d[i] + b.v * b.d[i]) / r.v;
    return r;
}
using std::hypot;

// cap_geometry (rheology.jl:556-567).
struct Geom { double a, b, p_y, R_y, p_d, t_d, p_q; };
Geom geometry(double k, double kq, double c, double pT) {
    Geom g;
    g.a = std::sqrt(1.0 + k * k);
    g.b = std::sqrt(1.0 + kq * kq);
    g.p_y = (g.a * pT + c) / (g.a - k);
    g.R_y = g.p_y - pT;
    g.p_d = g.p_y - g.R_y * k / g.a;
    g.t_d = g.R_y / g.a;
    g.p_q = g.p_d + kq * g.t_d;
    return g;
}

// cap_yield_function (rheology.jl:596-603) and cap_invariants (rheology.jl:614-622).
template <class S>
void invariants(const S& s, const S& p, double k, double kq, double c, const Geom& g, S& F, S& At, S& Ap) {
    if (val(p) + k * val(s) >= g.p_y) {
        F = s - k * p - c;
    } else {
        const S dp = p - g.p_y;
        F = g.a * (sqrt(s * s + dp * dp + EPS * EPS) - g.R_y);
    }
    if (val(p) + kq * val(s) >= g.p_q) {
        At = S(0.5);
        Ap = S(kq);
        return;
    }
    const S Rq = hypot(s, p - g.p_q);
    if (val(Rq) == 0.0) {
        At = S(0.0);
        Ap = S(0.0);
        return;
    }
    At = g.b * s / (2.0 * Rq);
    Ap = -g.b * (p - g.p_q) / Rq;
}

struct Ctx {
    double st, pt, eve, Kdt, k, kq, c, ereg, scale;
    Geom g;
};

// _cap_residual / scale (rheology.jl:624-628), with its Jacobian when J is non-null.
void residual(const Ctx& x, const double y[3], double r[3], double J[3][3]) {
    D3 s(y[0]), p(y[1]), lam(y[2]);
    s.d[0] = 1.0; p.d[1] = 1.0; lam.d[2] = 1.0;
    D3 F, At, Ap;
    invariants(s, p, x.k, x.kq, x.c, x.g, F, At, Ap);
    const D3 R[3] = {(s - x.st + 2.0 * x.eve * lam * At) / x.scale,
                     (p - x.pt - x.Kdt * lam * Ap) / x.scale,
                     (F - x.ereg * lam) / x.scale};
    for (int i = 0; i < 3; ++i) {
        r[i] = R[i].v;
        if (J)
            for (int j = 0; j < 3; ++j) J[i][j] = R[i].d[j];
    }
}

// A⁻¹ b by the adjugate (Cramer's rule).
void solve3(const double A[3][3], const double b[3], double x[3]) {
    const double c00 = A[1][1] * A[2][2] - A[1][2] * A[2][1];
    const double c01 = A[1][2] * A[2][0] - A[1][0] * A[2][2];
    const double c02 = A[1][0] * A[2][1] - A[1][1] * A[2][0];
    const double det = A[0][0] * c00 + A[0][1] * c01 + A[0][2] * c02;
    const double inv[3][3] = {
        {c00, A[0][2] * A[2][1] - A[0][1] * A[2][2], A[0][1] * A[1][2] - A[0][2] * A[1][1]},
        {c01, A[0][0] * A[2][2] - A[0][2] * A[2][0], A[0][2] * A[1][0] - A[0][0] * A[1][2]},
        {c02, A[0][1] * A[2][0] - A[0][0] * A[2][1], A[0][0] * A[1][1] - A[0][1] * A[1][0]}};
    for (int i = 0; i < 3; ++i) x[i] = (inv[i][0] * b[0] + inv[i][1] * b[1] + inv[i][2] * b[2]) / det;
}

struct Ret { double s, p, lam, At, Ap; bool converged; };

// cap_return_map (rheology.jl:640-698).
Ret return_map(double st, double pt, double eve, double Kdt, double k, double kq, double c, double pT, double ereg,
               int maxiter) {
    Ctx x{st, pt, eve, Kdt, k, kq, c, ereg, 1.0, geometry(k, kq, c, pT)};
    double F0, At0, Ap0;
    invariants(st, pt, k, kq, c, x.g, F0, At0, Ap0);
    Ret failed{st, pt, 0.0, At0, Ap0, false};
    if (F0 <= 0) return Ret{st, pt, 0.0, At0, Ap0, true};
    if (!(std::isfinite(Kdt) && Kdt > 0 && std::isfinite(eve) && eve > 0)) return failed;
    x.scale = std::max(std::max(std::fabs(st), std::fabs(pt)), std::max(std::fabs(F0), EPS));
    const double tol = 100 * EPS;
    double y[3] = {st, pt, 0.0}, r[3];
    residual(x, y, r, nullptr);
    auto norm_inf = [](const double* v) { return std::max(std::fabs(v[0]), std::max(std::fabs(v[1]), std::fabs(v[2]))); };
    bool converged = norm_inf(r) <= tol;
    for (int it = 0; it < maxiter; ++it) {
        if (converged) break;
        double J[3][3], rr[3], step[3];
        residual(x, y, rr, J);
        solve3(J, r, step);
        if (!(std::isfinite(step[0]) && std::isfinite(step[1]) && std::isfinite(step[2]))) return failed;
        double alpha = 1.0;
        bool accepted = false;
        const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        for (int ls = 0; ls < 24; ++ls) {
            const double cand[3] = {y[0] - alpha * step[0], y[1] - alpha * step[1], y[2] - alpha * step[2]};
            if (cand[0] >= 0 && cand[2] >= 0) {
                double rn[3];
                residual(x, cand, rn, nullptr);
                const double rn2 = rn[0] * rn[0] + rn[1] * rn[1] + rn[2] * rn[2];
                if (std::isfinite(rn[0]) && std::isfinite(rn[1]) && std::isfinite(rn[2]) &&
                    rn2 <= (1 - alpha / 10000) * r2) {
                    for (int i = 0; i < 3; ++i) { y[i] = cand[i]; r[i] = rn[i]; }
                    accepted = true;
                    break;
                }
            }
            alpha /= 2;
        }
        if (!accepted) return failed;
        converged = norm_inf(r) <= tol;
    }
    if (!converged) return failed;
    double J[3][3], rr[3], step[3];
    residual(x, y, rr, J);
    solve3(J, r, step);
    for (int i = 0; i < 3; ++i) y[i] -= step[i];
    double F, At, Ap;
    invariants(y[0], y[1], k, kq, c, x.g, F, At, Ap);
    return Ret{y[0], y[1], y[2], At, Ap, true};
}

// second_invariant (rheology.jl:206-212, :395-400).
double second_invariant(const double* t, int nc) {
    if (nc == 3) {
        const double zz = -t[0] - t[1];
        return std::sqrt((t[0] * t[0] + t[1] * t[1] + zz * zz) / 2 + t[2] * t[2] + EPS * EPS);
    }
    return std::sqrt((t[0] * t[0] + t[1] * t[1] + t[2] * t[2]) / 2 + t[3] * t[3] + t[4] * t[4] + t[5] * t[5] + EPS * EPS);
}

}  // namespace

extern "C" {

// femb200_cap_update on host arrays: cap_return_map (ncomp 0) or cap_local_update
// (rheology.jl:700-724) at every point.
int orc_cap_update(const femb200_cap_problem* p) {
    const int nc = p->ncomp;
    for (int64_t i = 0; i < p->n; ++i) {
        const double* tt = nc > 0 ? p->tau_trial + i * nc : nullptr;
        const double st = nc > 0 ? second_invariant(tt, nc) : p->s_trial[i];
        const double Pt = p->P_trial[i], eve = p->eta_ve[i], Kdt = p->K_dt[i];
        const Ret r = return_map(st, Pt, eve, Kdt, p->k[i], p->kq[i], p->c[i], p->pT[i], p->eta_reg[i], p->maxiter);
        const double lam = r.converged ? r.lam : std::numeric_limits<double>::quiet_NaN();
        const double gdot = lam * r.At, tdot = lam * r.Ap;
        if (p->tau && nc > 0)
            for (int j = 0; j < nc; ++j) p->tau[i * nc + j] = tt[j] - 2 * eve * gdot * tt[j] / st;
        if (p->tau_II) p->tau_II[i] = r.s;
        if (p->P) p->P[i] = nc > 0 ? Pt + Kdt * tdot : r.p;
        if (p->lambda) p->lambda[i] = r.lam;
        if (p->A_tau) p->A_tau[i] = r.At;
        if (p->A_p) p->A_p[i] = r.Ap;
        if (p->gamma_dot) p->gamma_dot[i] = gdot;
        if (p->theta_dot) p->theta_dot[i] = tdot;
        if (p->converged) p->converged[i] = r.converged ? 1 : 0;
    }
    return 0;
}

// cap_invariants(s, p, k, kq, c, pT) at n points of one material: F, Aτ, Ap.
int orc_cap_invariants(int64_t n, const double* s, const double* p, double k, double kq, double c, double pT,
                       double* F, double* At, double* Ap) {
    const Geom g = geometry(k, kq, c, pT);
    for (int64_t i = 0; i < n; ++i) invariants(s[i], p[i], k, kq, c, g, F[i], At[i], Ap[i]);
    return 0;
}

}  // extern "C"
