// cap.cuh — the Drucker–Prager tensile cap of Popov, Berlie & Kaus (2025), "A dilatant
// visco-elasto-viscoplasticity model with globally continuous tensile cap", GMD 18,
// 7035-7058 (src/stokes/assemblers/rheology.jl:510-724): cap geometry (their Eqs.
// 13-17), the composite yield function (Eq. 18), the flow coefficients and the coupled
// local return (Eq. 42). Pressure is compression-positive, so the tensile strength pT
// is ≤ 0. Every function returns its derivatives in (s, p) alongside its value, so the
// Newton Jacobian of the return is formed in closed form.
#pragma once
#include "common.cuh"

namespace femb {

template <class T> FEMB_HD T cap_eps();
template <> FEMB_HD double cap_eps<double>() { return 2.220446049250313e-16; }
template <> FEMB_HD float cap_eps<float>() { return 1.1920929e-07f; }

// The circle of radius R_y centred at (p_y, 0) of the meridional (P, τII) plane meets
// the pressure axis at pT and is tangent to τII = k·P + c at the delimiter (p_d, τ_d);
// the plastic potential's circle is centred at p_q. a = √(1 + k²), b = √(1 + kq²)
// make ‖∇F‖ = a and ‖∇Q‖ = b on both branches.
template <class T> struct CapGeom { T a, b, p_y, R_y, p_d, t_d, p_q; };

template <class T>
FEMB_HD CapGeom<T> cap_geometry(T k, T kq, T c, T pT) {
    CapGeom<T> g;
    g.a = sqrt(T(1) + k * k);
    g.b = sqrt(T(1) + kq * kq);
    g.p_y = (g.a * pT + c) / (g.a - k);   // R_y = p_y − pT and R_y = (k·p_y + c)/a
    g.R_y = g.p_y - pT;
    g.p_d = g.p_y - g.R_y * k / g.a;
    g.t_d = g.R_y / g.a;                   // = k·p_d + c by tangency
    g.p_q = g.p_d + kq * g.t_d;
    return g;
}

// Yield value, flow coefficients Aτ = ½ ∂Q/∂s and Ap = −∂Q/∂p, and the partial
// derivatives of each in (s, p). The yield and potential branches are chosen apart:
// the shear line where P + k·τII ≥ p_y (F = τII − k·P − c), else the cap
// F = a(√(τII² + (P − p_y)² + eps²) − R_y); the potential is linear where
// P + kq·τII ≥ p_q (Aτ = ½, Ap = kq), else circular about p_q with zero
// coefficients at its centre.
template <class T> struct CapFlow { T F, At, Ap, dF[2], dAt[2], dAp[2]; };

template <class T>
FEMB_HD CapFlow<T> cap_flow(T s, T p, T k, T kq, T c, const CapGeom<T>& g) {
    CapFlow<T> f;
    if (p + k * s >= g.p_y) {
        f.F = s - k * p - c;
        f.dF[0] = T(1);
        f.dF[1] = -k;
    } else {
        const T dp = p - g.p_y;
        const T R = sqrt(s * s + dp * dp + cap_eps<T>() * cap_eps<T>());
        const T aR = g.a / R;
        f.F = g.a * (R - g.R_y);
        f.dF[0] = aR * s;
        f.dF[1] = aR * dp;
    }
    f.dAt[0] = f.dAt[1] = f.dAp[0] = f.dAp[1] = T(0);
    if (p + kq * s >= g.p_q) {
        f.At = T(0.5);
        f.Ap = kq;
        return f;
    }
    const T d = p - g.p_q;
    const T R = hypot(s, d);
    if (R == T(0)) {
        f.At = f.Ap = T(0);
        return f;
    }
    // with u = s/R, w = d/R: Aτ = b·u/2, Ap = −b·w, ∂Aτ = b/(2R)·(w², −u·w),
    // ∂Ap = b/R·(u·w, −u²)
    const T iR = T(1) / R;
    const T u = s * iR, w = d * iR, bR = g.b * iR;
    f.At = T(0.5) * g.b * u;
    f.Ap = -g.b * w;
    f.dAt[0] = T(0.5) * bR * w * w;
    f.dAt[1] = -T(0.5) * bR * u * w;
    f.dAp[0] = bR * u * w;
    f.dAp[1] = -bR * u * u;
    return f;
}

// Scaled residual of the coupled return at y = (s, p, λ) and, when J is given, its
// Jacobian in (s, p, λ).
template <class T>
FEMB_HD void cap_residual(const T y[3], T st, T pt, T eve, T Kdt, T k, T kq, T c, T ereg, const CapGeom<T>& g,
                          T inv_scale, T r[3], T J[3][3]) {
    const CapFlow<T> f = cap_flow(y[0], y[1], k, kq, c, g);
    const T lam = y[2];
    r[0] = (y[0] - st + T(2) * eve * lam * f.At) * inv_scale;
    r[1] = (y[1] - pt - Kdt * lam * f.Ap) * inv_scale;
    r[2] = (f.F - ereg * lam) * inv_scale;
    if (!J) return;
    const T te = T(2) * eve * lam, kl = Kdt * lam;
    J[0][0] = (T(1) + te * f.dAt[0]) * inv_scale;
    J[0][1] = te * f.dAt[1] * inv_scale;
    J[0][2] = T(2) * eve * f.At * inv_scale;
    J[1][0] = -kl * f.dAp[0] * inv_scale;
    J[1][1] = (T(1) - kl * f.dAp[1]) * inv_scale;
    J[1][2] = -Kdt * f.Ap * inv_scale;
    J[2][0] = f.dF[0] * inv_scale;
    J[2][1] = f.dF[1] * inv_scale;
    J[2][2] = -ereg * inv_scale;
}

// x = A⁻¹ b for a 3×3 system by Gaussian elimination with partial pivoting (A is
// overwritten). The pivot row is found by conditional swaps with compile-time row
// indices, so the system stays in registers. A singular pivot gives non-finite entries.
template <class T>
FEMB_HD void cap_solve3(T A[3][3], const T b[3], T x[3]) {
    T r[3] = {b[0], b[1], b[2]};
    T ip[3];   // reciprocal pivots
#pragma unroll
    for (int col = 0; col < 3; ++col) {
#pragma unroll
        for (int i = col + 1; i < 3; ++i) {
            if (fabs(A[i][col]) > fabs(A[col][col])) {
#pragma unroll
                for (int j = 0; j < 3; ++j) { const T t = A[col][j]; A[col][j] = A[i][j]; A[i][j] = t; }
                const T t = r[col]; r[col] = r[i]; r[i] = t;
            }
        }
        ip[col] = T(1) / A[col][col];
#pragma unroll
        for (int i = col + 1; i < 3; ++i) {
            const T m = A[i][col] * ip[col];
#pragma unroll
            for (int j = col; j < 3; ++j) A[i][j] -= m * A[col][j];
            r[i] -= m * r[col];
        }
    }
#pragma unroll
    for (int i = 2; i >= 0; --i) {
        T acc = r[i];
#pragma unroll
        for (int j = i + 1; j < 3; ++j) acc -= A[i][j] * x[j];
        x[i] = acc * ip[i];
    }
}

template <class T> struct CapReturn { T s, p, lam, At, Ap; bool converged; };

// cap_return_map (rheology.jl:640-698).
template <class T>
FEMB_HD CapReturn<T> cap_return_map(T st, T pt, T eve, T Kdt, T k, T kq, T c, T pT, T ereg, int maxiter) {
    const CapGeom<T> g = cap_geometry(k, kq, c, pT);
    const CapFlow<T> f0 = cap_flow(st, pt, k, kq, c, g);
    CapReturn<T> out{st, pt, T(0), f0.At, f0.Ap, true};
    if (f0.F <= T(0)) return out;          // elastic
    out.converged = false;                 // the failure value: the trial state
    if (!(isfinite(Kdt) && Kdt > T(0) && isfinite(eve) && eve > T(0))) return out;
    const T scale = fmax(fmax(fabs(st), fabs(pt)), fmax(fabs(f0.F), cap_eps<T>()));
    const T inv_scale = T(1) / scale;
    const T tol = T(100) * cap_eps<T>();
    T x[3] = {st, pt, T(0)}, r[3], J[3][3];
    cap_residual(x, st, pt, eve, Kdt, k, kq, c, ereg, g, inv_scale, r, J);
    auto inf_norm = [](const T v[3]) { return fmax(fabs(v[0]), fmax(fabs(v[1]), fabs(v[2]))); };
    bool conv = inf_norm(r) <= tol;
    for (int it = 0; it < maxiter && !conv; ++it) {
        T step[3];
        cap_solve3(J, r, step);
        if (!(isfinite(step[0]) && isfinite(step[1]) && isfinite(step[2]))) return out;
        const T rr = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        T alpha = T(1);
        bool accepted = false;
        for (int ls = 0; ls < 24; ++ls) {
            const T cand[3] = {x[0] - alpha * step[0], x[1] - alpha * step[1], x[2] - alpha * step[2]};
            if (cand[0] >= T(0) && cand[2] >= T(0)) {
                T rn[3], Jn[3][3];
                cap_residual(cand, st, pt, eve, Kdt, k, kq, c, ereg, g, inv_scale, rn, Jn);
                const T rrn = rn[0] * rn[0] + rn[1] * rn[1] + rn[2] * rn[2];
                if (isfinite(rn[0]) && isfinite(rn[1]) && isfinite(rn[2]) && rrn <= (T(1) - alpha / T(10000)) * rr) {
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        x[i] = cand[i];
                        r[i] = rn[i];
#pragma unroll
                        for (int j = 0; j < 3; ++j) J[i][j] = Jn[i][j];
                    }
                    accepted = true;
                    break;
                }
            }
            alpha *= T(0.5);
        }
        if (!accepted) return out;
        conv = inf_norm(r) <= tol;
    }
    if (!conv) return out;
    // one more full Newton step at the converged point (a round-off change of the value)
    T step[3];
    cap_solve3(J, r, step);
    for (int i = 0; i < 3; ++i) x[i] -= step[i];
    const CapFlow<T> f = cap_flow(x[0], x[1], k, kq, c, g);
    return CapReturn<T>{x[0], x[1], x[2], f.At, f.Ap, true};
}

// second_invariant with the eps² floor (rheology.jl:206-212, :395-400): plane strain
// carries τzz = −τxx − τyy.
template <class T>
FEMB_HD T cap_second_invariant(const T* t, int ncomp) {
    if (ncomp == 3) {
        const T zz = -t[0] - t[1];
        return sqrt((t[0] * t[0] + t[1] * t[1] + zz * zz) / T(2) + t[2] * t[2] + cap_eps<T>() * cap_eps<T>());
    }
    return sqrt((t[0] * t[0] + t[1] * t[1] + t[2] * t[2]) / T(2) + t[3] * t[3] + t[4] * t[4] + t[5] * t[5] +
                cap_eps<T>() * cap_eps<T>());
}

}  // namespace femb
