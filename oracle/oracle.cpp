// oracle.cpp — TEST INFRASTRUCTURE ONLY: the CPU oracle of the dynamic-relaxation
// hot path. It is the parity checker for libfemtools_b200 and the timed CPU
// baseline; the product library never links it. Host pointers throughout; the
// argument structs are those of include/femtools_b200.h so that a test hands
// identical problems to both implementations.
//
// Parallelism: element work runs under OpenMP into per-element buffers and is
// scattered in element order afterwards, so results do not depend on the thread
// count (the reference's CPU() backend accumulates in element order as well).
#include "oracle_core.hpp"
#include "../include/femtools_b200.h"

#include <cstdio>
#include <cstdlib>
#include <string>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace orc;

namespace {

constexpr double EPS2 = std::numeric_limits<double>::epsilon() * std::numeric_limits<double>::epsilon();

thread_local std::string g_last_error;

inline const double* D(const void* p) { return static_cast<const double*>(p); }
// Julia's eps(x): the spacing of floats at |x|.
inline double julia_eps(double x) { x = std::fabs(x); return std::nextafter(x, INFINITY) - x; }
// max / min with Julia's semantics: NaN when either argument is NaN. std::max and
// std::min return their first argument when a comparison with NaN fails, which would
// hide a NaN residual from the reference's isnan / isfinite exits.
inline double jl_max(double a, double b) { return (std::isnan(a) || std::isnan(b)) ? NAN : std::max(a, b); }
inline double jl_min(double a, double b) { return (std::isnan(a) || std::isnan(b)) ? NAN : std::min(a, b); }
inline double* Dm(void* p) { return static_cast<double*>(p); }

// _phase_at (src/utils.jl:70-72): returns a 0-based phase index.
inline int phase_at(const int32_t* phases, int layout, int64_t node1, int i, int64_t iel, int n) {
    if (!phases) return 0;
    if (layout == FEMB200_PHASE_CELL) return phases[iel] - 1;
    if (layout == FEMB200_PHASE_ELEMENT_NODE) return phases[(int64_t)n * iel + i] - 1;
    return phases[node1 - 1] - 1;
}

// interp2ip_phase (src/utils.jl:37-44).
template <class S = double>
inline double interp_phase(const double* N, const double* var, const int* ph, int n) {
    double out = 0;
    for (int a = 0; a < n; ++a) out += N[a] * var[ph[a]];
    return out;
}

// Element-local data of one Stokes element (momentum_element_residual,
// src/stokes/assemblers/momentum_residuals.jl:497-528; pressure_element_residual,
// src/stokes/assemblers/pressure_residual.jl:306-326).
struct Elem {
    int D, NV, NP, NQ;
    int64_t iel;
    int64_t nodes[27];   // 1-based
    int64_t dofs[4];     // 1-based pressure DoFs
    double P[4], P0[4], T[4], T0[4], Q[4], Pf[4], Pnum[4], gam[4], MP[4];
    bool hasQ, hasPf;
    bool P0_ip; double P0q[27];
    int phv[27], php[4];
    const double* geo;   // NQ × (D²+1)
    const double* geoP;  // NQ
    bool has_told; double told[27][6];
    bool eta_ip; double etaq_ip[27];
};

void gather(const femb200_stokes_problem* p, int64_t e, Elem& el, bool need_P0 = true) {
    const Tables& t = tables_for(p->dim);
    el.D = p->dim; el.NV = t.nv; el.NP = t.np; el.NQ = t.nq; el.iel = e;
    const int NV = el.NV, NP = el.NP, NQ = el.NQ, DD = el.D;
    for (int a = 0; a < NV; ++a) el.nodes[a] = p->el2n[(int64_t)NV * e + a];
    for (int i = 0; i < NP; ++i) el.dofs[i] = p->dofsP[(int64_t)NP * e + i];
    for (int i = 0; i < NP; ++i) {
        int64_t d = el.dofs[i] - 1;
        el.P[i] = D(p->P)[d];
        el.T[i] = p->T ? D(p->T)[d] : 0.0;
        el.T0[i] = p->T0 ? D(p->T0)[d] : 0.0;
        el.Q[i] = p->Q ? D(p->Q)[d] : 0.0;
        el.Pf[i] = p->Pf ? D(p->Pf)[d] : 0.0;
        el.Pnum[i] = p->Pnum ? D(p->Pnum)[d] : 0.0;
        el.gam[i] = p->gammaP ? D(p->gammaP)[d] : 0.0;
        el.MP[i] = p->M_P ? D(p->M_P)[d] : 1.0;
    }
    el.hasQ = p->Q != nullptr; el.hasPf = p->Pf != nullptr;
    el.P0_ip = false;
    if (need_P0) {
        if (p->P_old && p->P_old_layout == FEMB200_FIELD_IP) {
            el.P0_ip = true;
            for (int q = 0; q < NQ; ++q) el.P0q[q] = D(p->P_old)[(int64_t)NQ * e + q];
        } else {
            const double* src = p->P_old ? D(p->P_old) : D(p->P0);
            for (int i = 0; i < NP; ++i) el.P0[i] = src ? src[el.dofs[i] - 1] : 0.0;
        }
    }
    for (int a = 0; a < NV; ++a) el.phv[a] = phase_at(p->phases_v, p->phases_v_layout, el.nodes[a], a, e, NV);
    for (int i = 0; i < NP; ++i) el.php[i] = phase_at(p->phases_P, p->phases_P_layout, el.dofs[i], i, e, NP);
    el.geo = D(p->geo_v) + (int64_t)e * NQ * (DD * DD + 1);
    el.geoP = D(p->geo_P) + (int64_t)e * NQ;
    const int NT = DD == 3 ? 6 : 3;
    el.has_told = p->tau_old_layout != FEMB200_FIELD_NONE && p->tau_old[0];
    for (int q = 0; q < NQ; ++q)
        for (int c = 0; c < NT; ++c) {
            double v = 0;
            if (el.has_told) {
                if (p->tau_old_layout == FEMB200_FIELD_IP) v = D(p->tau_old[c])[(int64_t)NQ * e + q];
                else {  // nodal history interpolated with the velocity shape functions (rheology.jl:47)
                    for (int a = 0; a < NV; ++a) v += t.N[q][a] * D(p->tau_old[c])[el.nodes[a] - 1];
                }
            }
            el.told[q][c] = v;
        }
    el.eta_ip = p->viscosity_ip != nullptr;
    if (el.eta_ip)
        for (int q = 0; q < NQ; ++q) el.etaq_ip[q] = D(p->viscosity_ip)[(int64_t)NQ * e + q];
}

// Physical gradients ∂N∂x = ∂N∂ξ · J⁻¹ at quadrature point q (mesh.jl:504-507).
inline void dNdx_at(const Tables& t, const double* geo, int D, int q, double out[27][3]) {
    const double* Ji = geo + q * (D * D + 1);
    for (int a = 0; a < t.nv; ++a)
        for (int k = 0; k < D; ++k) {
            double s = 0;
            for (int j = 0; j < D; ++j) s += t.dN[q][a][j] * Ji[j + D * k];
            out[a][k] = s;
        }
}

struct Plastic {
    double cphi, sphi, spsi, C, ereg, Kb;
};

// Maxwell coefficients (viscoelastic_coefficients_phase, rheology.jl:35-42).
inline void ve_coeffs(const double* N, double etaq, const double* G, const int* ph, int n, double dt,
                      double& etave, double& inv2Gdt) {
    double invG[FEMB200_MAX_PHASES];
    for (int i = 0; i < FEMB200_MAX_PHASES; ++i) invG[i] = 1.0 / G[i];
    double invGq = interp_phase(N, invG, ph, n);
    etave = 1.0 / (1.0 / etaq + invGq / dt);
    inv2Gdt = invGq / (2 * dt);
}

// 3-D stress with optional Drucker–Prager return (rheology.jl:413-472).
// grad[i][k] = ∂v_i/∂x_k. Returns λ through lam_out.
// SE (the Maxwell viscosity) and SP (the pressure) may be dual numbers as well,
// for the adjoint checks that differentiate with respect to them.
template <class S, class SE = double, class SP = double>
void stress3d(const S grad[3][3], SE etave, double inv2Gdt, const double told[6], const Plastic* pl,
              SP Pq, S tau[6], double* lam_out) {
    S tr = (grad[0][0] + grad[1][1] + grad[2][2]) / 3.0;
    S eps[6] = {grad[0][0] - tr, grad[1][1] - tr, grad[2][2] - tr,
                (grad[0][1] + grad[1][0]) / 2.0, (grad[0][2] + grad[2][0]) / 2.0, (grad[1][2] + grad[2][1]) / 2.0};
    for (int c = 0; c < 6; ++c) tau[c] = (2.0 * etave) * (eps[c] + told[c] * inv2Gdt);
    double lam_v = 0;
    if (pl) {
        S tII = sqrt((tau[0] * tau[0] + tau[1] * tau[1] + tau[2] * tau[2]) / 2.0 + tau[3] * tau[3] + tau[4] * tau[4] +
                     tau[5] * tau[5] + EPS2);
        S tIIs = tII + EPS2;
        S F = tII - pl->cphi * pl->C - pl->sphi * Pq;
        double dFdP = -pl->sphi, dQdP = -pl->spsi;
        S dQ[6] = {tau[0] / (2.0 * tIIs), tau[1] / (2.0 * tIIs), tau[2] / (2.0 * tIIs),
                   tau[3] / tIIs, tau[4] / tIIs, tau[5] / tIIs};
        S lam = val(F) > 0 ? F / (etave + pl->ereg + pl->Kb * 1.0 * dQdP * dFdP) : S(0.0);
        lam_v = val(lam);
        if (val(lam) > 0)
            for (int c = 0; c < 6; ++c) tau[c] = tau[c] - (2.0 * etave) * lam * dQ[c];
    }
    if (lam_out) *lam_out = lam_v;
}

// Plane-strain stress with the plane-strain Drucker–Prager return (rheology.jl:226-334).
template <class S>
void stress2d(const S grad[2][2], double etave, double inv2Gdt, const double told[3], const Plastic* pl,
              double Pq, S tau[3], double* lam_out) {
    S exx = grad[0][0], eyy = grad[1][1];
    S exy = (grad[0][1] + grad[1][0]) / 2.0;
    S tr = (exx + eyy) / 3.0;
    tau[0] = (2 * etave) * ((exx - tr) + told[0] * inv2Gdt);
    tau[1] = (2 * etave) * ((eyy - tr) + told[1] * inv2Gdt);
    tau[2] = (2 * etave) * (exy + told[2] * inv2Gdt);
    double lam_v = 0;
    if (pl) {
        S tzz = S(0.0) - tau[0] - tau[1];
        S tII = sqrt((tau[0] * tau[0] + tau[1] * tau[1] + tzz * tzz) / 2.0 + tau[2] * tau[2] + EPS2);
        S tIIs = tII + EPS2;
        S F = tII - pl->cphi * pl->C - pl->sphi * Pq;
        double dFdP = -pl->sphi, dQdP = -pl->spsi;
        S dQ[3] = {(2.0 * tau[0] + tau[1]) / (2.0 * tIIs), (tau[0] + 2.0 * tau[1]) / (2.0 * tIIs), tau[2] / tIIs};
        S lam = val(F) > 0 ? F / (etave + pl->ereg + pl->Kb * 1.0 * dQdP * dFdP) : S(0.0);
        lam_v = val(lam);
        if (val(lam) > 0)
            for (int c = 0; c < 3; ++c) tau[c] = tau[c] - (2 * etave) * lam * dQ[c];
    }
    if (lam_out) *lam_out = lam_v;
}

inline Plastic plastic_at(const femb200_stokes_material& m, const double* N, const int* ph, int n, double dt) {
    Plastic pl;
    pl.cphi = interp_phase(N, m.cos_phi, ph, n);
    pl.sphi = interp_phase(N, m.sin_phi, ph, n);
    pl.spsi = interp_phase(N, m.sin_psi, ph, n);
    pl.C = interp_phase(N, m.C, ph, n);
    pl.ereg = interp_phase(N, m.eta_reg, ph, n);
    pl.Kb = interp_phase(N, m.Kb, ph, n) * dt;  // Kb·Δt, multiplied as in rheology.jl:468
    return pl;
}

// integrate_PH_pressure_residual (pressure_residual.jl:132-158). `bulk` is ηb or K.
template <class S>
void pressure_element(const Tables& t, const Elem& el, const S v[3][27], const double* bulk, const double* alpha,
                      double dt, bool use_Q, S RP[4]) {
    const int D = el.D, NP = el.NP;
    for (int i = 0; i < NP; ++i) RP[i] = S(0.0);
    bool all_inf = true;
    for (int ph = 0; ph < FEMB200_MAX_PHASES; ++ph) if (!std::isinf(bulk[ph])) { all_inf = false; break; }
    double dNdx[27][3];
    for (int q = 0; q < el.NQ; ++q) {
        dNdx_at(t, el.geo, D, q, dNdx);
        double dO = el.geoP[q];
        const double* Nv = t.NP[q];
        double Qq = 0;
        if (use_Q) for (int i = 0; i < NP; ++i) Qq += Nv[i] * el.Q[i];
        double ebq = all_inf ? INFINITY : interp_phase(Nv, bulk, el.php, NP);
        double aq = interp_phase(Nv, alpha, el.php, NP);
        double dPinc = 0;
        if (el.P0_ip) { for (int i = 0; i < NP; ++i) dPinc += Nv[i] * el.P[i]; dPinc -= el.P0q[q]; }
        else for (int i = 0; i < NP; ++i) dPinc += Nv[i] * (el.P[i] - el.P0[i]);
        double dPdt = dPinc / (ebq * dt);
        double dT = 0;
        for (int i = 0; i < NP; ++i) dT += Nv[i] * (el.T[i] - el.T0[i]);
        double dTdt = aq * dT / dt;
        S div(0.0);
        for (int j = 0; j < D; ++j)
            for (int a = 0; a < el.NV; ++a) div = div + dNdx[a][j] * v[j][a];
        for (int i = 0; i < NP; ++i) RP[i] = RP[i] + Nv[i] * ((S(0.0) - div - dPdt + dTdt + Qq) * dO);
    }
}

// integrate_momentum_residual 3-D (momentum_residuals.jl:209-258) and plane strain
// (:136-189). `eta_ph` is the per-phase viscosity table (the material's, or the
// element-max table of the Jacobian diagnostics); `eta_const` > 0 replaces it
// with one value (the viscosity-matrix path of the diagnostics).
template <class S>
void momentum_element(const Tables& t, const Elem& el, const femb200_stokes_material& m, const S v[3][27],
                      const S* Pnum /*NP or null*/, const double* eta_ph, double eta_const, double dt,
                      S R[3][27], double* tau_store, int64_t nq_stride) {
    const int D = el.D, NV = el.NV, NP = el.NP, NQ = el.NQ;
    for (int c = 0; c < D; ++c) for (int a = 0; a < NV; ++a) R[c][a] = S(0.0);
    double beta[FEMB200_MAX_PHASES];
    for (int i = 0; i < FEMB200_MAX_PHASES; ++i) beta[i] = 1.0 / m.K[i];
    double dNdx[27][3];
    for (int q = 0; q < NQ; ++q) {
        dNdx_at(t, el.geo, D, q, dNdx);
        double dO = el.geo[q * (D * D + 1) + D * D];
        const double* Nv = t.N[q];
        const double* NPq = t.NP[q];
        double Pq = 0; for (int i = 0; i < NP; ++i) Pq += NPq[i] * el.P[i];
        double Pfq = 0; if (el.hasPf) for (int i = 0; i < NP; ++i) Pfq += NPq[i] * el.Pf[i];
        double Peq = el.hasPf ? Pq - Pfq : Pq;
        double etaq = eta_const > 0 ? eta_const : (el.eta_ip ? el.etaq_ip[q] : interp_phase(Nv, eta_ph, el.phv, NV));
        double etave, inv2Gdt;
        ve_coeffs(Nv, etaq, m.G, el.phv, NV, dt, etave, inv2Gdt);
        Plastic pl; const Plastic* plp = nullptr;
        if (m.plastic) { pl = plastic_at(m, Nv, el.phv, NV, dt); plp = &pl; }
        S grad[3][3];
        for (int i = 0; i < D; ++i)
            for (int k = 0; k < D; ++k) {
                S s(0.0);
                for (int a = 0; a < NV; ++a) s = s + dNdx[a][k] * v[i][a];
                grad[i][k] = s;
            }
        S sig[3][3];
        if (D == 3) {
            S tau[6];
            stress3d(grad, etave, inv2Gdt, el.told[q], plp, Peq, tau, nullptr);
            if (tau_store) for (int c = 0; c < 6; ++c) tau_store[c * nq_stride + q] = val(tau[c]);
            sig[0][0] = tau[0]; sig[1][1] = tau[1]; sig[2][2] = tau[2];
            sig[0][1] = sig[1][0] = tau[3]; sig[0][2] = sig[2][0] = tau[4]; sig[1][2] = sig[2][1] = tau[5];
        } else {
            S g2[2][2] = {{grad[0][0], grad[0][1]}, {grad[1][0], grad[1][1]}};
            S tau[3];
            stress2d(g2, etave, inv2Gdt, el.told[q], plp, Peq, tau, nullptr);
            if (tau_store) for (int c = 0; c < 3; ++c) tau_store[c * nq_stride + q] = val(tau[c]);
            sig[0][0] = tau[0]; sig[1][1] = tau[1]; sig[0][1] = sig[1][0] = tau[2];
        }
        // Pq_local = total pressure after the yield model (unchanged by DruckerPrager).
        S Ptot = S(el.hasPf ? Peq + Pfq : Pq);
        if (Pnum) { S pn(0.0); for (int i = 0; i < NP; ++i) pn = pn + NPq[i] * Pnum[i]; Ptot = Ptot + pn; }
        double Tq = 0; for (int i = 0; i < NP; ++i) Tq += NPq[i] * el.T[i];
        // eos_density (momentum_residuals.jl:11-16)
        double rhoq = interp_phase(Nv, m.rho0, el.phv, NV) *
                      (1 - interp_phase(Nv, m.alpha, el.phv, NV) * (Tq - m.Tref) + interp_phase(Nv, beta, el.phv, NV) * Pq);
        // accumulate_momentum (momentum_residuals.jl:28-33)
        for (int i = 0; i < D; ++i) {
            double bg = rhoq * m.g[i];
            for (int a = 0; a < NV; ++a) {
                S s(0.0);
                for (int j = 0; j < D; ++j) s = s + dNdx[a][j] * (j == i ? sig[j][i] - Ptot : sig[j][i]);
                R[i][a] = R[i][a] + (s - Nv[a] * bg) * dO;
            }
        }
    }
}

template <class S>
void load_v(const femb200_stokes_problem* p, const Elem& el, S v[3][27]) {
    for (int c = 0; c < el.D; ++c)
        for (int a = 0; a < el.NV; ++a) v[c][a] = S(D(p->v[c])[el.nodes[a] - 1]);
    for (int c = el.D; c < 3; ++c) for (int a = 0; a < 27; ++a) v[c][a] = S(0.0);
}

inline const double* bulk_table(const femb200_stokes_problem* p, int finite_K) {
    return finite_K ? p->mat.K : p->mat.eta_b;
}

int check_problem(const femb200_stokes_problem* p) {
    if (!p) { g_last_error = "null problem"; return FEMB200_EINVAL; }
    if (!((p->dim == 3 && p->nv == 27 && p->np == 4 && p->nq == 27) || (p->dim == 2 && p->nv == 9 && p->np == 3 && p->nq == 9))) {
        g_last_error = "oracle supports Hex27/P1 (3-D) and Q9/P1 (2-D) only"; return FEMB200_EUNSUPPORTED;
    }
    if (p->dtype != FEMB200_F64 || p->geo_dtype != FEMB200_F64) { g_last_error = "oracle is FP64 only"; return FEMB200_EUNSUPPORTED; }
    if (p->mat.nphases < 1 || p->mat.nphases > FEMB200_MAX_PHASES) { g_last_error = "bad nphases"; return FEMB200_EINVAL; }
    return FEMB200_OK;
}

// ---- assemblies -----------------------------------------------------------

void pressure_residual_impl(const femb200_stokes_problem* p, double dt, int finite_K) {
    const Tables& t = tables_for(p->dim);
    double* RP = Dm(p->RP);
    std::fill(RP, RP + p->nnodesP, 0.0);
    const double* bulk = bulk_table(p, finite_K);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < p->nels; ++e) {
        Elem el; gather(p, e, el);
        double v[3][27]; load_v(p, el, v);
        double R[4];
        pressure_element<double>(t, el, v, bulk, p->mat.alpha, dt, p->Q != nullptr, R);
        for (int i = 0; i < el.NP; ++i) RP[el.dofs[i] - 1] += R[i];  // element-private DoFs
    }
}

void momentum_residual_impl(const femb200_stokes_problem* p, double dt, bool with_pnum, double** tau_store_cols = nullptr) {
    const Tables& t = tables_for(p->dim);
    const int NV = t.nv, Dm_ = p->dim;
    std::vector<double> buf((size_t)p->nels * NV * Dm_);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < p->nels; ++e) {
        Elem el; gather(p, e, el, false);
        double v[3][27]; load_v(p, el, v);
        double R[3][27];
        double pn[4]; for (int i = 0; i < el.NP; ++i) pn[i] = el.Pnum[i];
        double tstore[6 * 27];
        momentum_element<double>(t, el, p->mat, v, with_pnum ? pn : nullptr, p->mat.eta, 0.0, dt, R,
                                 tau_store_cols ? tstore : nullptr, 27);
        if (tau_store_cols) {
            const int NT = Dm_ == 3 ? 6 : 3;
            for (int c = 0; c < NT; ++c)
                for (int q = 0; q < el.NQ; ++q) tau_store_cols[c][(int64_t)el.NQ * e + q] = tstore[c * 27 + q];
        }
        double* b = &buf[(size_t)e * NV * Dm_];
        for (int c = 0; c < Dm_; ++c) for (int a = 0; a < NV; ++a) b[c * NV + a] = R[c][a];
    }
    for (int c = 0; c < Dm_; ++c) std::fill(Dm(p->Rv[c]), Dm(p->Rv[c]) + p->nnodes, 0.0);
    for (int64_t e = 0; e < p->nels; ++e) {
        const double* b = &buf[(size_t)e * NV * Dm_];
        for (int a = 0; a < NV; ++a) {
            int64_t n = p->el2n[(int64_t)NV * e + a] - 1;
            for (int c = 0; c < Dm_; ++c) Dm(p->Rv[c])[n] += b[c * NV + a];
        }
    }
}

// Augmented Jacobian diagnostics (momentum_residuals.jl:929-970, 1044-1117).
// Elements [e0, e1) only when a range is given (the timed CPU sample assembles the
// full-size arrays one block of elements at a time).
template <int NVT>
void jacobian_impl_t(const femb200_stokes_problem* p, double dt, int finite_K, int64_t e0, int64_t e1) {
    using DU = Dual<NVT>;
    const Tables& t = tables_for(p->dim);
    const int NV = t.nv, DD = p->dim;
    std::vector<double> buf((size_t)(e1 - e0) * NV * DD * 2);
    const double* bulk = bulk_table(p, finite_K);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t e = e0; e < e1; ++e) {
        Elem el; gather(p, e, el);
        // The diagnostics read dr.P0 for the pressure storage term (DR.jl:468).
        el.P0_ip = false;
        for (int i = 0; i < el.NP; ++i) el.P0[i] = p->P0 ? D(p->P0)[el.dofs[i] - 1] : 0.0;
        // η_pc: element-max viscosity (_element_max_phase_property, momentum_residuals.jl:36-44).
        double eta_pc[FEMB200_MAX_PHASES];
        double eta_const = 0;
        if (el.eta_ip) {
            eta_const = el.etaq_ip[0];
            for (int q = 1; q < el.NQ; ++q) eta_const = std::max(eta_const, el.etaq_ip[q]);
        } else {
            double mx = p->mat.eta[el.phv[0]];
            for (int a = 1; a < NV; ++a) mx = std::max(mx, p->mat.eta[el.phv[a]]);
            for (int i = 0; i < FEMB200_MAX_PHASES; ++i) eta_pc[i] = mx;
        }
        double vd[3][27]; load_v(p, el, vd);
        double rows[3][27] = {{0}}, diag[3][27] = {{0}};
        for (int j = 0; j < DD; ++j) {   // direction differentiated (the block column)
            DU v[3][27];
            for (int c = 0; c < 3; ++c) for (int a = 0; a < 27; ++a) v[c][a] = DU(vd[c][a]);
            for (int b = 0; b < NV; ++b) v[j][b].d[b] = 1.0;
            DU RP[4];
            pressure_element<DU>(t, el, v, bulk, p->mat.alpha, dt, false, RP);
            DU pn[4];
            for (int i = 0; i < el.NP; ++i) pn[i] = (el.gam[i] * RP[i]) / el.MP[i];
            DU R[3][27];
            momentum_element<DU>(t, el, p->mat, v, pn, eta_pc, eta_const, dt, R, nullptr, 27);
            for (int i = 0; i < DD; ++i)
                for (int a = 0; a < NV; ++a) {
                    double s = 0;
                    for (int b = 0; b < NV; ++b) s += std::fabs(R[i][a].d[b]);
                    rows[i][a] += s;
                    if (i == j) diag[i][a] = std::fabs(R[i][a].d[a]);
                }
        }
        double* o = &buf[(size_t)(e - e0) * NV * DD * 2];
        for (int i = 0; i < DD; ++i)
            for (int a = 0; a < NV; ++a) { o[(i * NV + a) * 2] = rows[i][a]; o[(i * NV + a) * 2 + 1] = diag[i][a]; }
    }
    for (int c = 0; c < DD; ++c) {
        std::fill(Dm(p->dRdv[c]), Dm(p->dRdv[c]) + p->nnodes, 0.0);
        std::fill(Dm(p->PC[c]), Dm(p->PC[c]) + p->nnodes, 0.0);
    }
    for (int64_t e = e0; e < e1; ++e) {
        const double* o = &buf[(size_t)(e - e0) * NV * DD * 2];
        for (int i = 0; i < DD; ++i)
            for (int a = 0; a < NV; ++a) {
                int64_t n = p->el2n[(int64_t)NV * e + a] - 1;
                Dm(p->dRdv[i])[n] += o[(i * NV + a) * 2];
                Dm(p->PC[i])[n] += o[(i * NV + a) * 2 + 1];
            }
    }
}

void jacobian_impl(const femb200_stokes_problem* p, double dt, int finite_K, int64_t e0 = 0, int64_t e1 = -1) {
    if (e1 < 0) e1 = p->nels;
    if (p->dim == 3) jacobian_impl_t<27>(p, dt, finite_K, e0, e1);
    else jacobian_impl_t<9>(p, dt, finite_K, e0, e1);
}

// ---- adjoint checks -----------------------------------------------------------
// The whole Hex27 Stokes element residual with every input a scalar of type S: the
// velocities, the element's pressure DoFs and the viscosity at each quadrature
// point. Rv carries Pnum = γP·RP/M_P formed inline from the element's own RP (the
// augmented residual the DR loop drives to zero, DR.jl:674-676), RP is the
// continuity residual. It restates pressure_element and momentum_element with
// those inputs typed S so that forward-mode duals can seed any of them; the
// reference's adjoint operator (FrozenAdjointOperator,
// src/stokes/assemblers/adjoint_operator.jl:3-73, applied at :640-660) is the
// transpose of this function's Jacobian.
template <class S>
void stokes_element_all(const Tables& t, const Elem& el, const femb200_stokes_material& m, const S v[3][27],
                        const S Pe[4], const S etaq[27], const double* bulk, double dt, bool with_pnum, S Rv[3][27],
                        S RP[4]) {
    const int D = 3, NV = 27, NP = 4, NQ = 27;
    bool all_inf = true;
    for (int ph = 0; ph < FEMB200_MAX_PHASES; ++ph) if (!std::isinf(bulk[ph])) { all_inf = false; break; }
    double beta[FEMB200_MAX_PHASES];
    for (int i = 0; i < FEMB200_MAX_PHASES; ++i) beta[i] = 1.0 / m.K[i];
    double dNdx[27][3];
    // pressure residual (pressure_residual.jl:132-158)
    for (int i = 0; i < NP; ++i) RP[i] = S(0.0);
    for (int q = 0; q < NQ; ++q) {
        dNdx_at(t, el.geo, D, q, dNdx);
        const double dO = el.geoP[q];
        const double* Nv = t.NP[q];
        const double ebq = all_inf ? INFINITY : interp_phase(Nv, bulk, el.php, NP);
        const double aq = interp_phase(Nv, m.alpha, el.php, NP);
        S dPinc(0.0);
        if (el.P0_ip) { for (int i = 0; i < NP; ++i) dPinc = dPinc + Nv[i] * Pe[i]; dPinc = dPinc - el.P0q[q]; }
        else for (int i = 0; i < NP; ++i) dPinc = dPinc + Nv[i] * (Pe[i] - el.P0[i]);
        const S dPdt = all_inf ? S(0.0) : dPinc / (ebq * dt);
        double dT = 0;
        for (int i = 0; i < NP; ++i) dT += Nv[i] * (el.T[i] - el.T0[i]);
        const double dTdt = aq * dT / dt;
        S div(0.0);
        for (int j = 0; j < D; ++j)
            for (int a = 0; a < NV; ++a) div = div + dNdx[a][j] * v[j][a];
        for (int i = 0; i < NP; ++i) RP[i] = RP[i] + Nv[i] * ((S(0.0) - div - dPdt + dTdt) * dO);
    }
    S pn[4];
    for (int i = 0; i < NP; ++i) pn[i] = with_pnum ? (el.gam[i] * RP[i]) / el.MP[i] : S(0.0);
    // momentum residual (momentum_residuals.jl:209-258)
    for (int c = 0; c < D; ++c) for (int a = 0; a < NV; ++a) Rv[c][a] = S(0.0);
    double invG[FEMB200_MAX_PHASES];
    for (int i = 0; i < FEMB200_MAX_PHASES; ++i) invG[i] = 1.0 / m.G[i];
    for (int q = 0; q < NQ; ++q) {
        dNdx_at(t, el.geo, D, q, dNdx);
        const double dO = el.geo[q * (D * D + 1) + D * D];
        const double* Nv = t.N[q];
        const double* NPq = t.NP[q];
        S Pq(0.0); for (int i = 0; i < NP; ++i) Pq = Pq + NPq[i] * Pe[i];
        double Pfq = 0; if (el.hasPf) for (int i = 0; i < NP; ++i) Pfq += NPq[i] * el.Pf[i];
        const S Peq = el.hasPf ? Pq - Pfq : Pq;
        const double invGq = interp_phase(Nv, invG, el.phv, NV);
        const S etave = 1.0 / (1.0 / etaq[q] + invGq / dt);
        const double inv2Gdt = invGq / (2 * dt);
        Plastic pl; const Plastic* plp = nullptr;
        if (m.plastic) { pl = plastic_at(m, Nv, el.phv, NV, dt); plp = &pl; }
        S grad[3][3];
        for (int i = 0; i < D; ++i)
            for (int k = 0; k < D; ++k) {
                S g(0.0);
                for (int a = 0; a < NV; ++a) g = g + dNdx[a][k] * v[i][a];
                grad[i][k] = g;
            }
        S tau[6];
        stress3d<S, S, S>(grad, etave, inv2Gdt, el.told[q], plp, Peq, tau, nullptr);
        const S sig[3][3] = {{tau[0], tau[3], tau[4]}, {tau[3], tau[1], tau[5]}, {tau[4], tau[5], tau[2]}};
        S Ptot = el.hasPf ? Peq + Pfq : Pq;
        S pq(0.0); for (int i = 0; i < NP; ++i) pq = pq + NPq[i] * pn[i];
        Ptot = Ptot + pq;
        double Tq = 0; for (int i = 0; i < NP; ++i) Tq += NPq[i] * el.T[i];
        const S rhoq = interp_phase(Nv, m.rho0, el.phv, NV) *
                       (1.0 - interp_phase(Nv, m.alpha, el.phv, NV) * (Tq - m.Tref) + interp_phase(Nv, beta, el.phv, NV) * Pq);
        for (int i = 0; i < D; ++i) {
            const S bg = rhoq * m.g[i];
            for (int a = 0; a < NV; ++a) {
                S sa(0.0);
                for (int j = 0; j < D; ++j) sa = sa + dNdx[a][j] * (j == i ? sig[j][i] - Ptot : sig[j][i]);
                Rv[i][a] = Rv[i][a] + (sa - Nv[a] * bg) * dO;
            }
        }
    }
}

// Viscosity at each quadrature point: the given per-point field, or the phase
// interpolation of the material's (interp2ip_phase, src/utils.jl:37-44).
void element_viscosity(const Tables& t, const Elem& el, const femb200_stokes_material& m, double eta[27]) {
    for (int q = 0; q < el.NQ; ++q) eta[q] = el.eta_ip ? el.etaq_ip[q] : interp_phase(t.N[q], m.eta, el.phv, el.NV);
}

// (∂R/∂u)ᵀλ over the mesh: dv = (dRv/dv)ᵀλv + (dRP/dv)ᵀλP, dP = (dRv/dP)ᵀλv +
// (dRP/dP)ᵀλP, from the element Jacobians by forward-mode duals (27 partials per
// velocity component, 4 for the pressure DoFs).
void adjoint_residual_impl(const femb200_stokes_problem* p, double dt, int finite_K, bool with_pnum,
                           const double* const lam_v[3], const double* lam_P, double* const out_dv[3], double* out_dP) {
    const Tables& t = tables_for(3);
    const double* bulk = bulk_table(p, finite_K);
    std::vector<double> buf((size_t)p->nels * 85);
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t e = 0; e < p->nels; ++e) {
        Elem el; gather(p, e, el);
        double vd[3][27]; load_v(p, el, vd);
        double eta[27]; element_viscosity(t, el, p->mat, eta);
        double lv[3][27], lp[4];
        for (int c = 0; c < 3; ++c) for (int a = 0; a < 27; ++a) lv[c][a] = lam_v[c][el.nodes[a] - 1];
        for (int i = 0; i < 4; ++i) lp[i] = lam_P[el.dofs[i] - 1];
        double* o = &buf[(size_t)e * 85];
        {
            using DU = Dual<27>;
            for (int j = 0; j < 3; ++j) {
                DU v[3][27], Pe[4], et[27], Rv[3][27], RP[4];
                for (int c = 0; c < 3; ++c) for (int a = 0; a < 27; ++a) v[c][a] = DU(vd[c][a]);
                for (int b = 0; b < 27; ++b) v[j][b].d[b] = 1.0;
                for (int i = 0; i < 4; ++i) Pe[i] = DU(el.P[i]);
                for (int q = 0; q < 27; ++q) et[q] = DU(eta[q]);
                stokes_element_all<DU>(t, el, p->mat, v, Pe, et, bulk, dt, with_pnum, Rv, RP);
                for (int b = 0; b < 27; ++b) {
                    double s = 0;
                    for (int c = 0; c < 3; ++c) for (int a = 0; a < 27; ++a) s += lv[c][a] * Rv[c][a].d[b];
                    for (int i = 0; i < 4; ++i) s += lp[i] * RP[i].d[b];
                    o[j * 27 + b] = s;
                }
            }
        }
        {
            using DU = Dual<4>;
            DU v[3][27], Pe[4], et[27], Rv[3][27], RP[4];
            for (int c = 0; c < 3; ++c) for (int a = 0; a < 27; ++a) v[c][a] = DU(vd[c][a]);
            for (int i = 0; i < 4; ++i) { Pe[i] = DU(el.P[i]); Pe[i].d[i] = 1.0; }
            for (int q = 0; q < 27; ++q) et[q] = DU(eta[q]);
            stokes_element_all<DU>(t, el, p->mat, v, Pe, et, bulk, dt, with_pnum, Rv, RP);
            for (int k = 0; k < 4; ++k) {
                double s = 0;
                for (int c = 0; c < 3; ++c) for (int a = 0; a < 27; ++a) s += lv[c][a] * Rv[c][a].d[k];
                for (int i = 0; i < 4; ++i) s += lp[i] * RP[i].d[k];
                o[81 + k] = s;
            }
        }
    }
    for (int c = 0; c < 3; ++c) std::fill(out_dv[c], out_dv[c] + p->nnodes, 0.0);
    std::fill(out_dP, out_dP + p->nnodesP, 0.0);
    for (int64_t e = 0; e < p->nels; ++e) {
        const double* o = &buf[(size_t)e * 85];
        for (int c = 0; c < 3; ++c)
            for (int a = 0; a < 27; ++a) out_dv[c][p->el2n[27 * e + a] - 1] += o[c * 27 + a];
        for (int i = 0; i < 4; ++i) out_dP[p->dofsP[4 * e + i] - 1] += o[81 + i];
    }
}

// λ·∂R/∂η_q for the viscosity at every quadrature point (the per-point field
// p->viscosity_ip, or the phase-interpolated viscosity), nq × nels.
void viscosity_sensitivity_impl(const femb200_stokes_problem* p, double dt, int finite_K, bool with_pnum,
                                const double* const lam_v[3], const double* lam_P, double* out) {
    const Tables& t = tables_for(3);
    const double* bulk = bulk_table(p, finite_K);
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t e = 0; e < p->nels; ++e) {
        Elem el; gather(p, e, el);
        double vd[3][27]; load_v(p, el, vd);
        double eta[27]; element_viscosity(t, el, p->mat, eta);
        using DU = Dual<27>;
        DU v[3][27], Pe[4], et[27], Rv[3][27], RP[4];
        for (int c = 0; c < 3; ++c) for (int a = 0; a < 27; ++a) v[c][a] = DU(vd[c][a]);
        for (int i = 0; i < 4; ++i) Pe[i] = DU(el.P[i]);
        for (int q = 0; q < 27; ++q) { et[q] = DU(eta[q]); et[q].d[q] = 1.0; }
        stokes_element_all<DU>(t, el, p->mat, v, Pe, et, bulk, dt, with_pnum, Rv, RP);
        for (int q = 0; q < 27; ++q) {
            double s = 0;
            for (int c = 0; c < 3; ++c) for (int a = 0; a < 27; ++a) s += lam_v[c][el.nodes[a] - 1] * Rv[c][a].d[q];
            for (int i = 0; i < 4; ++i) s += lam_P[el.dofs[i] - 1] * RP[i].d[q];
            out[27 * e + q] = s;
        }
    }
}

// Pressure mass and scale (pressure_scaling.jl:118-216).
void pressure_scaling_impl(const femb200_stokes_problem* p, double gfact, double dt, int finite_K) {
    const Tables& t = tables_for(p->dim);
    const int NV = t.nv, NP = t.np, NQ = t.nq;
    double* MP = Dm(p->M_P); double* gP = Dm(p->gammaP);
    std::fill(MP, MP + p->nnodesP, 0.0);
    std::fill(gP, gP + p->nnodesP, 0.0);
    const double* Ktab = finite_K ? p->mat.K : p->mat.eta_b;
    double beta[FEMB200_MAX_PHASES];
    for (int i = 0; i < FEMB200_MAX_PHASES; ++i) beta[i] = 1.0 / Ktab[i];
    const double* eta_tab = p->mat.use_scaling_eta ? p->mat.scaling_eta : p->mat.eta;
    for (int64_t e = 0; e < p->nels; ++e) {
        Elem el; gather(p, e, el, false);
        for (int q = 0; q < NQ; ++q) {
            double dO = el.geoP[q];
            const double* Nv = t.N[q];
            const double* NPq = t.NP[q];
            double etaq = (el.eta_ip && !p->mat.use_scaling_eta) ? el.etaq_ip[q] : interp_phase(Nv, eta_tab, el.phv, NV);
            // pressure_scale_at_ip (pressure_scaling.jl:206-211)
            double gnum = gfact * etaq;
            double bq = interp_phase(Nv, beta, el.phv, NV);
            double gphy = bq == 0 ? gnum : dt / bq;
            double gq = gphy * gnum / (gphy + gnum);
            for (int a = 0; a < NP; ++a) {
                int64_t d = el.dofs[a] - 1;
                double w = NPq[a] * NPq[a] * dO;
                MP[d] += w;
                gP[d] += w * gq;
            }
        }
    }
    for (int64_t i = 0; i < p->nnodesP; ++i) gP[i] = MP[i] == 0 ? 0.0 : gP[i] / MP[i];
}

void dirichlet(double* x, const int32_t* dofs, const double* vals, int64_t n) {
    for (int64_t i = 0; i < n; ++i) x[dofs[i] - 1] = vals ? vals[i] : 0.0;
}

double norm2(const double* x, int64_t n) {
    double s = 0;
    for (int64_t i = 0; i < n; ++i) s += x[i] * x[i];
    return std::sqrt(s);
}

// _checked_λmax (src/utils.jl:152-158)
int checked_lmax(const double* J, const double* PC, int64_t n, const char* label, double& out) {
    double m = -INFINITY;
    for (int64_t i = 0; i < n; ++i) { double r = J[i] / PC[i]; if (std::isnan(r)) { m = NAN; break; } m = std::max(m, r); }
    if (!(std::isfinite(m) && m > 0)) {
        char b[256];
        std::snprintf(b, sizeof b, "%s preconditioner produced invalid λmax = %g; check for zero or non-finite preconditioner entries", label, m);
        g_last_error = b;
        return FEMB200_ELAMBDA;
    }
    out = m;
    return FEMB200_OK;
}

// ---- thermal ----------------------------------------------------------------

struct TElem {
    int NV, NQ, D;
    int64_t nodes[27];
    double T0[27], s[27], P[27], Phi[27];
    int ph[27];
    const double* geo;
    bool hasPhi;
};

// integrate_residual (src/heat_diffusion/assembly/residual.jl:58-87)
template <class S>
void thermal_element(const Tables& t, const TElem& el, const femb200_thermal_problem* tp, const S* T, double dt,
                     double Tref, S* Re) {
    const int NV = el.NV, DD = el.D;
    for (int a = 0; a < NV; ++a) Re[a] = S(0.0);
    double beta[FEMB200_MAX_PHASES];
    for (int i = 0; i < FEMB200_MAX_PHASES; ++i) beta[i] = 1.0 / tp->K[i];
    double dNdx[27][3];
    for (int q = 0; q < el.NQ; ++q) {
        dNdx_at(t, el.geo, DD, q, dNdx);
        double dO = el.geo[q * (DD * DD + 1) + DD * DD];
        const double* Nv = t.N[q];
        S Tq(0.0); for (int a = 0; a < NV; ++a) Tq = Tq + Nv[a] * T[a];
        double Pq = 0; for (int a = 0; a < NV; ++a) Pq += Nv[a] * el.P[a];
        double kq = interp_phase(Nv, tp->k, el.ph, NV);
        double aq = interp_phase(Nv, tp->alpha, el.ph, NV);
        double bq = interp_phase(Nv, beta, el.ph, NV);
        S rhoq = interp_phase(Nv, tp->rho0, el.ph, NV) * (1.0 - aq * (Tq - Tref) + bq * Pq);
        S dtrc = dt / (rhoq * interp_phase(Nv, tp->Cp, el.ph, NV));
        S gT[3];
        for (int k = 0; k < DD; ++k) { S s(0.0); for (int b = 0; b < NV; ++b) s = s + dNdx[b][k] * T[b]; gT[k] = s; }
        double T0q = 0, sq = 0;
        for (int a = 0; a < NV; ++a) { T0q += Nv[a] * el.T0[a]; sq += Nv[a] * el.s[a]; }
        S Hq = el.hasPhi ? dtrc * el.Phi[q] : S(0.0);
        S rate = T0q - Tq + dtrc * sq + Hq;
        for (int i = 0; i < NV; ++i) {
            S KT(0.0);
            for (int k = 0; k < DD; ++k) KT = KT + dNdx[i][k] * gT[k];
            KT = kq * KT;
            Re[i] = Re[i] + (rate * Nv[i] * dO - dtrc * KT * dO);
        }
    }
}

void tgather(const femb200_thermal_problem* tp, int64_t e, TElem& el) {
    const Tables& t = tables_for(tp->dim);
    el.NV = t.nv; el.NQ = t.nq; el.D = tp->dim;
    for (int a = 0; a < el.NV; ++a) {
        el.nodes[a] = tp->el2n[(int64_t)el.NV * e + a];
        int64_t n = el.nodes[a] - 1;
        el.T0[a] = D(tp->T0)[n];
        el.s[a] = tp->source ? D(tp->source)[n] : 0.0;
        el.P[a] = tp->P ? D(tp->P)[n] : 0.0;
        el.ph[a] = phase_at(tp->phases, tp->phases_layout, el.nodes[a], a, e, el.NV);
    }
    el.hasPhi = tp->source_ip != nullptr;
    if (el.hasPhi) for (int q = 0; q < el.NQ; ++q) el.Phi[q] = D(tp->source_ip)[(int64_t)el.NQ * e + q];
    el.geo = D(tp->geo) + (int64_t)e * el.NQ * (el.D * el.D + 1);
}

template <int NVT>
void thermal_assemble_t(const femb200_thermal_problem* tp, double dt, double Tref, bool jac) {
    const Tables& t = tables_for(tp->dim);
    const int NV = t.nv;
    std::vector<double> buf((size_t)tp->nels * NV * 3);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < tp->nels; ++e) {
        TElem el; tgather(tp, e, el);
        double T[27]; for (int a = 0; a < NV; ++a) T[a] = D(tp->T)[el.nodes[a] - 1];
        double Re[27];
        thermal_element<double>(t, el, tp, T, dt, Tref, Re);
        double* o = &buf[(size_t)e * NV * 3];
        for (int a = 0; a < NV; ++a) o[3 * a] = Re[a];
        if (jac) {
            Dual<NVT> Td[27];
            for (int a = 0; a < NV; ++a) { Td[a] = Dual<NVT>(T[a]); Td[a].d[a] = 1.0; }
            Dual<NVT> Rd[27];
            thermal_element<Dual<NVT>>(t, el, tp, Td, dt, Tref, Rd);
            for (int a = 0; a < NV; ++a) {
                double s = 0; for (int b = 0; b < NV; ++b) s += std::fabs(Rd[a].d[b]);
                o[3 * a + 1] = s; o[3 * a + 2] = std::fabs(Rd[a].d[a]);
            }
        }
    }
    std::fill(Dm(tp->R), Dm(tp->R) + tp->nnodes, 0.0);
    if (jac) {
        std::fill(Dm(tp->dRdT), Dm(tp->dRdT) + tp->nnodes, 0.0);
        std::fill(Dm(tp->PC), Dm(tp->PC) + tp->nnodes, 0.0);
    }
    for (int64_t e = 0; e < tp->nels; ++e) {
        const double* o = &buf[(size_t)e * NV * 3];
        for (int a = 0; a < NV; ++a) {
            int64_t n = tp->el2n[(int64_t)NV * e + a] - 1;
            Dm(tp->R)[n] += o[3 * a];
            if (jac) { Dm(tp->dRdT)[n] += o[3 * a + 1]; Dm(tp->PC)[n] += o[3 * a + 2]; }
        }
    }
}

void thermal_assemble(const femb200_thermal_problem* tp, double dt, double Tref, bool jac) {
    if (tp->dim == 3) thermal_assemble_t<27>(tp, dt, Tref, jac);
    else thermal_assemble_t<9>(tp, dt, Tref, jac);
}

// shear_dissipation (shear_heating.jl:79-103): stress power less elastic power at one
// point; g[i][k] = ∂v_i/∂x_k, stresses in assembler order (xx, yy, xy) or
// (xx, yy, zz, xy, xz, yz); plane strain carries τzz = −(τxx + τyy) in the elastic term.
double shear_dissipation(int dim, const double* tau, const double* o, const double g[3][3], double inv2Gdt) {
    if (dim == 3) {
        const double power = tau[0] * g[0][0] + tau[1] * g[1][1] + tau[2] * g[2][2] + tau[3] * (g[0][1] + g[1][0]) +
                             tau[4] * (g[0][2] + g[2][0]) + tau[5] * (g[1][2] + g[2][1]);
        const double elastic = (tau[0] * (tau[0] - o[0]) + tau[1] * (tau[1] - o[1]) + tau[2] * (tau[2] - o[2]) +
                                2 * (tau[3] * (tau[3] - o[3]) + tau[4] * (tau[4] - o[4]) + tau[5] * (tau[5] - o[5]))) *
                               inv2Gdt;
        return power - elastic;
    }
    const double tzz = -(tau[0] + tau[1]), tzzo = -(o[0] + o[1]);
    const double power = tau[0] * g[0][0] + tau[1] * g[1][1] + tau[2] * (g[0][1] + g[1][0]);
    const double elastic = (tau[0] * (tau[0] - o[0]) + tau[1] * (tau[1] - o[1]) + tzz * (tzz - tzzo) +
                            2 * tau[2] * (tau[2] - o[2])) * inv2Gdt;
    return power - elastic;
}

// shear_heating_element (shear_heating.jl:47-73).
void shear_heating_impl(const femb200_stokes_problem* p, double dt, double* phi) {
    const Tables& t = tables_for(p->dim);
    const int DD = p->dim;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < p->nels; ++e) {
        Elem el; gather(p, e, el, false);
        double v[3][27]; load_v(p, el, v);
        double dNdx[27][3];
        for (int q = 0; q < el.NQ; ++q) {
            dNdx_at(t, el.geo, DD, q, dNdx);
            const double* Nv = t.N[q];
            double Pq = 0; for (int i = 0; i < el.NP; ++i) Pq += t.NP[q][i] * el.P[i];
            double Pfq = 0; if (el.hasPf) for (int i = 0; i < el.NP; ++i) Pfq += t.NP[q][i] * el.Pf[i];
            double Peq = el.hasPf ? Pq - Pfq : Pq;
            double etaq = el.eta_ip ? el.etaq_ip[q] : interp_phase(Nv, p->mat.eta, el.phv, el.NV);
            double etave, inv2Gdt;
            ve_coeffs(Nv, etaq, p->mat.G, el.phv, el.NV, dt, etave, inv2Gdt);
            Plastic pl; const Plastic* plp = nullptr;
            if (p->mat.plastic) { pl = plastic_at(p->mat, Nv, el.phv, el.NV, dt); plp = &pl; }
            double g[3][3];
            for (int i = 0; i < DD; ++i)
                for (int k = 0; k < DD; ++k) { double s = 0; for (int a = 0; a < el.NV; ++a) s += dNdx[a][k] * v[i][a]; g[i][k] = s; }
            double tau[6];
            if (DD == 3) {
                stress3d<double>(g, etave, inv2Gdt, el.told[q], plp, Peq, tau, nullptr);
            } else {
                double g2[2][2] = {{g[0][0], g[0][1]}, {g[1][0], g[1][1]}};
                stress2d<double>(g2, etave, inv2Gdt, el.told[q], plp, Peq, tau, nullptr);
            }
            phi[(int64_t)el.NQ * e + q] = shear_dissipation(DD, tau, el.told[q], g, inv2Gdt);
        }
    }
}

void transfer_T(double* TP, const double* T, const int32_t* dofsP, const int32_t* el2nP, int64_t n) {
    for (int64_t i = 0; i < n; ++i) TP[dofsP[i] - 1] = T[el2nP[i] - 1];
}

// _stokes_λmin (DR.jl:32-37)
double stokes_lmin(double step, const double* rate, const double* R, const double* R0, const double* PC, int64_t n) {
    double den = 0; for (int64_t i = 0; i < n; ++i) { double r = step * rate[i]; den += r * r; }
    if (den == 0) return 0;
    double num = 0; for (int64_t i = 0; i < n; ++i) num += (step * rate[i]) * ((R[i] - R0[i]) / PC[i]);
    return std::fabs(num) / den;
}

void stokes_cheb(double dtau, double lmin, double c_fact, double& a, double& b) {
    double c = 2 * std::sqrt(lmin) * c_fact;
    a = 2 * dtau * dtau / (2 + c * dtau);
    b = (2 - c * dtau) / (2 + c * dtau);
}

// The coupled thermal state carried through the Stokes loop (DR.jl:133, :604-663).
struct Coupled {
    femb200_thermal_problem* t;
    double Tref;
    double* phi;   // nq × nels or null
};

// The Stokes part of one inner DR iteration (DR.jl:664-698): pressure residual,
// Pnum = γP·RP/M_P, momentum residual with Pnum, the Dirichlet pins of Rv and of the
// rate, the negated Chebyshev velocity update (helpers.jl:31-41) and the pins of v.
void stokes_inner_step(const femb200_stokes_problem* p, double dt, int finite_K, const double alpha[3],
                       const double beta[3]) {
    const int DD = p->dim;
    const int64_t nn = p->nnodes, nP = p->nnodesP;
    pressure_residual_impl(p, dt, finite_K);
    for (int64_t i = 0; i < nP; ++i) Dm(p->Pnum)[i] = D(p->gammaP)[i] * D(p->RP)[i] / D(p->M_P)[i];
    momentum_residual_impl(p, dt, true);
    for (int k = 0; k < DD; ++k) {
        if (p->body_force[k]) for (int64_t i = 0; i < nn; ++i) Dm(p->Rv[k])[i] -= D(p->body_force[k])[i];
        dirichlet(Dm(p->Rv[k]), p->bc_dofs[k], nullptr, p->bc_n[k]);
    }
    for (int k = 0; k < DD; ++k) dirichlet(Dm(p->rate[k]), p->bc_dofs[k], nullptr, p->bc_n[k]);
    for (int k = 0; k < DD; ++k) {
        double* r = Dm(p->rate[k]); double* v = Dm(p->v[k]);
        const double* R = D(p->Rv[k]); const double* PC = D(p->PC[k]);
        double na = -alpha[k];
        for (int64_t i = 0; i < nn; ++i) { double nr = beta[k] * r[i] + R[i] / PC[i]; r[i] = nr; v[i] += na * nr; }
    }
    for (int k = 0; k < DD; ++k) dirichlet(Dm(p->v[k]), p->bc_dofs[k], D(p->bc_vals[k]), p->bc_n[k]);
}

// The velocity error and the per-component λmin of a check (DR.jl:700-726).
double stokes_check_norms(const femb200_stokes_problem* p, const double alpha[3], double lmin[3]) {
    const int DD = p->dim;
    const int64_t nn = p->nnodes;
    double ev = 0; for (int k = 0; k < DD; ++k) ev = jl_max(ev, norm2(D(p->Rv[k]), nn));
    ev /= 2 * std::sqrt((double)nn);
    for (int k = 0; k < DD; ++k) lmin[k] = stokes_lmin(alpha[k], D(p->rate[k]), D(p->Rv[k]), D(p->Rv0[k]), D(p->PC[k]), nn);
    return ev;
}

// _solve_stokes_dyrel! (src/stokes/solvers/DR.jl:348-802).
int solve_dyrel(const femb200_stokes_problem* p, const femb200_stokes_controls* c, femb200_stokes_stats* st,
                Coupled* cp) {
    const int DD = p->dim;
    const int64_t nn = p->nnodes, nP = p->nnodesP;
    const double dt = c->dt;
    const int finite_K = c->finite_K;
    const bool freeze = c->freeze_jacobian < 0 ? (p->mat.plastic == 0) : (c->freeze_jacobian != 0);
    const int64_t nout = c->check_interval;
    const double cfl = c->cfl_v > 0 ? c->cfl_v : 0.98, cf = c->c_fact > 0 ? c->c_fact : 0.9;
    static const char* labels[3] = {"stokes vx", "stokes vy", "stokes vz"};
    std::memset(st, 0, sizeof(*st));

    for (int k = 0; k < DD; ++k) {
        std::fill(Dm(p->rate[k]), Dm(p->rate[k]) + nn, 0.0);
        std::fill(Dm(p->Rv0[k]), Dm(p->Rv0[k]) + nn, 0.0);
    }
    femb200_stokes_problem pj = *p;   // the diagnostics read dr.P0 regardless of P_old
    jacobian_impl(&pj, dt, finite_K);
    double lmax[3] = {0, 0, 0};
    for (int k = 0; k < DD; ++k) {
        int rc = checked_lmax(D(p->dRdv[k]), D(p->PC[k]), nn, labels[k], lmax[k]);
        if (rc) return rc;
    }
    double lmax_g = *std::max_element(lmax, lmax + DD);
    int64_t jac_assemblies = 1;
    double alpha[3], beta[3], dtau[3];
    for (int k = 0; k < DD; ++k) { dtau[k] = 2 / std::sqrt(lmax[k]) * cfl; stokes_cheb(dtau[k], 0.0, cf, alpha[k], beta[k]); }

    double err_min = INFINITY, eps = c->tolerance;
    double err = 2 * eps, err_abs = INFINITY, err_rel = INFINITY;
    double err_v0 = 1.0, err_P0 = 1.0, err_v00 = 1.0, err_v = INFINITY, err_P = INFINITY;
    int64_t iter = 0, itPH_done = 0;
    bool converged = false;
    double rel_drop = c->rel_drop0;
    int64_t hist = 0;
    auto push_hist = [&](double it, double ev, double eP) {
        if (!c->history || hist >= c->history_capacity) { ++hist; return; }
        double* h = c->history + hist * (4 + DD);
        h[0] = it; h[1] = ev; h[2] = eP; h[3] = 0;
        for (int k = 0; k < DD; ++k) h[4 + k] = norm2(D(p->Rv[k]), nn) / (2 * std::sqrt((double)nn));
        ++hist;
    };

    // coupled thermal state
    int64_t thermal_iter = 0;
    double err_T = cp ? INFINITY : 0;
    bool thermal_converged = cp == nullptr;
    double aT = 0, bT = 0, lmaxT = 0, nr0T = 0;
    auto shear_heat = [&]() { if (cp && cp->phi) shear_heating_impl(p, dt, cp->phi); };
    if (cp) {
        std::fill(Dm(cp->t->rate), Dm(cp->t->rate) + cp->t->nnodes, 0.0);
        std::fill(Dm(cp->t->R0), Dm(cp->t->R0) + cp->t->nnodes, 0.0);
        shear_heat();
    }

    std::vector<double> Pnum_tmp;
    for (int64_t itPH = 1; itPH <= c->max_ph_iterations; ++itPH) {
        itPH_done = itPH;
        pressure_residual_impl(p, dt, finite_K);
        momentum_residual_impl(p, dt, false);
        for (int k = 0; k < DD; ++k) {
            if (p->body_force[k]) for (int64_t i = 0; i < nn; ++i) Dm(p->Rv[k])[i] -= D(p->body_force[k])[i];
            dirichlet(Dm(p->Rv[k]), p->bc_dofs[k], nullptr, p->bc_n[k]);
        }
        {
            double s = 0; for (int64_t i = 0; i < nP; ++i) { double r = D(p->RP)[i] / D(p->M_P)[i]; s += r * r; }
            err_P = std::sqrt(s) / std::sqrt((double)nP);
        }
        err_v = 0; for (int k = 0; k < DD; ++k) err_v = jl_max(err_v, norm2(D(p->Rv[k]), nn));
        err_v /= 2 * std::sqrt((double)nn);
        push_hist((double)iter, err_v, err_P);
        if (itPH == 1) { err_P0 = err_P + julia_eps(err_P); err_v0 = err_v + julia_eps(err_v); }
        else if (itPH == 2) { err_P0 = err_P + julia_eps(err_P); }
        double err_v_rel = err_v / err_v0, err_P_rel = err_P / err_P0;
        err_abs = jl_max(err_v, err_P);
        err_rel = jl_max(err_v_rel, err_P_rel);
        err = jl_min(err_abs, err_rel);
        if (std::isnan(err)) { char b[128]; std::snprintf(b, sizeof b, "NaN detected in outer loop at PH=%lld", (long long)itPH); g_last_error = b; return FEMB200_ENAN; }
        if (err > 1e10) { char b[128]; std::snprintf(b, sizeof b, "Kaboom! Error > 1e10 in outer loop at PH=%lld", (long long)itPH); g_last_error = b; return FEMB200_EKABOOM; }
        if (err < eps && thermal_converged) { converged = true; break; }
        if (err > err_min * 1.05) rel_drop = std::max(rel_drop * 0.1, 1.0e-3);
        err_min = std::min(err_min, err);
        double eps_vel = err * rel_drop;
        int64_t itPT = 0;
        while ((err > eps_vel || !thermal_converged) && itPT <= c->iter_max) {
            ++itPT; ++iter;
            bool do_check = iter % nout == 0;
            if (do_check) for (int k = 0; k < DD; ++k) std::copy(D(p->Rv[k]), D(p->Rv[k]) + nn, Dm(p->Rv0[k]));
            if (cp) {
                femb200_thermal_problem* tp = cp->t;
                ++thermal_iter;
                bool tcheck = thermal_iter == 1 || thermal_iter % nout == 0;
                if (tcheck) std::copy(D(tp->R), D(tp->R) + tp->nnodes, Dm(tp->R0));
                femb200_thermal_problem tt = *tp; tt.source_ip = cp->phi;
                thermal_assemble(&tt, dt, cp->Tref, tcheck);
                dirichlet(Dm(tp->R), tp->bc_dofs, nullptr, tp->bc_n);
                dirichlet(Dm(tp->rate), tp->bc_dofs, nullptr, tp->bc_n);
                if (tcheck) { int rc = checked_lmax(D(tp->dRdT), D(tp->PC), tp->nnodes, "thermal diffusion", lmaxT); if (rc) return rc; }
                for (int64_t i = 0; i < tp->nnodes; ++i) Dm(tp->rate)[i] = D(tp->R)[i] / D(tp->PC)[i] + bT * D(tp->rate)[i];
                for (int64_t i = 0; i < tp->nnodes; ++i) Dm(tp->T)[i] += aT * D(tp->rate)[i];
                dirichlet(Dm(tp->T), tp->bc_dofs, D(tp->bc_vals), tp->bc_n);
                transfer_T(Dm(p->T), D(tp->T), p->dofsP, p->el2nP, (int64_t)p->np * p->nels);
                if (tcheck) {
                    double nrT = norm2(D(tp->R), tp->nnodes);
                    if (thermal_iter == 1) nr0T = std::max(nrT, julia_eps(nrT));
                    err_T = nrT / nr0T;
                    if (!std::isfinite(err_T)) { char b[128]; std::snprintf(b, sizeof b, "non-finite thermal residual at coupled iteration %lld", (long long)thermal_iter); g_last_error = b; return FEMB200_ENONFINITE; }
                    double dtT = 2 / std::sqrt(lmaxT) * tp->cfl;
                    double den = 0; for (int64_t i = 0; i < tp->nnodes; ++i) { double r = dtT * D(tp->rate)[i]; den += r * r; }
                    double lminT = 0;
                    if (!(thermal_iter == 1 || den == 0)) {
                        double num = 0;
                        for (int64_t i = 0; i < tp->nnodes; ++i) num += (dtT * D(tp->rate)[i]) * ((D(tp->R)[i] - D(tp->R0)[i]) / D(tp->PC)[i]);
                        lminT = std::fabs(num) / den;
                    }
                    stokes_cheb(dtT, lminT, tp->c_fact, aT, bT);
                    thermal_converged = err_T < tp->eps;
                    shear_heat();
                }
            }
            // update_stokes_velocity! with the negated Chebyshev step (DR.jl:692-695, helpers.jl:31-41)
            stokes_inner_step(p, dt, finite_K, alpha, beta);
            if (do_check) {
                double lmin[3];
                const double ev = stokes_check_norms(p, alpha, lmin);
                if (iter == nout) err_v00 = ev + julia_eps(ev);
                err = ev <= eps ? ev : jl_max(ev / err_v00, ev);
                if (std::isnan(err)) { char b[128]; std::snprintf(b, sizeof b, "NaN detected in inner loop PH=%lld PT=%lld", (long long)itPH, (long long)itPT); g_last_error = b; return FEMB200_ENAN; }
                if (err > 1e10) { char b[128]; std::snprintf(b, sizeof b, "Kaboom! Error > 1e10 in inner loop PH=%lld PT=%lld", (long long)itPH, (long long)itPT); g_last_error = b; return FEMB200_EKABOOM; }
                {
                    double s = 0; for (int64_t i = 0; i < nP; ++i) { double r = D(p->RP)[i] / D(p->M_P)[i]; s += r * r; }
                    push_hist((double)iter, ev, std::sqrt(s) / std::sqrt((double)nP));
                }
                if (!freeze) {
                    ++jac_assemblies;
                    jacobian_impl(&pj, dt, finite_K);
                    for (int k = 0; k < DD; ++k) {
                        int rc = checked_lmax(D(p->dRdv[k]), D(p->PC[k]), nn, labels[k], lmax[k]);
                        if (rc) return rc;
                    }
                    lmax_g = *std::max_element(lmax, lmax + DD);
                }
                for (int k = 0; k < DD; ++k) { dtau[k] = 2 / std::sqrt(lmax[k]) * cfl; stokes_cheb(dtau[k], lmin[k], cf, alpha[k], beta[k]); }
            }
            if (iter > c->max_iterations) break;
        }
        for (int64_t i = 0; i < nP; ++i) Dm(p->P)[i] += D(p->gammaP)[i] * D(p->RP)[i] / D(p->M_P)[i];
        if (iter > c->max_iterations) break;
    }
    st->itPH = itPH_done; st->iter = iter; st->err = err; st->err_abs = err_abs; st->err_rel = err_rel;
    st->err_v = err_v; st->err_P = err_P; st->converged = converged; st->reached_total_iter = iter > c->max_iterations;
    st->lambda_max = *std::max_element(lmax, lmax + DD); st->lambda_max_gershgorin = lmax_g;
    st->jacobian_assemblies = jac_assemblies; st->history_len = std::min<int64_t>(hist, c->history_capacity);
    st->err_T = err_T; st->thermal_iterations = thermal_iter;
    return FEMB200_OK;
}

int solve_stokes_impl(const femb200_stokes_problem* p, const femb200_stokes_controls* c, femb200_stokes_stats* st, Coupled* cp) {
    int rc = check_problem(p);
    if (rc) return rc;
    if (c->assemble_scaling) pressure_scaling_impl(p, c->pressure_factor, c->dt, c->finite_K);
    rc = solve_dyrel(p, c, st, cp);
    if (rc) return rc;
    if (!st->converged && c->throw_on_failure) {
        char b[256];
        std::snprintf(b, sizeof b, "Stokes solve did not converge after %lld iterations (residual = %g, tolerance = %g)",
                      (long long)st->iter, st->err_abs, c->tolerance);
        g_last_error = b;
        return FEMB200_ENOTCONV;
    }
    return FEMB200_OK;
}

// ---- LithostaticPressureDR ----------------------------------------------------
// lp_integrate_residual (src/lithostatic_pressure/assembly/residual.jl:48-63) on one
// element given its shape functions N[q][a], physical gradients dNdx[q][a][k] and
// weights dO[q]: R_i = Σ_q (ρ_q ∇N_i·g − ∇N_i·∇P) dΩ, ρ_q = ρ0_q (1 − α_q (T_q − Tref) + β_q P_q).
template <class S>
void lp_element(int NV, int D, int NQ, const double* N, const double* dNdx, const double* dO, const S* P,
                const double* T, const int* ph, const double* rho0, const double* alpha, const double* beta,
                double Tref, const double* g, S* Re) {
    for (int a = 0; a < NV; ++a) Re[a] = S(0.0);
    for (int q = 0; q < NQ; ++q) {
        const double* Nq = N + q * NV;
        const double* G = dNdx + (size_t)q * NV * D;
        double Tq = 0;
        for (int a = 0; a < NV; ++a) Tq += Nq[a] * T[a];
        S Pq(0.0);
        for (int a = 0; a < NV; ++a) Pq = Pq + Nq[a] * P[a];
        const double aq = interp_phase(Nq, alpha, ph, NV), bq = interp_phase(Nq, beta, ph, NV);
        const S rho = interp_phase(Nq, rho0, ph, NV) * (1.0 - aq * (Tq - Tref) + bq * Pq);
        S gP[3] = {S(0.0), S(0.0), S(0.0)};
        for (int k = 0; k < D; ++k)
            for (int b = 0; b < NV; ++b) gP[k] = gP[k] + G[b * D + k] * P[b];
        for (int i = 0; i < NV; ++i) {
            double ng = 0;
            S np(0.0);
            for (int k = 0; k < D; ++k) { ng += G[i * D + k] * g[k]; np = np + G[i * D + k] * gP[k]; }
            Re[i] = Re[i] + (rho * ng - np) * dO[q];
        }
    }
}

// Residual of one element and, with jac, the absolute row sums and diagonal of its
// ForwardDiff Jacobian in P (lp_element_jacobian, residual.jl:22-36).
template <int NVT>
void lp_element_all(int NV, int D, int NQ, const double* N, const double* dNdx, const double* dO, const double* P,
                    const double* T, const int* ph, const double* rho0, const double* alpha, const double* beta,
                    double Tref, const double* g, bool jac, double* R, double* rows, double* diag) {
    lp_element<double>(NV, D, NQ, N, dNdx, dO, P, T, ph, rho0, alpha, beta, Tref, g, R);
    if (!jac) return;
    Dual<NVT> Pd[27], Rd[27];
    for (int a = 0; a < NV; ++a) { Pd[a] = Dual<NVT>(P[a]); Pd[a].d[a] = 1.0; }
    lp_element<Dual<NVT>>(NV, D, NQ, N, dNdx, dO, Pd, T, ph, rho0, alpha, beta, Tref, g, Rd);
    for (int a = 0; a < NV; ++a) {
        double sum = 0;
        for (int b = 0; b < NV; ++b) sum += std::fabs(Rd[a].d[b]);
        rows[a] = sum;
        diag[a] = std::fabs(Rd[a].d[a]);
    }
}

void lp_assemble(const femb200_lithostatic_problem* p, double Tref, const double* g, bool jac) {
    const Tables& t = tables_for(p->dim);
    const int NV = t.nv, NQ = t.nq, D = p->dim;
    double beta[FEMB200_MAX_PHASES];
    for (int i = 0; i < FEMB200_MAX_PHASES; ++i) beta[i] = 1.0 / p->K[i];
    std::fill(p->R, p->R + p->nnodes, 0.0);
    if (jac) { std::fill(p->dRdP, p->dRdP + p->nnodes, 0.0); std::fill(p->PC, p->PC + p->nnodes, 0.0); }
    for (int64_t e = 0; e < p->nels; ++e) {
        double N[27 * 27], G[27 * 27 * 3], dO[27], P[27], T[27], R[27], rows[27], diag[27];
        int ph[27];
        const double* geo = p->geo + (size_t)e * NQ * (D * D + 1);
        for (int q = 0; q < NQ; ++q) {
            double d[27][3];
            dNdx_at(t, geo, D, q, d);
            for (int a = 0; a < NV; ++a) {
                N[q * NV + a] = t.N[q][a];
                for (int k = 0; k < D; ++k) G[((size_t)q * NV + a) * D + k] = d[a][k];
            }
            dO[q] = geo[q * (D * D + 1) + D * D];
        }
        for (int a = 0; a < NV; ++a) {
            const int64_t node = p->el2n[(int64_t)NV * e + a];
            P[a] = p->P[node - 1];
            T[a] = p->T ? p->T[node - 1] : 0.0;
            ph[a] = phase_at(p->phases, p->phases_layout, node, a, e, NV);
        }
        if (NV == 27) lp_element_all<27>(NV, D, NQ, N, G, dO, P, T, ph, p->rho0, p->alpha, beta, Tref, g, jac, R, rows, diag);
        else lp_element_all<9>(NV, D, NQ, N, G, dO, P, T, ph, p->rho0, p->alpha, beta, Tref, g, jac, R, rows, diag);
        for (int a = 0; a < NV; ++a) {
            const int64_t n = p->el2n[(int64_t)NV * e + a] - 1;
            p->R[n] += R[a];
            if (jac) { p->dRdP[n] += rows[a]; p->PC[n] += diag[a]; }
        }
    }
}

// solve_dynamic_relaxation! (src/dynamic_relaxation/solver.jl:61-122) for P.
int lp_solve_impl(const femb200_lithostatic_problem* p, const femb200_lithostatic_controls* c, femb200_thermal_stats* st) {
    const int64_t n = p->nnodes;
    double aT = 0, bT = 0, nr0 = 0, last_rel = NAN, lmax = 0;
    for (int64_t it = 1; it <= c->max_iterations; ++it) {
        bool dj = (it % c->check_interval == 0) || it == 1;
        if (dj) std::copy(p->R, p->R + n, p->R0);
        lp_assemble(p, c->Tref, c->g, dj);
        dirichlet(p->R, p->bc_dofs, nullptr, p->bc_n);
        dirichlet(p->rate, p->bc_dofs, nullptr, p->bc_n);
        if (dj) { int rc = checked_lmax(p->dRdP, p->PC, n, "lithostatic pressure", lmax); if (rc) return rc; }
        for (int64_t i = 0; i < n; ++i) p->rate[i] = p->R[i] / p->PC[i] + bT * p->rate[i];
        for (int64_t i = 0; i < n; ++i) p->P[i] += aT * p->rate[i];
        dirichlet(p->P, p->bc_dofs, p->bc_vals, p->bc_n);
        if (dj) {
            double nr = norm2(p->R, n);
            if (it == 1) nr0 = std::max(nr, julia_eps(nr));
            if (std::isnan(nr / nr0)) { char b[64]; std::snprintf(b, sizeof b, "NaNs at PT iter %lld", (long long)it); g_last_error = b; return FEMB200_ENAN; }
            double dtau = 2 / std::sqrt(lmax) * p->cfl;
            double den = 0; for (int64_t i = 0; i < n; ++i) { double r = dtau * p->rate[i]; den += r * r; }
            double lmin = 0;
            if (!(it == 1 || den == 0)) {
                double num = 0;
                for (int64_t i = 0; i < n; ++i) num += dtau * p->rate[i] * ((p->R[i] - p->R0[i]) / p->PC[i]);
                lmin = std::fabs(num) / den;
            }
            double cc = 2 * std::sqrt(lmin) * p->c_fact;
            aT = 2 * dtau * dtau / (2 + cc * dtau);
            bT = (2 - cc * dtau) / (2 + cc * dtau);
            last_rel = nr / nr0;
            if (last_rel < c->tolerance) { st->converged = 1; st->iterations = it; st->residual = last_rel; return 0; }
        }
    }
    st->converged = 0; st->iterations = c->max_iterations; st->residual = last_rel;
    if (c->throw_on_failure) {
        char b[256];
        std::snprintf(b, sizeof b, "Lithostatic pressure DR solver did not converge after %lld pseudo-transient iterations (relative residual = %g)",
                      (long long)c->max_iterations, last_rel);
        g_last_error = b;
        return FEMB200_ENOTCONV;
    }
    return 0;
}

// ---- CellPressureStokesDR (viscous Hex27, four cell-local pressure modes) ----
// The modes (1, ξ, η, ζ) at the Gauss points (pressure_mode_table,
// momentum_residuals.jl:618-621); ξ, η, ζ are the P1 rows 2..4 of the tables.
inline double cp_mode(const Tables& t, int q, int m) { return m == 0 ? 1.0 : t.NP[q][m]; }

// ∂N_a/∂x_k at q from the element geometry (element_geometry, mesh.jl:504-507).
inline void cp_dNdx(const Tables& t, const double* g, int q, int a, double out[3]) {
    for (int k = 0; k < 3; ++k) out[k] = t.dN[q][a][0] * g[3 * k] + t.dN[q][a][1] * g[1 + 3 * k] + t.dN[q][a][2] * g[2 + 3 * k];
}

// stokes_preconditioner_3d_kernel! (momentum_residuals.jl:728-745)
void cp_preconditioner_impl(const femb200_cell_pressure_problem* p) {
    const Tables& t = tables_for(3);
    for (int c = 0; c < 3; ++c) std::fill(p->diagonal[c], p->diagonal[c] + p->nnodes, 0.0);
    std::fill(p->pressure_mass, p->pressure_mass + 4 * p->nels, 0.0);
    for (int64_t e = 0; e < p->nels; ++e) {
        const double eta = p->eta[p->phases[e] - 1];
        for (int q = 0; q < 27; ++q) {
            const double* g = p->geo_v + (e * 27 + q) * 10;
            const double dO = g[9];
            for (int a = 0; a < 27; ++a) {
                double gr[3];
                cp_dNdx(t, g, q, a, gr);
                const int64_t node = p->el2n[27 * e + a] - 1;
                const double n2 = gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2];
                for (int c = 0; c < 3; ++c) p->diagonal[c][node] += eta * (n2 + gr[c] * gr[c] / 3) * dO;
            }
            for (int m = 0; m < 4; ++m) p->pressure_mass[4 * e + m] += cp_mode(t, q, m) * cp_mode(t, q, m) * dO;
        }
    }
}

// velocity gradient ∂v_c/∂x_k at q
inline void cp_grad(const Tables& t, const femb200_cell_pressure_problem* p, int64_t e, int q, double gv[3][3]) {
    const double* g = p->geo_v + (e * 27 + q) * 10;
    for (int c = 0; c < 3; ++c)
        for (int k = 0; k < 3; ++k) gv[c][k] = 0;
    for (int a = 0; a < 27; ++a) {
        double gr[3];
        cp_dNdx(t, g, q, a, gr);
        const int64_t node = p->el2n[27 * e + a] - 1;
        for (int c = 0; c < 3; ++c)
            for (int k = 0; k < 3; ++k) gv[c][k] += p->v[c][node] * gr[k];
    }
}

// stokes_pressure_residual_3d_kernel! (pressure_residual.jl:352-364): RP = −Σ mode ∇·v dΩ
void cp_pressure_residual_impl(const femb200_cell_pressure_problem* p) {
    const Tables& t = tables_for(3);
    for (int64_t e = 0; e < p->nels; ++e) {
        double r[4] = {0, 0, 0, 0};
        for (int q = 0; q < 27; ++q) {
            double gv[3][3];
            cp_grad(t, p, e, q, gv);
            const double dO = p->geo_v[(e * 27 + q) * 10 + 9];
            const double div = gv[0][0] + gv[1][1] + gv[2][2];
            for (int m = 0; m < 4; ++m) r[m] -= cp_mode(t, q, m) * (div * dO);
        }
        for (int m = 0; m < 4; ++m) p->RP[4 * e + m] = r[m];
    }
}

// stokes_momentum_residual_3d_kernel! (momentum_residuals.jl:675-700) through
// integrate_momentum_residual (:221-258) with G = K = ∞, α = 0: viscous stress 2ηε̇′,
// pressure from the modes, ρ = interp(ρ0), accumulate_momentum (:28-33).
void cp_momentum_residual_impl(const femb200_cell_pressure_problem* p) {
    const Tables& t = tables_for(3);
    for (int c = 0; c < 3; ++c) std::fill(p->Rv[c], p->Rv[c] + p->nnodes, 0.0);
    for (int64_t e = 0; e < p->nels; ++e) {
        const int ph = p->phases[e] - 1;
        double R[3][27] = {{0}};
        for (int q = 0; q < 27; ++q) {
            const double* g = p->geo_v + (e * 27 + q) * 10;
            const double dO = g[9];
            double gv[3][3];
            cp_grad(t, p, e, q, gv);
            double eta_q = 0, rho_q = 0;     // interp2ip_phase over the cell's (single) phase
            for (int a = 0; a < 27; ++a) { eta_q += t.N[q][a] * p->eta[ph]; rho_q += t.N[q][a] * p->rho[ph]; }
            const double tr = (gv[0][0] + gv[1][1] + gv[2][2]) / 3;
            double Pq = 0;
            for (int m = 0; m < 4; ++m) Pq += cp_mode(t, q, m) * p->P[4 * e + m];
            double sig[3][3];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    sig[i][j] = 2 * eta_q * ((gv[i][j] + gv[j][i]) / 2 - (i == j ? tr : 0.0)) - (i == j ? Pq : 0.0);
            for (int a = 0; a < 27; ++a) {
                double gr[3];
                cp_dNdx(t, g, q, a, gr);
                for (int i = 0; i < 3; ++i) {
                    double f = 0;
                    for (int j = 0; j < 3; ++j) f += gr[j] * sig[j][i];
                    R[i][a] += (f - t.N[q][a] * (rho_q * p->g[i])) * dO;
                }
            }
        }
        for (int a = 0; a < 27; ++a) {
            const int64_t node = p->el2n[27 * e + a] - 1;
            for (int i = 0; i < 3; ++i) p->Rv[i][node] += R[i][a];
        }
    }
}

inline void cp_dirichlet(double* x, const int32_t* dofs, const double* vals, int64_t n) {
    for (int64_t i = 0; i < n; ++i) x[dofs[i] - 1] = vals ? vals[i] : 0.0;
}

// _relax_cell_pressure_stokes! (DR.jl:1004-1057)
int cp_solve_impl(const femb200_cell_pressure_problem* p, const femb200_cell_pressure_controls* c,
                  femb200_cell_pressure_stats* st) {
    std::memset(st, 0, sizeof(*st));
    cp_preconditioner_impl(p);
    for (int k = 0; k < 3; ++k) cp_dirichlet(p->v[k], p->bc_dofs[k], p->bc_vals[k], p->bc_n[k]);
    double err_v = INFINITY, err_P = INFINITY, err = INFINITY;
    int64_t iter = 0, hist = 0;
    for (int64_t it = 1; it <= c->max_iterations; ++it) {
        iter = it;
        cp_pressure_residual_impl(p);
        for (int64_t i = 0; i < 4 * p->nels; ++i) p->P[i] += c->pressure_step * p->RP[i] / p->pressure_mass[i];
        double s0 = 0, s1 = 0;
        for (int64_t e = 0; e < p->nels; ++e) { s0 += p->P[4 * e] * p->pressure_mass[4 * e]; s1 += p->pressure_mass[4 * e]; }
        const double pmean = s0 / s1;
        for (int64_t e = 0; e < p->nels; ++e) p->P[4 * e] -= pmean;
        cp_momentum_residual_impl(p);
        for (int k = 0; k < 3; ++k) {
            if (p->load[k])
                for (int64_t i = 0; i < p->nnodes; ++i) p->Rv[k][i] -= p->load[k][i];
            cp_dirichlet(p->Rv[k], p->bc_dofs[k], nullptr, p->bc_n[k]);
            for (int64_t i = 0; i < p->nnodes; ++i) p->v[k][i] -= c->velocity_step * p->Rv[k][i] / p->diagonal[k][i];
            cp_dirichlet(p->v[k], p->bc_dofs[k], p->bc_vals[k], p->bc_n[k]);
        }
        if (!(it % c->check_interval == 0 || it == c->max_iterations)) continue;
        err_v = 0;
        for (int k = 0; k < 3; ++k) {
            double ss = 0;
            for (int64_t i = 0; i < p->nnodes; ++i) ss += p->Rv[k][i] * p->Rv[k][i];
            err_v = jl_max(err_v, std::sqrt(ss));
        }
        double sp = 0;
        for (int64_t i = 0; i < 4 * p->nels; ++i) sp += p->RP[i] * p->RP[i];
        err_P = std::sqrt(sp);
        err = jl_max(err_v, err_P);
        if (!std::isfinite(err)) { g_last_error = "non-finite residual in 3-D Stokes solve"; return FEMB200_ENONFINITE; }
        if (c->history && hist < c->history_capacity) {
            c->history[3 * hist] = (double)it; c->history[3 * hist + 1] = err_v; c->history[3 * hist + 2] = err_P;
            ++hist;
        }
        if (err < c->tolerance) break;
    }
    st->converged = err < c->tolerance;
    st->iterations = iter;
    st->residual = err; st->err_v = err_v; st->err_P = err_P;
    st->reached_total_iter = iter >= c->max_iterations && !st->converged;
    st->history_len = hist;
    if (!st->converged && c->throw_on_failure) {
        char b[160];
        std::snprintf(b, sizeof b, "3-D Stokes solve did not converge after %lld iterations (residual = %g, tolerance = %g)",
                      (long long)iter, err, c->tolerance);
        g_last_error = b;
        return FEMB200_ENOTCONV;
    }
    return FEMB200_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C API used by the tests and by bench.py's CPU baseline.
// ---------------------------------------------------------------------------
extern "C" {

const char* orc_last_error(void) { return g_last_error.c_str(); }

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

// Reference tables: N (nq×nv), dN (nq×nv×dim), NP (nq×np), w (nq).
int orc_tables(int dim, double* N, double* dN, double* NP, double* w, int32_t* prow) {
    const Tables& t = tables_for(dim);
    for (int q = 0; q < t.nq; ++q) {
        for (int a = 0; a < t.nv; ++a) {
            N[q * t.nv + a] = t.N[q][a];
            for (int j = 0; j < t.dim; ++j) dN[(q * t.nv + a) * t.dim + j] = t.dN[q][a][j];
        }
        for (int i = 0; i < t.np; ++i) NP[q * t.np + i] = t.NP[q][i];
        w[q] = t.w[q];
    }
    for (int i = 0; i < t.np; ++i) prow[i] = t.prow[i] + 1;
    return 0;
}

// Structured Hex27 (dim 3) or Q9 (dim 2) mixed mesh on a box: coordinates
// (dim × nnodes), el2n, P1-disc DoFs (generate_discontinuous_linear_mesh,
// mixed_mesh.jl:436-457) and the pressure-carrying velocity nodes.
int orc_structured_mesh(int dim, int nx, int ny, int nz, const double* lo, const double* hi, double* coords,
                        int32_t* el2n, int32_t* dofsP, int32_t* el2nP) {
    const Tables& t = tables_for(dim);
    int64_t n[3] = {2 * nx + 1, 2 * ny + 1, dim == 3 ? 2 * nz + 1 : 1};
    int64_t ne[3] = {nx, ny, dim == 3 ? nz : 1};
    int64_t inode = 0;
    for (int64_t k = 0; k < n[2]; ++k)
        for (int64_t j = 0; j < n[1]; ++j)
            for (int64_t i = 0; i < n[0]; ++i, ++inode) {
                int64_t idx[3] = {i, j, k};
                for (int d = 0; d < dim; ++d) {
                    // LinRange(lo, hi, n): ((n-1-i)·lo + i·hi)/(n-1), exact for lo = 0
                    double len = (double)(n[d] - 1);
                    coords[dim * inode + d] = lo[d] == 0.0 ? (double)idx[d] / len * hi[d]
                                                           : ((len - idx[d]) / len) * lo[d] + ((double)idx[d] / len) * hi[d];
                }
            }
    (void)ne;
    int64_t nels = (int64_t)nx * ny * (dim == 3 ? nz : 1);
    if (dim == 3) hex27_el2n(nx, ny, nz, el2n); else q9_el2n(nx, ny, el2n);
    for (int64_t e = 0; e < nels; ++e)
        for (int i = 0; i < t.np; ++i) {
            dofsP[t.np * e + i] = (int32_t)(t.np * e + i + 1);
            el2nP[t.np * e + i] = el2n[(int64_t)t.nv * e + t.prow[i]];
        }
    return 0;
}

int orc_geometry(int dim, int64_t nels, const double* coords, const int32_t* el2n, double* geo_v, double* geo_P) {
    geometry(dim, nels, coords, el2n, geo_v, geo_P);
    return 0;
}

// compute_strain_rate_stress_postprocess from integration-point stresses
// (src/postprocess/postprocess.jl:17-79 in 2-D, :168-215 in 3-D): per element the
// dΩ-weighted averages of ε (from ∂N∂x = ∂N∂ξ·J⁻¹, mesh.jl:504-507), its deviatoric
// second invariant, τ and τII. 3-D invariants carry the eps² floor of
// second_invariant (rheology.jl:395-400); the 2-D ones are formed without it (:52-53).
int orc_strain_rate_stress(int dim, int64_t nels, const int32_t* el2n, const double* geo_v, const double* const* v,
                           const double* const* tau, double* const* out) {
    const Tables& t = tables_for(dim);
    const int D = dim, NV = t.nv, NQ = t.nq, S = D * D + 1, NF = dim == 3 ? 14 : 10;
    const double e2 = 2.220446049250313e-16 * 2.220446049250313e-16;
    for (int64_t e = 0; e < nels; ++e) {
        double tot[14] = {0}, vol = 0;
        for (int q = 0; q < NQ; ++q) {
            const double* g = geo_v + ((int64_t)e * NQ + q) * S;
            double gv[3][3] = {{0}};
            for (int a = 0; a < NV; ++a) {
                const int64_t node = el2n[(int64_t)NV * e + a] - 1;
                for (int k = 0; k < D; ++k) {
                    double dNdx = 0;
                    for (int j = 0; j < D; ++j) dNdx += t.dN[q][a][j] * g[j + D * k];
                    for (int c = 0; c < D; ++c) gv[c][k] += dNdx * v[c][node];
                }
            }
            const double dO = g[D * D];
            const int64_t iq = (int64_t)e * NQ + q;
            double f[14];
            if (D == 3) {
                const double eps_[6] = {gv[0][0], gv[1][1], gv[2][2], (gv[0][1] + gv[1][0]) / 2,
                                        (gv[0][2] + gv[2][0]) / 2, (gv[1][2] + gv[2][1]) / 2};
                const double tr = (eps_[0] + eps_[1] + eps_[2]) / 3;
                const double dv[6] = {eps_[0] - tr, eps_[1] - tr, eps_[2] - tr, eps_[3], eps_[4], eps_[5]};
                const double eII = std::sqrt((dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]) / 2 + dv[3] * dv[3] +
                                             dv[4] * dv[4] + dv[5] * dv[5] + e2);
                double tq[6];
                for (int c = 0; c < 6; ++c) tq[c] = tau[c][iq];
                const double tII = std::sqrt((tq[0] * tq[0] + tq[1] * tq[1] + tq[2] * tq[2]) / 2 + tq[3] * tq[3] +
                                             tq[4] * tq[4] + tq[5] * tq[5] + e2);
                for (int c = 0; c < 6; ++c) f[c] = eps_[c];
                f[6] = eII;
                for (int c = 0; c < 6; ++c) f[7 + c] = tq[c];
                f[13] = tII;
            } else {
                const double exx = gv[0][0], eyy = gv[1][1], ezz = 0.0, exy = (gv[0][1] + gv[1][0]) / 2;
                const double tr = (exx + eyy + ezz) / 3;
                const double d0 = exx - tr, d1 = eyy - tr, d2 = ezz - tr;
                const double eII = std::sqrt((d0 * d0 + d1 * d1 + d2 * d2) / 2 + exy * exy);
                const double txx = tau[0][iq], tyy = tau[1][iq], txy = tau[2][iq], tzz = -(txx + tyy);
                const double tII = std::sqrt((txx * txx + tyy * tyy + tzz * tzz) / 2 + txy * txy);
                const double ff[10] = {exx, eyy, ezz, exy, eII, txx, tyy, tzz, txy, tII};
                for (int k = 0; k < 10; ++k) f[k] = ff[k];
            }
            for (int k = 0; k < NF; ++k) tot[k] += f[k] * dO;
            vol += dO;
        }
        for (int k = 0; k < NF; ++k) out[k][e] = tot[k] / vol;
    }
    return 0;
}

int orc_pressure_residual(const femb200_stokes_problem* p, double dt, int32_t finite_K) {
    int rc = check_problem(p); if (rc) return rc;
    pressure_residual_impl(p, dt, finite_K);
    return 0;
}

int orc_momentum_residual(const femb200_stokes_problem* p, double dt, int32_t with_pnum) {
    int rc = check_problem(p); if (rc) return rc;
    momentum_residual_impl(p, dt, with_pnum != 0);
    return 0;
}

int orc_stokes_residuals(const femb200_stokes_problem* p, double dt, int32_t finite_K) {
    int rc = check_problem(p); if (rc) return rc;
    pressure_residual_impl(p, dt, finite_K);
    for (int64_t i = 0; i < p->nnodesP; ++i) Dm(p->Pnum)[i] = D(p->gammaP)[i] * D(p->RP)[i] / D(p->M_P)[i];
    momentum_residual_impl(p, dt, true);
    return 0;
}

int orc_jacobian_diagnostics(const femb200_stokes_problem* p, double dt, int32_t finite_K) {
    int rc = check_problem(p); if (rc) return rc;
    jacobian_impl(p, dt, finite_K);
    return 0;
}

int orc_pressure_scaling(const femb200_stokes_problem* p, double gamma_fact, double dt, int32_t finite_K) {
    int rc = check_problem(p); if (rc) return rc;
    pressure_scaling_impl(p, gamma_fact, dt, finite_K);
    return 0;
}

int orc_store_stress(const femb200_stokes_problem* p, double dt) {
    int rc = check_problem(p); if (rc) return rc;
    // update_stokes_current_stress! uses the material viscosity dr.η (DR.jl:890)
    femb200_stokes_problem q = *p; q.viscosity_ip = nullptr;
    double* cols[6];
    for (int c = 0; c < 6; ++c) cols[c] = static_cast<double*>(q.tau[c]);
    momentum_residual_impl(&q, dt, false, cols);
    return 0;
}

int orc_solve_stokes(const femb200_stokes_problem* p, const femb200_stokes_controls* c, femb200_stokes_stats* st) {
    return solve_stokes_impl(p, c, st, nullptr);
}

// Timed CPU sample of the solve: `iterations` inner DR iterations exactly as the
// solve runs them (stokes_inner_step, with the given Chebyshev steps and the
// preconditioner already in p->PC), then, when `check` is set, one check's work
// without its Jacobian assembly: Rv → Rv0 before the last iteration, the velocity
// error and λmin. Returns the velocity error of the check (0 without one) in *err_v.
int orc_dr_iterations(const femb200_stokes_problem* p, double dt, int32_t finite_K, const double* alpha,
                      const double* beta, int64_t iterations, int32_t check, double* err_v) {
    int rc = check_problem(p); if (rc) return rc;
    double ev = 0;
    for (int64_t it = 1; it <= iterations; ++it) {
        const bool last_check = check && it == iterations;
        if (last_check)
            for (int k = 0; k < p->dim; ++k) std::copy(D(p->Rv[k]), D(p->Rv[k]) + p->nnodes, Dm(p->Rv0[k]));
        stokes_inner_step(p, dt, finite_K, alpha, beta);
        if (last_check) { double lmin[3]; ev = stokes_check_norms(p, alpha, lmin); }
    }
    if (err_v) *err_v = ev;
    return 0;
}

// The Jacobian diagnostics assembled from elements [e0, e1) into the full-size
// dRdv / PC arrays (zeroed first), the assembly of the solve restricted to a block.
int orc_jacobian_range(const femb200_stokes_problem* p, double dt, int32_t finite_K, int64_t e0, int64_t e1) {
    int rc = check_problem(p); if (rc) return rc;
    if (e0 < 0 || e1 > p->nels || e0 > e1) { g_last_error = "element range outside 0:nels"; return FEMB200_EINVAL; }
    jacobian_impl(p, dt, finite_K, e0, e1);
    return 0;
}

int orc_thermal_residual(const femb200_thermal_problem* t, double dt, double Tref, int32_t jac) {
    thermal_assemble(t, dt, Tref, jac != 0);
    return 0;
}

// solve_dynamic_relaxation! (src/dynamic_relaxation/solver.jl:61-122).
int orc_solve_thermal(const femb200_thermal_problem* tp, const femb200_thermal_controls* c, femb200_thermal_stats* st) {
    const int64_t n = tp->nnodes;
    double aT = 0, bT = 0, nr0 = 0, last_rel = NAN, lmax = 0;
    for (int64_t it = 1; it <= c->max_iterations; ++it) {
        bool dj = (it % c->check_interval == 0) || it == 1;
        if (dj) std::copy(D(tp->R), D(tp->R) + n, Dm(tp->R0));
        thermal_assemble(tp, c->dt, c->Tref, dj);
        dirichlet(Dm(tp->R), tp->bc_dofs, nullptr, tp->bc_n);
        dirichlet(Dm(tp->rate), tp->bc_dofs, nullptr, tp->bc_n);
        if (dj) { int rc = checked_lmax(D(tp->dRdT), D(tp->PC), n, "thermal diffusion", lmax); if (rc) return rc; }
        for (int64_t i = 0; i < n; ++i) Dm(tp->rate)[i] = D(tp->R)[i] / D(tp->PC)[i] + bT * D(tp->rate)[i];
        for (int64_t i = 0; i < n; ++i) Dm(tp->T)[i] += aT * D(tp->rate)[i];
        dirichlet(Dm(tp->T), tp->bc_dofs, D(tp->bc_vals), tp->bc_n);
        if (dj) {
            double nr = norm2(D(tp->R), n);
            if (it == 1) nr0 = std::max(nr, julia_eps(nr));
            if (std::isnan(nr / nr0)) { char b[64]; std::snprintf(b, sizeof b, "NaNs at PT iter %lld", (long long)it); g_last_error = b; return FEMB200_ENAN; }
            double dtau = 2 / std::sqrt(lmax) * tp->cfl;
            double den = 0; for (int64_t i = 0; i < n; ++i) { double r = dtau * D(tp->rate)[i]; den += r * r; }
            double lmin = 0;
            if (!(it == 1 || den == 0)) {
                double num = 0;
                for (int64_t i = 0; i < n; ++i) num += dtau * D(tp->rate)[i] * ((D(tp->R)[i] - D(tp->R0)[i]) / D(tp->PC)[i]);
                lmin = std::fabs(num) / den;
            }
            double cc = 2 * std::sqrt(lmin) * tp->c_fact;
            aT = 2 * dtau * dtau / (2 + cc * dtau);
            bT = (2 - cc * dtau) / (2 + cc * dtau);
            last_rel = nr / nr0;
            if (last_rel < c->tolerance) { st->converged = 1; st->iterations = it; st->residual = last_rel; return 0; }
        }
    }
    st->converged = 0; st->iterations = c->max_iterations; st->residual = last_rel;
    if (c->throw_on_failure) {
        char b[256];
        std::snprintf(b, sizeof b, "Thermal diffusion DR solver did not converge after %lld pseudo-transient iterations (relative residual = %g)",
                      (long long)c->max_iterations, last_rel);
        g_last_error = b;
        return FEMB200_ENOTCONV;
    }
    return 0;
}

int orc_transfer_temperature(double* TP, const double* T, const int32_t* dofsP, const int32_t* el2nP, int64_t n) {
    transfer_T(TP, T, dofsP, el2nP, n);
    return 0;
}

int orc_stokes_adjoint_residual(const femb200_stokes_problem* p, double dt, int32_t finite_K, int32_t with_pnum,
                                const double* const lam_v[3], const double* lam_P, double* const out_dv[3],
                                double* out_dP) {
    int rc = check_problem(p);
    if (rc) return rc;
    if (p->dim != 3) { g_last_error = "the adjoint oracle is 3-D (Hex27) only"; return FEMB200_EUNSUPPORTED; }
    adjoint_residual_impl(p, dt, finite_K, with_pnum != 0, lam_v, lam_P, out_dv, out_dP);
    return FEMB200_OK;
}

int orc_stokes_viscosity_sensitivity(const femb200_stokes_problem* p, double dt, int32_t finite_K, int32_t with_pnum,
                                     const double* const lam_v[3], const double* lam_P, double* out_eta_ip) {
    int rc = check_problem(p);
    if (rc) return rc;
    if (p->dim != 3) { g_last_error = "the adjoint oracle is 3-D (Hex27) only"; return FEMB200_EUNSUPPORTED; }
    viscosity_sensitivity_impl(p, dt, finite_K, with_pnum != 0, lam_v, lam_P, out_eta_ip);
    return FEMB200_OK;
}

// One synthetic thermal element (the reference's integrate_residual unit-test setup):
// nq points with shape values N (nq × nv), physical gradients dNdx (nq × nv × dim) and
// weights dOmega; nodal T, T0, source, P and 1-based phases; the material of tp.
int orc_thermal_element_custom(int dim, int nv, int nq, const double* N, const double* dNdx, const double* dOmega,
                               const double* T, const double* T0, const double* src, const double* P,
                               const int32_t* ph, const femb200_thermal_problem* tp, double dt, double Tref,
                               double* R_out) {
    if (nv > 27 || nq > 27 || (dim != 2 && dim != 3)) return FEMB200_EINVAL;
    static thread_local Tables t;
    std::memset(&t, 0, sizeof(t));
    t.dim = dim; t.nv = nv; t.nq = nq;
    for (int q = 0; q < nq; ++q)
        for (int a = 0; a < nv; ++a) {
            t.N[q][a] = N[q * nv + a];
            for (int j = 0; j < dim; ++j) t.dN[q][a][j] = dNdx[(q * nv + a) * dim + j];
        }
    std::vector<double> geo((size_t)nq * (dim * dim + 1), 0.0);
    for (int q = 0; q < nq; ++q) {
        for (int d = 0; d < dim; ++d) geo[q * (dim * dim + 1) + d + dim * d] = 1.0;
        geo[q * (dim * dim + 1) + dim * dim] = dOmega[q];
    }
    TElem el;
    std::memset(&el, 0, sizeof(el));
    el.NV = nv; el.NQ = nq; el.D = dim; el.geo = geo.data(); el.hasPhi = false;
    for (int a = 0; a < nv; ++a) {
        el.T0[a] = T0[a]; el.s[a] = src ? src[a] : 0.0; el.P[a] = P ? P[a] : 0.0; el.ph[a] = ph ? ph[a] - 1 : 0;
    }
    double Re[27];
    thermal_element<double>(t, el, tp, T, dt, Tref, Re);
    for (int a = 0; a < nv; ++a) R_out[a] = Re[a];
    return 0;
}

// shear_dissipation at one point: g is ∂v_i/∂x_k row-major (dim × dim).
int orc_shear_dissipation(int dim, const double* tau, const double* tau_old, const double* grad, double inv2Gdt,
                          double* out) {
    if (dim != 2 && dim != 3) return FEMB200_EINVAL;
    double g[3][3] = {{0}};
    for (int i = 0; i < dim; ++i)
        for (int k = 0; k < dim; ++k) g[i][k] = grad[i * dim + k];
    *out = shear_dissipation(dim, tau, tau_old, g, inv2Gdt);
    return 0;
}

int orc_shear_heating(const femb200_stokes_problem* p, double dt, double* phi) {
    int rc = check_problem(p); if (rc) return rc;
    shear_heating_impl(p, dt, phi);
    return 0;
}

// solve_coupled! (src/stokes/solvers/DR.jl:89-135).
int orc_solve_coupled(femb200_thermal_problem* t, const femb200_stokes_problem* p, const femb200_stokes_controls* c,
                      double Tref, int32_t shear_heating, double* phi, femb200_stokes_stats* st) {
    int rc = check_problem(p); if (rc) return rc;
    transfer_T(Dm(p->T), D(t->T), p->dofsP, p->el2nP, (int64_t)p->np * p->nels);
    transfer_T(Dm(p->T0), D(t->T0), p->dofsP, p->el2nP, (int64_t)p->np * p->nels);
    if (shear_heating && phi) std::fill(phi, phi + (int64_t)p->nq * p->nels, 0.0);
    Coupled cp{t, Tref, shear_heating ? phi : nullptr};
    rc = solve_stokes_impl(p, c, st, &cp);
    return rc;
}

int orc_cell_pressure_preconditioner(const femb200_cell_pressure_problem* p) {
    cp_preconditioner_impl(p);
    return 0;
}

int orc_cell_pressure_residuals(const femb200_cell_pressure_problem* p, int32_t which) {
    if (which & 1) cp_pressure_residual_impl(p);
    if (which & 2) cp_momentum_residual_impl(p);
    return 0;
}

int orc_solve_cell_pressure(const femb200_cell_pressure_problem* p, const femb200_cell_pressure_controls* c,
                            femb200_cell_pressure_stats* st) {
    return cp_solve_impl(p, c, st);
}

int orc_lithostatic_residual(const femb200_lithostatic_problem* p, double Tref, const double* g, int32_t jac) {
    lp_assemble(p, Tref, g, jac != 0);
    return 0;
}

int orc_solve_lithostatic(const femb200_lithostatic_problem* p, const femb200_lithostatic_controls* c,
                          femb200_thermal_stats* st) {
    return lp_solve_impl(p, c, st);
}

// One element of the lithostatic residual from given shape functions N (nq × nv),
// physical gradients dNdx (nq × nv × dim) and weights dΩ (nq): the element-level
// checks of the reference's tests are stated this way.
int orc_lithostatic_element_custom(int dim, int nv, int nq, const double* N, const double* dNdx, const double* dO,
                                   const double* P, const double* T, const int32_t* ph, const double* rho0,
                                   const double* alpha, const double* K, double Tref, const double* g,
                                   double* R, double* rows, double* diag) {
    if (nv > 9 || nq > 27 || (dim != 2 && dim != 3)) return FEMB200_EINVAL;
    double beta[FEMB200_MAX_PHASES];
    for (int i = 0; i < FEMB200_MAX_PHASES; ++i) beta[i] = 1.0 / K[i];
    int p0[27];
    for (int a = 0; a < nv; ++a) p0[a] = ph[a] - 1;
    lp_element_all<9>(nv, dim, nq, N, dNdx, dO, P, T, p0, rho0, alpha, beta, Tref, g, true, R, rows, diag);
    return 0;
}

}  // extern "C"

// Element-level entry point with caller-supplied tables and physical gradients,
// used to restate the reference's element unit tests, which build one-point
// elements with J⁻¹ = I (_stokes_geo_el, test/test_stokes.jl:42-43).
extern "C" int orc_element_custom(int dim, int nv, int np, int nq, const double* N, const double* dNdx,
                                  const double* dOmega, const double* NPt, const double* v, const double* P,
                                  const double* P0, const double* T, const double* T0, const double* Q,
                                  const double* Pnum, const int32_t* phv, const int32_t* php,
                                  const double* tau_old, const double* P0_ip,
                                  const femb200_stokes_material* m, double dt, int32_t finite_K,
                                  double* R_out, double* RP_out, double* tau_out) {
    if (nv > 27 || np > 4 || nq > 27 || (dim != 2 && dim != 3)) return FEMB200_EINVAL;
    static thread_local Tables t;
    std::memset(&t, 0, sizeof(t));
    t.dim = dim; t.nv = nv; t.np = np; t.nq = nq;
    for (int q = 0; q < nq; ++q) {
        for (int a = 0; a < nv; ++a) {
            t.N[q][a] = N[q * nv + a];
            for (int j = 0; j < dim; ++j) t.dN[q][a][j] = dNdx[(q * nv + a) * dim + j];
        }
        for (int i = 0; i < np; ++i) t.NP[q][i] = NPt[q * np + i];
    }
    Elem el; std::memset(&el, 0, sizeof(el));
    el.D = dim; el.NV = nv; el.NP = np; el.NQ = nq; el.iel = 0;
    std::vector<double> geo((size_t)nq * (dim * dim + 1), 0.0), geoP(nq);
    for (int q = 0; q < nq; ++q) {
        for (int d = 0; d < dim; ++d) geo[q * (dim * dim + 1) + d + dim * d] = 1.0;
        geo[q * (dim * dim + 1) + dim * dim] = dOmega[q];
        geoP[q] = dOmega[q];
    }
    el.geo = geo.data(); el.geoP = geoP.data();
    for (int i = 0; i < np; ++i) {
        el.P[i] = P[i]; el.P0[i] = P0 ? P0[i] : 0.0; el.T[i] = T ? T[i] : 0.0; el.T0[i] = T0 ? T0[i] : 0.0;
        el.Q[i] = Q ? Q[i] : 0.0; el.Pnum[i] = Pnum ? Pnum[i] : 0.0; el.MP[i] = 1.0;
        el.php[i] = php ? php[i] - 1 : 0;
    }
    el.hasQ = Q != nullptr; el.hasPf = false;
    el.P0_ip = P0_ip != nullptr;
    if (P0_ip) for (int q = 0; q < nq; ++q) el.P0q[q] = P0_ip[q];
    for (int a = 0; a < nv; ++a) el.phv[a] = phv ? phv[a] - 1 : 0;
    const int NT = dim == 3 ? 6 : 3;
    el.has_told = tau_old != nullptr;
    for (int q = 0; q < nq; ++q) for (int c = 0; c < NT; ++c) el.told[q][c] = tau_old ? tau_old[q * NT + c] : 0.0;
    el.eta_ip = false;
    double vv[3][27] = {{0}};
    for (int c = 0; c < dim; ++c) for (int a = 0; a < nv; ++a) vv[c][a] = v[c * nv + a];
    double RP[4];
    pressure_element<double>(t, el, vv, finite_K ? m->K : m->eta_b, m->alpha, dt, Q != nullptr, RP);
    if (RP_out) for (int i = 0; i < np; ++i) RP_out[i] = RP[i];
    double R[3][27];
    double tst[6 * 27];
    momentum_element<double>(t, el, *m, vv, Pnum, m->eta, 0.0, dt, R, tst, 27);
    if (R_out) for (int c = 0; c < dim; ++c) for (int a = 0; a < nv; ++a) R_out[c * nv + a] = R[c][a];
    if (tau_out) for (int q = 0; q < nq; ++q) for (int c = 0; c < NT; ++c) tau_out[q * NT + c] = tst[c * 27 + q];
    return 0;
}
