// simple.cu — thread-per-element kernels: pressure scaling (setup, once per
// solve), the Q9/P1-disc plane-strain residual and Jacobian diagnostics (2-D
// problems are small), and the thermal-diffusion residual/Jacobian.
#include "kernels.cuh"

namespace femb {

__constant__ DevThermalMaterial c_tmat;

namespace {

template <int DIM> struct Tabs;
template <> struct Tabs<3> {
    static constexpr int NV = 27, NQ = 27, NP = 4;
    FEMB_D static double N(int q, int a) { return c_tab.N3[q][a]; }
    FEMB_D static double dN(int q, int a, int j) { return c_tab.dN3[q][a][j]; }
    FEMB_D static double NPq(int q, int p) { return c_tab.NP3[q][p]; }
    FEMB_D static double sumN(int q) { return c_tab.sumN3[q]; }
};
template <> struct Tabs<2> {
    static constexpr int NV = 9, NQ = 9, NP = 3;
    FEMB_D static double N(int q, int a) { return c_tab.N2[q][a]; }
    FEMB_D static double dN(int q, int a, int j) { return c_tab.dN2[q][a][j]; }
    FEMB_D static double NPq(int q, int p) { return c_tab.NP2[q][p]; }
    FEMB_D static double sumN(int q) { return c_tab.sumN2[q]; }
};

// interp2ip_phase over the element's velocity-node phases (utils.jl:37-44).
template <int DIM, class T>
FEMB_D T interp(int q, const double* var, const int* ph) {
    T out = T(0);
#pragma unroll
    for (int a = 0; a < Tabs<DIM>::NV; ++a) out += (T)Tabs<DIM>::N(q, a) * (T)var[ph[a]];
    return out;
}

// viscosity_weighted_pressure_scaling_kernel! (pressure_scaling.jl:166-211);
// Q9 and Hex27 use the positive Jacobi weight N² (:201-203).
template <int DIM, class T, class TG>
__global__ void pressure_scaling_kernel(const int32_t* el2n, const int32_t* dofsP, const TG* geo_P, const int32_t* phv,
                                        int phv_layout, const T* eta_ip, int use_eta_ip, T* MP, T* gP, int64_t nels,
                                        T gfact, T dt) {
    using TB = Tabs<DIM>;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nels) return;
    int ph[TB::NV];
    for (int a = 0; a < TB::NV; ++a)
        ph[a] = phase_of(phv, phv_layout, (int64_t)__ldg(el2n + TB::NV * e + a), a, e, TB::NV);
    int dof[TB::NP];
    for (int p = 0; p < TB::NP; ++p) dof[p] = __ldg(dofsP + TB::NP * e + p) - 1;
    for (int q = 0; q < TB::NQ; ++q) {
        const T dO = (T)ld(geo_P + e * TB::NQ + q);
        const T etaq = use_eta_ip ? ld(eta_ip + e * TB::NQ + q) : interp<DIM, T>(q, c_mat.eta_scaling, ph);
        const T gnum = gfact * etaq;
        const T bq = interp<DIM, T>(q, c_mat.inv_Kscale, ph);
        const T gphy = bq == T(0) ? gnum : dt / bq;
        const T gq = gphy * gnum / (gphy + gnum);
        for (int p = 0; p < TB::NP; ++p) {
            const T NPv = (T)TB::NPq(q, p);
            const T w = NPv * NPv * dO;
            atomic_add(MP + dof[p], w);
            atomic_add(gP + dof[p], w * gq);
        }
    }
}

template <class T>
__global__ void scaling_finalize_kernel(T* gP, const T* MP, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) gP[i] = MP[i] == T(0) ? T(0) : gP[i] / MP[i];
}

// Plane-strain stress with the plane-strain Drucker–Prager return (rheology.jl:226-334).
// Returns the trial state needed by the linearisation.
template <class T>
struct PsState {
    T tt[3], tau[3], etave, lam, tII, tIIs, den;
};

template <class T>
FEMB_D void ps_stress(const T g[2][2], T etave, T inv2Gdt, const T told[3], bool plastic, T cphi, T sphi, T spsi, T C,
                      T ereg, T Kb, T dt, T Peq, PsState<T>& s) {
    const T exx = g[0][0], eyy = g[1][1], exy = (g[0][1] + g[1][0]) / T(2);
    const T tr = (exx + eyy) / T(3);
    s.tt[0] = (T(2) * etave) * ((exx - tr) + told[0] * inv2Gdt);
    s.tt[1] = (T(2) * etave) * ((eyy - tr) + told[1] * inv2Gdt);
    s.tt[2] = (T(2) * etave) * (exy + told[2] * inv2Gdt);
    s.etave = etave;
    s.lam = T(0); s.tII = T(1); s.tIIs = T(1); s.den = T(1);
    for (int c = 0; c < 3; ++c) s.tau[c] = s.tt[c];
    if (!plastic) return;
    const T tzz = -s.tt[0] - s.tt[1];
    const T tII = sqrt((s.tt[0] * s.tt[0] + s.tt[1] * s.tt[1] + tzz * tzz) / T(2) + s.tt[2] * s.tt[2] + eps2<T>());
    const T tIIs = tII + eps2<T>();
    const T F = tII - cphi * C - sphi * Peq;
    const T den = etave + ereg + Kb * dt * (-spsi) * (-sphi);
    const T lam = F > T(0) ? F / den : T(0);
    s.lam = lam; s.tII = tII; s.tIIs = tIIs; s.den = den;
    if (lam > T(0)) {
        const T dQ[3] = {(T(2) * s.tt[0] + s.tt[1]) / (T(2) * tIIs), (s.tt[0] + T(2) * s.tt[1]) / (T(2) * tIIs), s.tt[2] / tIIs};
        for (int c = 0; c < 3; ++c) s.tau[c] = s.tt[c] - T(2) * etave * lam * dQ[c];
    }
}

template <class T>
FEMB_D void ps_dstress(const PsState<T>& s, const T dg[2][2], T dtau[3]) {
    const T dexx = dg[0][0], deyy = dg[1][1], dexy = (dg[0][1] + dg[1][0]) / T(2);
    const T tr = (dexx + deyy) / T(3);
    const T two_e = T(2) * s.etave;
    const T d[3] = {two_e * (dexx - tr), two_e * (deyy - tr), two_e * dexy};
    if (!(s.lam > T(0))) { for (int c = 0; c < 3; ++c) dtau[c] = d[c]; return; }
    const T* t = s.tt;
    const T dtII = ((T(2) * t[0] + t[1]) * d[0] + (t[0] + T(2) * t[1]) * d[1]) / (T(2) * s.tII) + t[2] * d[2] / s.tII;
    const T dlam = dtII / s.den;
    const T h = T(2) * s.tIIs;
    const T mq[3] = {(T(2) * t[0] + t[1]) / h, (t[0] + T(2) * t[1]) / h, t[2] / s.tIIs};
    const T dm[3] = {(T(2) * d[0] + d[1]) / h - (T(2) * t[0] + t[1]) * dtII / (h * s.tIIs),
                     (d[0] + T(2) * d[1]) / h - (t[0] + T(2) * t[1]) * dtII / (h * s.tIIs),
                     d[2] / s.tIIs - t[2] * dtII / (s.tIIs * s.tIIs)};
    for (int c = 0; c < 3; ++c) dtau[c] = d[c] - two_e * (dlam * mq[c] + s.lam * dm[c]);
}

// Gather of one Q9 element (momentum_element_residual, momentum_residuals.jl:497-528).
template <class T, class TG>
struct Q9El {
    int node[9], dof[3], ph[9], php[3];
    T v[2][9], P[3], P0[3], Tt[3], T0[3], Q[3], Pf[3], gam[3], MP[3];
    bool uniform;
};

template <class T, class TG>
FEMB_D void q9_gather(const H27Args<T, TG>& a, int64_t e, Q9El<T, TG>& el) {
    for (int i = 0; i < 9; ++i) {
        el.node[i] = __ldg(a.el2n + 9 * e + i) - 1;
        el.v[0][i] = ld(a.v[0] + el.node[i]);
        el.v[1][i] = ld(a.v[1] + el.node[i]);
        el.ph[i] = phase_of(a.phv, a.phv_layout, (int64_t)el.node[i] + 1, i, e, 9);
    }
    el.uniform = true;
    for (int i = 1; i < 9; ++i) el.uniform = el.uniform && el.ph[i] == el.ph[0];
    for (int p = 0; p < 3; ++p) {
        el.dof[p] = __ldg(a.dofsP + 3 * e + p) - 1;
        const int d = el.dof[p];
        el.P[p] = ld(a.P + d);
        el.P0[p] = a.P0 ? ld(a.P0 + d) : T(0);
        el.Tt[p] = a.temp ? ld(a.temp + d) : T(0);
        el.T0[p] = a.temp0 ? ld(a.temp0 + d) : T(0);
        el.Q[p] = a.Q ? ld(a.Q + d) : T(0);
        el.Pf[p] = a.Pf ? ld(a.Pf + d) : T(0);
        el.gam[p] = a.gammaP ? ld(a.gammaP + d) : T(0);
        el.MP[p] = a.MP ? ld(a.MP + d) : T(1);
        el.php[p] = phase_of(a.php, a.php_layout, (int64_t)d + 1, p, e, 3);
    }
}

template <class T, class TG>
FEMB_D void q9_dndx(const TG* G, int q, T dn[9][2], T& dO) {
    const TG* g = G + q * 5;
    const T J00 = (T)g[0], J10 = (T)g[1], J01 = (T)g[2], J11 = (T)g[3];
    dO = (T)g[4];
    for (int a = 0; a < 9; ++a) {
        const T r0 = (T)c_tab.dN2[q][a][0], r1 = (T)c_tab.dN2[q][a][1];
        dn[a][0] = r0 * J00 + r1 * J10;
        dn[a][1] = r0 * J01 + r1 * J11;
    }
}

// Pressure residual of one Q9 element (pressure_residual.jl:132-158).
template <class T, class TG>
FEMB_D void q9_pressure(const H27Args<T, TG>& a, int64_t e, const Q9El<T, TG>& el, T RP[3]) {
    for (int p = 0; p < 3; ++p) RP[p] = T(0);
    const TG* G = a.geo_v + e * 9 * 5;
    for (int q = 0; q < 9; ++q) {
        T dn[9][2], dO;
        q9_dndx<T, TG>(G, q, dn, dO);
        const T dOP = (T)ld(a.geo_P + e * 9 + q);
        T ebq = T(0), aq = T(0), dPinc = T(0), dT = T(0), Qq = T(0);
        for (int p = 0; p < 3; ++p) {
            const T N = (T)c_tab.NP2[q][p];
            if (!c_mat.all_bulk_inf) ebq += N * (T)c_mat.bulk[el.php[p]];
            aq += N * (T)c_mat.alpha[el.php[p]];
            dT += N * (el.Tt[p] - el.T0[p]);
            Qq += N * el.Q[p];
            dPinc += a.P_old_ip ? N * el.P[p] : N * (el.P[p] - el.P0[p]);
        }
        if (a.P_old_ip) dPinc -= ld(a.P_old_ip + e * 9 + q);
        const T dPdt = c_mat.all_bulk_inf ? T(0) : dPinc / (ebq * a.dt);
        const T dTdt = aq * dT / a.dt;
        T div = T(0);
        for (int j = 0; j < 2; ++j)
            for (int i = 0; i < 9; ++i) div += dn[i][j] * el.v[j][i];
        const T f = (-div - dPdt + dTdt + Qq) * dOP;
        for (int p = 0; p < 3; ++p) RP[p] += (T)c_tab.NP2[q][p] * f;
    }
}

template <class T, class TG>
__global__ void q9_residual_kernel(H27Args<T, TG> a) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.nels) return;
    Q9El<T, TG> el;
    q9_gather<T, TG>(a, e, el);
    T RP[3];
    q9_pressure<T, TG>(a, e, el, RP);
    T Pn[3];
    for (int p = 0; p < 3; ++p) {
        if (a.write_RP) a.RP[el.dof[p]] = RP[p];
        Pn[p] = !a.with_pnum ? T(0) : (a.Pnum_in ? ld(a.Pnum_in + el.dof[p]) : el.gam[p] * RP[p] / el.MP[p]);
        if (a.with_pnum && a.Pnum_out) a.Pnum_out[el.dof[p]] = Pn[p];
    }
    if (!a.do_momentum && !a.phi) return;
    T R[2][9];
    for (int c = 0; c < 2; ++c) for (int i = 0; i < 9; ++i) R[c][i] = T(0);
    const TG* G = a.geo_v + e * 9 * 5;
    const bool plastic = c_mat.plastic != 0;
    for (int q = 0; q < 9; ++q) {
        T dn[9][2], dO;
        q9_dndx<T, TG>(G, q, dn, dO);
        T g[2][2];
        for (int c = 0; c < 2; ++c)
            for (int k = 0; k < 2; ++k) {
                T s = T(0);
                for (int i = 0; i < 9; ++i) s += dn[i][k] * el.v[c][i];
                g[c][k] = s;
            }
        const T etaq = a.eta_ip ? ld(a.eta_ip + e * 9 + q) : interp<2, T>(q, c_mat.eta, el.ph);
        const T invG = interp<2, T>(q, c_mat.invG, el.ph);
        const T etave = T(1) / (T(1) / etaq + invG / a.dt);
        const T inv2Gdt = invG / (T(2) * a.dt);
        T told[3];
        for (int c = 0; c < 3; ++c) told[c] = a.told[c] ? ld(a.told[c] + e * 9 + q) : T(0);
        T Pq = T(0), Pfq = T(0), Pnq = T(0), Tq = T(0);
        for (int p = 0; p < 3; ++p) {
            const T N = (T)c_tab.NP2[q][p];
            Pq += N * el.P[p]; Pfq += N * el.Pf[p]; Pnq += N * Pn[p]; Tq += N * el.Tt[p];
        }
        const T Peq = a.Pf ? Pq - Pfq : Pq;
        T cphi = 0, sphi = 0, spsi = 0, C = 0, ereg = 0, Kb = 0;
        if (plastic) {
            cphi = interp<2, T>(q, c_mat.cos_phi, el.ph); sphi = interp<2, T>(q, c_mat.sin_phi, el.ph);
            spsi = interp<2, T>(q, c_mat.sin_psi, el.ph); C = interp<2, T>(q, c_mat.C, el.ph);
            ereg = interp<2, T>(q, c_mat.eta_reg, el.ph); Kb = interp<2, T>(q, c_mat.Kb, el.ph);
        }
        PsState<T> st;
        ps_stress<T>(g, etave, inv2Gdt, told, plastic, cphi, sphi, spsi, C, ereg, Kb, a.dt, Peq, st);
        if (a.tau_store[0]) for (int c = 0; c < 3; ++c) a.tau_store[c][e * 9 + q] = st.tau[c];
        if (a.phi) {
            // shear_dissipation plane strain (shear_heating.jl:79-88)
            const T* t = st.tau;
            const T tzz = -(t[0] + t[1]), tzzo = -(told[0] + told[1]);
            const T power = t[0] * g[0][0] + t[1] * g[1][1] + t[2] * (g[0][1] + g[1][0]);
            const T el_ = (t[0] * (t[0] - told[0]) + t[1] * (t[1] - told[1]) + tzz * (tzz - tzzo) +
                           T(2) * t[2] * (t[2] - told[2])) * inv2Gdt;
            a.phi[e * 9 + q] = power - el_;
        }
        const T Ptot = (a.Pf ? Peq + Pfq : Pq) + Pnq;
        const T rhoq = interp<2, T>(q, c_mat.rho0, el.ph) *
                       (T(1) - interp<2, T>(q, c_mat.alpha, el.ph) * (Tq - (T)c_mat.Tref) + interp<2, T>(q, c_mat.beta, el.ph) * Pq);
        const T sg[2][2] = {{st.tau[0] - Ptot, st.tau[2]}, {st.tau[2], st.tau[1] - Ptot}};
        for (int c = 0; c < 2; ++c) {
            const T bg = rhoq * (T)c_mat.g[c];
            for (int i = 0; i < 9; ++i)
                R[c][i] += (dn[i][0] * sg[0][c] + dn[i][1] * sg[1][c] - (T)c_tab.N2[q][i] * bg) * dO;
        }
    }
    if (!a.do_momentum) return;
    for (int c = 0; c < 2; ++c)
        for (int i = 0; i < 9; ++i) atomic_add(a.Rv[c] + el.node[i], R[c][i]);
}

// Q9 augmented Jacobian diagnostics (momentum_residuals.jl:929-1117), exact
// directional derivatives of the plane-strain residual per column.
template <class T, class TG>
__global__ void q9_jacobian_kernel(H27JacArgs<T, TG> a) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.nels) return;
    H27Args<T, TG> ra{};
    ra.el2n = a.el2n; ra.dofsP = a.dofsP; ra.geo_v = a.geo_v; ra.geo_P = a.geo_P;
    ra.v[0] = a.v[0]; ra.v[1] = a.v[1]; ra.P = a.P; ra.P0 = a.P0; ra.temp = a.temp; ra.temp0 = a.temp0;
    ra.Pf = a.Pf; ra.gammaP = a.gammaP; ra.MP = a.MP; ra.phv = a.phv; ra.phv_layout = a.phv_layout;
    ra.php = a.php; ra.php_layout = a.php_layout;
    Q9El<T, TG> el;
    q9_gather<T, TG>(ra, e, el);
    const TG* G = a.geo_v + e * 9 * 5;
    const bool plastic = c_mat.plastic != 0;
    T eta_pc;
    bool scalar = a.eta_ip != nullptr;
    if (scalar) {
        eta_pc = ld(a.eta_ip + e * 9);
        for (int q = 1; q < 9; ++q) eta_pc = fmax(eta_pc, ld(a.eta_ip + e * 9 + q));
    } else {
        eta_pc = (T)c_mat.eta[el.ph[0]];
        for (int i = 1; i < 9; ++i) eta_pc = fmax(eta_pc, (T)c_mat.eta[el.ph[i]]);
    }
    // ∂RP_p/∂v_(b,j) scaled by γ/M_P
    T BPm[3][18];
    for (int p = 0; p < 3; ++p) for (int k = 0; k < 18; ++k) BPm[p][k] = T(0);
    for (int q = 0; q < 9; ++q) {
        T dn[9][2], dO;
        q9_dndx<T, TG>(G, q, dn, dO);
        const T dOP = (T)ld(a.geo_P + e * 9 + q);
        for (int p = 0; p < 3; ++p) {
            const T w = (T)c_tab.NP2[q][p] * dOP;
            for (int b = 0; b < 9; ++b)
                for (int j = 0; j < 2; ++j) BPm[p][b * 2 + j] -= w * dn[b][j];
        }
    }
    for (int p = 0; p < 3; ++p) for (int k = 0; k < 18; ++k) BPm[p][k] = BPm[p][k] * el.gam[p] / el.MP[p];
    T rows[2][9], diag[2][9];
    for (int c = 0; c < 2; ++c) for (int i = 0; i < 9; ++i) { rows[c][i] = T(0); diag[c][i] = T(0); }
    for (int col = 0; col < 18; ++col) {
        const int b = col / 2, j = col % 2;
        T dR[2][9];
        for (int c = 0; c < 2; ++c) for (int i = 0; i < 9; ++i) dR[c][i] = T(0);
        for (int q = 0; q < 9; ++q) {
            T dn[9][2], dO;
            q9_dndx<T, TG>(G, q, dn, dO);
            T g[2][2];
            for (int c = 0; c < 2; ++c)
                for (int k = 0; k < 2; ++k) {
                    T s = T(0);
                    for (int i = 0; i < 9; ++i) s += dn[i][k] * el.v[c][i];
                    g[c][k] = s;
                }
            const T etaq = scalar ? eta_pc : eta_pc * (T)c_tab.sumN2[q];
            const T invG = interp<2, T>(q, c_mat.invG, el.ph);
            const T etave = T(1) / (T(1) / etaq + invG / a.dt);
            const T inv2Gdt = invG / (T(2) * a.dt);
            T told[3];
            for (int c = 0; c < 3; ++c) told[c] = a.told[c] ? ld(a.told[c] + e * 9 + q) : T(0);
            T Pq = T(0), Pfq = T(0);
            for (int p = 0; p < 3; ++p) { Pq += (T)c_tab.NP2[q][p] * el.P[p]; Pfq += (T)c_tab.NP2[q][p] * el.Pf[p]; }
            const T Peq = a.Pf ? Pq - Pfq : Pq;
            T cphi = 0, sphi = 0, spsi = 0, C = 0, ereg = 0, Kb = 0;
            if (plastic) {
                cphi = interp<2, T>(q, c_mat.cos_phi, el.ph); sphi = interp<2, T>(q, c_mat.sin_phi, el.ph);
                spsi = interp<2, T>(q, c_mat.sin_psi, el.ph); C = interp<2, T>(q, c_mat.C, el.ph);
                ereg = interp<2, T>(q, c_mat.eta_reg, el.ph); Kb = interp<2, T>(q, c_mat.Kb, el.ph);
            }
            PsState<T> st;
            ps_stress<T>(g, etave, inv2Gdt, told, plastic, cphi, sphi, spsi, C, ereg, Kb, a.dt, Peq, st);
            T dg[2][2] = {{T(0), T(0)}, {T(0), T(0)}};
            dg[j][0] = dn[b][0]; dg[j][1] = dn[b][1];
            T dtau[3];
            ps_dstress<T>(st, dg, dtau);
            T dPn = T(0);
            for (int p = 0; p < 3; ++p) dPn += (T)c_tab.NP2[q][p] * BPm[p][col];
            const T sg[2][2] = {{dtau[0] - dPn, dtau[2]}, {dtau[2], dtau[1] - dPn}};
            for (int c = 0; c < 2; ++c)
                for (int i = 0; i < 9; ++i) dR[c][i] += (dn[i][0] * sg[0][c] + dn[i][1] * sg[1][c]) * dO;
        }
        for (int c = 0; c < 2; ++c)
            for (int i = 0; i < 9; ++i) {
                rows[c][i] += fabs(dR[c][i]);
                if (c == j && i == b) diag[c][i] = fabs(dR[c][i]);
            }
    }
    for (int c = 0; c < 2; ++c)
        for (int i = 0; i < 9; ++i) {
            atomic_add(a.dRdv[c] + el.node[i], rows[c][i]);
            atomic_add(a.PC[c] + el.node[i], diag[c][i]);
        }
}

// Thermal element residual (heat_diffusion/assembly/residual.jl:58-87) and the
// exact Jacobian row sums / diagonal of its ForwardDiff diagnostics (:30-48).
template <int DIM, class T, class TG>
__global__ void thermal_kernel(ThermalArgs<T, TG> a) {
    using TB = Tabs<DIM>;
    constexpr int NV = TB::NV, NQ = TB::NQ, S = DIM * DIM + 1;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (a.group ? a.ngroup : a.nels)) return;
    const int64_t e = a.group ? (int64_t)__ldg(a.group + t) - 1 : t;
    int node[NV], ph[NV];
    T Tl[NV];
    for (int i = 0; i < NV; ++i) {
        node[i] = __ldg(a.el2n + NV * e + i) - 1;
        Tl[i] = ld(a.Tn + node[i]);
        ph[i] = phase_of(a.ph, a.ph_layout, (int64_t)node[i] + 1, i, e, NV);
    }
    const TG* G = a.geo + e * NQ * S;
    T R[NV];
    for (int i = 0; i < NV; ++i) R[i] = T(0);
    for (int q = 0; q < NQ; ++q) {
        const TG* g = G + q * S;
        const T dO = (T)g[DIM * DIM];
        T Tq = T(0), Pq = T(0), T0q = T(0), sq = T(0), kq = T(0), aq = T(0), bq = T(0), rq = T(0), cq = T(0);
        for (int i = 0; i < NV; ++i) {
            const T N = (T)TB::N(q, i);
            const int n = node[i];
            Tq += N * Tl[i];
            Pq += N * (a.P ? ld(a.P + n) : T(0));
            T0q += N * ld(a.T0 + n);
            sq += N * (a.src ? ld(a.src + n) : T(0));
            kq += N * (T)c_tmat.k[ph[i]];
            aq += N * (T)c_tmat.alpha[ph[i]];
            bq += N * (T)c_tmat.beta[ph[i]];
            rq += N * (T)c_tmat.rho0[ph[i]];
            cq += N * (T)c_tmat.Cp[ph[i]];
        }
        const T rhoq = rq * (T(1) - aq * (Tq - a.Tref) + bq * Pq);
        const T dtrc = a.dt / (rhoq * cq);
        T gT[DIM];
        for (int k = 0; k < DIM; ++k) gT[k] = T(0);
        T dn[NV][DIM];
        for (int i = 0; i < NV; ++i)
            for (int k = 0; k < DIM; ++k) {
                T s = T(0);
                for (int j = 0; j < DIM; ++j) s += (T)TB::dN(q, i, j) * (T)g[j + DIM * k];
                dn[i][k] = s;
                gT[k] += s * Tl[i];
            }
        const T Phi = a.src_ip ? ld(a.src_ip + e * NQ + q) : T(0);
        const T Hq = a.src_ip ? dtrc * Phi : T(0);
        const T rate = T0q - Tq + dtrc * sq + Hq;
        for (int i = 0; i < NV; ++i) {
            T KT = T(0);
            for (int k = 0; k < DIM; ++k) KT += dn[i][k] * gT[k];
            KT = kq * KT;
            R[i] += rate * (T)TB::N(q, i) * dO - dtrc * KT * dO;
        }
    }
    for (int i = 0; i < NV; ++i) {
        if (a.group) a.R[node[i]] += R[i];
        else atomic_add(a.R + node[i], R[i]);
    }
    if (!a.jac) return;
    // Jacobian rows: J[i][b] = Σ_q dΩ [ (−N_b + ∂dtrc_b (s_q + Φ_q)) N_i − ∂dtrc_b KT_i − dtrc k ∇N_i·∇N_b ]
    // with ∂dtrc/∂T_b = dtrc·αq·ρ0q·N_b/ρq (EOS dependence of the density).
    for (int i = 0; i < NV; ++i) {
        T Jrow[NV];
        for (int b = 0; b < NV; ++b) Jrow[b] = T(0);
        for (int q = 0; q < NQ; ++q) {
            const TG* g = G + q * S;
            const T dO = (T)g[DIM * DIM];
            T Tq = T(0), Pq = T(0), sq = T(0), kq = T(0), aq = T(0), bq = T(0), rq = T(0), cq = T(0);
            T gT[DIM];
            for (int k = 0; k < DIM; ++k) gT[k] = T(0);
            for (int m = 0; m < NV; ++m) {
                const T N = (T)TB::N(q, m);
                Tq += N * Tl[m];
                Pq += N * (a.P ? ld(a.P + node[m]) : T(0));
                sq += N * (a.src ? ld(a.src + node[m]) : T(0));
                kq += N * (T)c_tmat.k[ph[m]]; aq += N * (T)c_tmat.alpha[ph[m]]; bq += N * (T)c_tmat.beta[ph[m]];
                rq += N * (T)c_tmat.rho0[ph[m]]; cq += N * (T)c_tmat.Cp[ph[m]];
                for (int k = 0; k < DIM; ++k) {
                    T s = T(0);
                    for (int jj = 0; jj < DIM; ++jj) s += (T)TB::dN(q, m, jj) * (T)g[jj + DIM * k];
                    gT[k] += s * Tl[m];
                }
            }
            const T rhoq = rq * (T(1) - aq * (Tq - a.Tref) + bq * Pq);
            const T dtrc = a.dt / (rhoq * cq);
            const T Ni = (T)TB::N(q, i);
            const T Phi = a.src_ip ? ld(a.src_ip + e * NQ + q) : T(0);
            T dni[DIM];
            for (int k = 0; k < DIM; ++k) {
                dni[k] = T(0);
                for (int jj = 0; jj < DIM; ++jj) dni[k] += (T)TB::dN(q, i, jj) * (T)g[jj + DIM * k];
            }
            T KTi = T(0);
            for (int k = 0; k < DIM; ++k) KTi += dni[k] * gT[k];
            const T cfac = dtrc * aq * rq / rhoq;   // ∂dtrc/∂T_b = cfac·N_b
            for (int b = 0; b < NV; ++b) {
                const T Nb = (T)TB::N(q, b);
                const T ddt = cfac * Nb;
                T KK = T(0);
                for (int k = 0; k < DIM; ++k) {
                    T dnb = T(0);
                    for (int jj = 0; jj < DIM; ++jj) dnb += (T)TB::dN(q, b, jj) * (T)g[jj + DIM * k];
                    KK += dni[k] * dnb;
                }
                Jrow[b] += ((-Nb + ddt * (sq + Phi)) * Ni - ddt * kq * KTi - dtrc * kq * KK) * dO;
            }
        }
        T row = T(0);
        for (int b = 0; b < NV; ++b) row += fabs(Jrow[b]);
        if (a.group) {
            a.dRdT[node[i]] += row;
            a.PC[node[i]] += fabs(Jrow[i]);
        } else {
            atomic_add(a.dRdT + node[i], row);
            atomic_add(a.PC + node[i], fabs(Jrow[i]));
        }
    }
}

// Lithostatic-pressure element residual (lp_integrate_residual,
// src/lithostatic_pressure/assembly/residual.jl:48-63): R_i = Σ_q (ρ_q ∇N_i·g − ∇N_i·∇P) dΩ
// with ρ_q = ρ0_q (1 − α_q (T_q − Tref) + β_q P_q), and the row sums and diagonal of its
// Jacobian (the ForwardDiff diagnostics of lp_element_jacobian, :22-36), in closed form:
// ∂R_i/∂P_b = Σ_q (ρ0_q β_q N_b ∇N_i·g − ∇N_i·∇N_b) dΩ.
template <int DIM>
__global__ void lithostatic_kernel(LithoArgs a) {
    using TB = Tabs<DIM>;
    constexpr int NV = TB::NV, NQ = TB::NQ, S = DIM * DIM + 1;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.nels) return;
    int node[NV], ph[NV];
    double Pl[NV], Tl[NV];
    for (int i = 0; i < NV; ++i) {
        node[i] = __ldg(a.el2n + NV * e + i) - 1;
        Pl[i] = a.P[node[i]];
        Tl[i] = a.Tn ? __ldg(a.Tn + node[i]) : 0.0;
        ph[i] = phase_of(a.ph, a.ph_layout, (int64_t)node[i] + 1, i, e, NV);
    }
    const double* G = a.geo + e * NQ * S;
    double R[NV];
    for (int i = 0; i < NV; ++i) R[i] = 0.0;
    for (int q = 0; q < NQ; ++q) {
        const double* g = G + q * S;
        const double dO = g[DIM * DIM];
        double Tq = 0, Pq = 0, aq = 0, bq = 0, rq = 0;
        for (int i = 0; i < NV; ++i) {
            const double N = TB::N(q, i);
            Tq += N * Tl[i]; Pq += N * Pl[i];
            aq += N * a.alpha[ph[i]]; bq += N * a.beta[ph[i]]; rq += N * a.rho0[ph[i]];
        }
        const double rho = rq * (1.0 - aq * (Tq - a.Tref) + bq * Pq);
        double dn[NV][DIM], gP[DIM];
        for (int k = 0; k < DIM; ++k) gP[k] = 0.0;
        for (int i = 0; i < NV; ++i)
            for (int k = 0; k < DIM; ++k) {
                double s = 0;
                for (int j = 0; j < DIM; ++j) s += TB::dN(q, i, j) * g[j + DIM * k];
                dn[i][k] = s;
                gP[k] += s * Pl[i];
            }
        for (int i = 0; i < NV; ++i) {
            double ng = 0, np = 0;
            for (int k = 0; k < DIM; ++k) { ng += dn[i][k] * a.g[k]; np += dn[i][k] * gP[k]; }
            R[i] += (rho * ng - np) * dO;
        }
    }
    for (int i = 0; i < NV; ++i) atomicAdd(a.R + node[i], R[i]);
    if (!a.jac) return;
    for (int i = 0; i < NV; ++i) {
        double Jrow[NV];
        for (int b = 0; b < NV; ++b) Jrow[b] = 0.0;
        for (int q = 0; q < NQ; ++q) {
            const double* g = G + q * S;
            const double dO = g[DIM * DIM];
            double bq = 0, rq = 0;
            for (int m = 0; m < NV; ++m) {
                const double N = TB::N(q, m);
                bq += N * a.beta[ph[m]]; rq += N * a.rho0[ph[m]];
            }
            double dni[DIM], ng = 0;
            for (int k = 0; k < DIM; ++k) {
                double s = 0;
                for (int j = 0; j < DIM; ++j) s += TB::dN(q, i, j) * g[j + DIM * k];
                dni[k] = s;
                ng += s * a.g[k];
            }
            const double cf = rq * bq * ng;
            for (int b = 0; b < NV; ++b) {
                double kk = 0;
                for (int k = 0; k < DIM; ++k) {
                    double s = 0;
                    for (int j = 0; j < DIM; ++j) s += TB::dN(q, b, j) * g[j + DIM * k];
                    kk += dni[k] * s;
                }
                Jrow[b] += (cf * TB::N(q, b) - kk) * dO;
            }
        }
        double row = 0;
        for (int b = 0; b < NV; ++b) row += fabs(Jrow[b]);
        atomicAdd(a.dRdP + node[i], row);
        atomicAdd(a.PC + node[i], fabs(Jrow[i]));
    }
}

inline unsigned nb(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

cudaError_t launch_lithostatic(const LithoArgs& a, cudaStream_t st) {
    if (a.nels <= 0) return cudaSuccess;
    count_launch();
    if (a.dim == 3) lithostatic_kernel<3><<<nb(a.nels, 64), 64, 0, st>>>(a);
    else lithostatic_kernel<2><<<nb(a.nels, 128), 128, 0, st>>>(a);
    return cudaGetLastError();
}

template <class T, class TG>
cudaError_t launch_pressure_scaling(int dim, const int32_t* el2n, const int32_t* dofsP, const TG* geo_P,
                                    const int32_t* phv, int phv_layout, const T* eta_ip, int use_eta_ip, T* MP, T* gP,
                                    int64_t nels, int64_t nnodesP, T gfact, T dt, cudaStream_t st) {
    count_launch();
    if (dim == 3)
        pressure_scaling_kernel<3, T, TG><<<nb(nels, 128), 128, 0, st>>>(el2n, dofsP, geo_P, phv, phv_layout, eta_ip,
                                                                         use_eta_ip, MP, gP, nels, gfact, dt);
    else
        pressure_scaling_kernel<2, T, TG><<<nb(nels, 128), 128, 0, st>>>(el2n, dofsP, geo_P, phv, phv_layout, eta_ip,
                                                                         use_eta_ip, MP, gP, nels, gfact, dt);
    count_launch();
    scaling_finalize_kernel<T><<<nb(nnodesP, 256), 256, 0, st>>>(gP, MP, nnodesP);
    return cudaGetLastError();
}

template <class T, class TG>
cudaError_t launch_q9_residual(const H27Args<T, TG>& args, cudaStream_t st) {
    count_launch();
    q9_residual_kernel<T, TG><<<nb(args.nels, 128), 128, 0, st>>>(args);
    return cudaGetLastError();
}

template <class T, class TG>
cudaError_t launch_q9_jacobian(const H27JacArgs<T, TG>& args, cudaStream_t st) {
    count_launch();
    q9_jacobian_kernel<T, TG><<<nb(args.nels, 64), 64, 0, st>>>(args);
    return cudaGetLastError();
}

template <class T, class TG>
cudaError_t launch_thermal(const ThermalArgs<T, TG>& a, int num_sms, cudaStream_t st) {
    (void)num_sms;
    const int64_t n = a.group ? a.ngroup : a.nels;
    if (n <= 0) return cudaSuccess;
    count_launch();
    if (a.dim == 3) thermal_kernel<3, T, TG><<<nb(n, 64), 64, 0, st>>>(a);
    else thermal_kernel<2, T, TG><<<nb(n, 128), 128, 0, st>>>(a);
    return cudaGetLastError();
}

#define FEMB_INST2(T, TG)                                                                                            \
    template cudaError_t launch_pressure_scaling<T, TG>(int, const int32_t*, const int32_t*, const TG*,             \
                                                        const int32_t*, int, const T*, int, T*, T*, int64_t,       \
                                                        int64_t, T, T, cudaStream_t);                              \
    template cudaError_t launch_q9_residual<T, TG>(const H27Args<T, TG>&, cudaStream_t);                            \
    template cudaError_t launch_q9_jacobian<T, TG>(const H27JacArgs<T, TG>&, cudaStream_t);                         \
    template cudaError_t launch_thermal<T, TG>(const ThermalArgs<T, TG>&, int, cudaStream_t);
FEMB_INST2(double, double)
FEMB_INST2(float, float)
FEMB_INST2(double, float)
FEMB_INST2(float, double)
#undef FEMB_INST2

}  // namespace femb
