// adjoint3d.cu — the hand-written adjoint (reverse-mode) residual of the Hex27/P1-disc
// Stokes element, for the frozen-operator adjoint solve.
//
// At a forward state u = (v, P) the DR loop drives the augmented residual
//   Rv(v, P, Pnum(v, P)),  RP(v, P),   Pnum = Γ·RP,  Γ = γP/M_P (element-local)
// to zero (DR.jl:674-676). Its transposed Jacobian applied to λ = (λv, λP) is
//   dv = (∂Rv/∂v)ᵀλv + (∂RP/∂v)ᵀμ,    dP = (∂Rv/∂P)ᵀλv + (∂RP/∂P)ᵀμ,
//   μ  = λP + Γ·(∂Rv/∂Pnum)ᵀλv,
// the operator the reference assembles as element blocks A, B, C, D, W
// (FrozenAdjointOperator, src/stokes/assemblers/adjoint_operator.jl:3-73, applied
// at :640-660; its Enzyme form in solvers/DR_adjoint.jl:156-205). Here it is applied
// matrix-free: per element the λ gradient and the forward state's trial stress are
// formed at the 27 points with the sum-factorised stages of hex27.cuh, the
// cotangent of the stress is pulled back through the Drucker–Prager radial return
// (rheology.jl:441-472) and the Maxwell trial stress (:413-439) by hand, and the
// result goes out through the transposed contraction. No element blocks are
// stored, so the memory is that of the forward sweep.
//
// The same pass optionally writes λ·∂R/∂η_q, the sensitivity to the viscosity of
// every integration point (for gradients with respect to a viscosity field), by
// one forward-mode derivative of the point stress in η.
#include "kernels.cuh"
#include "hex27.cuh"

namespace femb {

namespace {

// One forward-mode partial (the viscosity direction of the sensitivity).
template <class T>
struct D1 {
    T v, d;
};
template <class T> FEMB_D D1<T> operator+(D1<T> a, D1<T> b) { return {a.v + b.v, a.d + b.d}; }
template <class T> FEMB_D D1<T> operator-(D1<T> a, D1<T> b) { return {a.v - b.v, a.d - b.d}; }
template <class T> FEMB_D D1<T> operator*(D1<T> a, D1<T> b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
template <class T> FEMB_D D1<T> operator/(D1<T> a, D1<T> b) { return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
template <class T> FEMB_D D1<T> cst(T x) { return {x, T(0)}; }
template <class T> FEMB_D D1<T> dsqrt(D1<T> a) {
    const T r = sqrt(a.v);
    return {r, a.d / (T(2) * r)};
}

// Point stress with the Drucker–Prager return (rheology.jl:413-472) as a function
// of the viscosity: τ and ∂τ/∂η.
template <class T>
FEMB_D void stress_eta(const T ed[6], const T told[6], T eta, T invG, T dt, bool plastic, T cC, T sphi, T rest,
                       T Peq, T EPS2, D1<T> tau[6]) {
    const D1<T> et = {eta, T(1)};
    const D1<T> etave = cst(T(1)) / (cst(T(1)) / et + cst(invG / dt));
    const T inv2Gdt = invG / (T(2) * dt);
    for (int c = 0; c < 6; ++c) tau[c] = cst(T(2)) * etave * cst(ed[c] + told[c] * inv2Gdt);
    if (!plastic) return;
    const D1<T> J = cst(T(0.5)) * (tau[0] * tau[0] + tau[1] * tau[1] + tau[2] * tau[2]) + tau[3] * tau[3] +
                    tau[4] * tau[4] + tau[5] * tau[5] + cst(EPS2);
    const D1<T> tII = dsqrt(J);
    const D1<T> tIIs = tII + cst(EPS2);
    const D1<T> F = tII - cst(cC) - cst(sphi * Peq);
    if (!(F.v > T(0))) return;
    const D1<T> lam = F / (etave + cst(rest));
    const D1<T> f = cst(T(2)) * etave * lam / tIIs;
    for (int c = 0; c < 3; ++c) tau[c] = tau[c] - cst(T(0.5)) * f * tau[c];
    for (int c = 3; c < 6; ++c) tau[c] = tau[c] - f * tau[c];
}

}  // namespace

template <class T>
__global__ void __launch_bounds__(H27_THREADS) hex27_adjoint_kernel(AdjArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const bool lane_ok = lane < 27;
    // lanes 27..31 carry no element; they work in a private scratch slot (3)
    using LY = H27Layout<T>;   // stage layout (bank-conflict-free in FP64)
    const int s = lane_ok ? lane / 9 : 3, m = lane_ok ? lane % 9 : LY::IDLE_M, m1 = m % 3, m2 = m / 3;
    T* E = reinterpret_cast<T*>(smem_raw) + ((size_t)warp * 4 + s) * LY::SLOT;
    int* PH = reinterpret_cast<int*>(reinterpret_cast<T*>(smem_raw) + (size_t)wpb * 4 * LY::SLOT) + (warp * 4 + s) * 28;

    Tab1D<T> tb; tb.load();
    const T dt = a.dt;
    const T gvec[3] = {(T)c_mat.g[0], (T)c_mat.g[1], (T)c_mat.g[2]};
    const T zero3[3] = {T(0), T(0), T(0)};
    const bool plastic = c_mat.plastic != 0;
    const bool bulk_inf = c_mat.all_bulk_inf != 0;
    const T EPS2 = eps2<T>();

    const int64_t stride = (int64_t)gridDim.x * wpb * 3;
    for (int64_t base = ((int64_t)blockIdx.x * wpb + warp) * 3; base < a.nels; base += stride) {
        const int64_t e = base + (lane_ok ? s : 0);
        const bool act = lane_ok && e < a.nels;
        const int64_t ec = act ? e : 0;

        // ---- gather λv and the forward v on the owned x-line ----
        int node[3];
        T lv[3][3], vv[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            node[i] = act ? __ldg(a.el2n + 27 * ec + c_tab.tn3[tidx(i, m1, m2)]) - 1 : 0;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                lv[c][i] = act ? ld(a.lam_v[c] + node[i]) : T(0);
                vv[c][i] = act ? ld(a.v[c] + node[i]) : T(0);
            }
        }
        int p0 = 0;
        bool uniform = true;
        if (a.phv_layout == FEMB200_PHASE_CELL || !a.phv) {
            p0 = a.phv ? (act ? __ldg(a.phv + ec) - 1 : 0) : 0;
        } else {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int li = c_tab.tn3[tidx(i, m1, m2)];
                PH[tidx(i, m1, m2)] = act ? phase_of(a.phv, a.phv_layout, (int64_t)node[i] + 1, li, ec, 27) : 0;
            }
            __syncwarp();
            p0 = PH[0];
            bool same = PH[tidx(0, m1, m2)] == p0 && PH[tidx(1, m1, m2)] == p0 && PH[tidx(2, m1, m2)] == p0;
            const unsigned bal = __ballot_sync(0xffffffffu, same || !lane_ok);
            uniform = ((bal >> (s * 9)) & 0x1ffu) == 0x1ffu;
        }
        int dof[4], php[4];
        T Pl[4], Pfl[4], Gam[4], lP[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            dof[p] = act ? __ldg(a.dofsP + 4 * ec + p) - 1 : 0;
            Pl[p] = act ? ld(a.P + dof[p]) : T(0);
            Pfl[p] = (act && a.Pf) ? ld(a.Pf + dof[p]) : T(0);
            Gam[p] = (act && a.with_pnum && a.gammaP) ? ld(a.gammaP + dof[p]) / (a.MP ? ld(a.MP + dof[p]) : T(1)) : T(0);
            lP[p] = act ? ld(a.lam_P + dof[p]) : T(0);
            php[p] = act ? phase_of(a.php, a.php_layout, (int64_t)dof[p] + 1, p, ec, 4) : 0;
        }

        // ---- reference gradients (and the λ value) at the owned points ----
        T gl[3][3][3], gv[3][3][3], lval[3][3];
        h27_gradient<T, LY>(tb, lv, E, m1, m2, gl);
        {
            const T* E1 = E + 6 * LY::K1;   // stage-Y output: the ξη-interpolated λ is the third block
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    T acc = T(0);
#pragma unroll
                    for (int k = 0; k < 3; ++k) acc += tb.B[q][k] * E1[(c * 3 + 2) * LY::K2 + LY::l2(m1, m2, k)];
                    lval[c][q] = acc;
                }
        }
        __syncwarp();
        h27_gradient<T, LY>(tb, vv, E, m1, m2, gv);

        // ---- s = (∂Rv/∂Pnum)ᵀλv = −∫ N^P ∇·λv over the owned points ----
        T NPq[3][4];
        T sp[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
        for (int qz = 0; qz < 3; ++qz) {
            const int q = tidx(m1, m2, qz);
            const T* G = a.geo_v + ((int64_t)ec * 27 + q) * 10;
            T Ji[9];
#pragma unroll
            for (int r = 0; r < 9; ++r) Ji[r] = act ? (T)ld(G + r) : T(0);
            const T dO = act ? (T)ld(G + 9) : T(0);
            const T xi = (T)c_tab.qx[m1], et = (T)c_tab.qx[m2], ze = (T)c_tab.qx[qz];
            NPq[qz][0] = T(1) - xi - et - ze; NPq[qz][1] = xi; NPq[qz][2] = et; NPq[qz][3] = ze;
            T divl = T(0);
#pragma unroll
            for (int c = 0; c < 3; ++c) divl += gl[c][0][qz] * Ji[3 * c] + gl[c][1][qz] * Ji[1 + 3 * c] + gl[c][2][qz] * Ji[2 + 3 * c];
#pragma unroll
            for (int p = 0; p < 4; ++p) sp[p] -= NPq[qz][p] * divl * dO;
        }
        T* RPs = E + 6 * LY::K1 + 9 * LY::K2;   // after the gradient's stages
        static_assert(6 * LY::K1 + 9 * LY::K2 + 36 <= LY::SLOT, "mode reduction scratch");
#pragma unroll
        for (int p = 0; p < 4; ++p) RPs[m * 4 + p] = sp[p];
        __syncwarp();
        T mu[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            T acc = T(0);
#pragma unroll
            for (int t = 0; t < 9; ++t) acc += RPs[t * 4 + p];
            mu[p] = lP[p] + Gam[p] * acc;
        }
        __syncwarp();

        // ---- pointwise pull-back of the stress cotangent ----
        T Fb[3][3][3];
        T dPp[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
        for (int qz = 0; qz < 3; ++qz) {
            const int q = tidx(m1, m2, qz);
            const T* Gp = a.geo_v + ((int64_t)ec * 27 + q) * 10;
            T J[9];
#pragma unroll
            for (int r = 0; r < 9; ++r) J[r] = act ? (T)ld(Gp + r) : T(0);
            const T dO = act ? (T)ld(Gp + 9) : T(0);
            const T dOP = act ? (T)ld(a.geo_P + (int64_t)ec * 27 + q) : T(0);
            // physical gradients of the forward velocity and of λv
            T gq[3][3], G[3][3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    gq[c][k] = gv[c][0][qz] * J[3 * k] + gv[c][1][qz] * J[1 + 3 * k] + gv[c][2][qz] * J[2 + 3 * k];
                    G[c][k] = gl[c][0][qz] * J[3 * k] + gl[c][1][qz] * J[1 + 3 * k] + gl[c][2][qz] * J[2 + 3 * k];
                }
            T etaov;
            const T* eov = nullptr;
            if (a.eta_ip) { etaov = act ? ld(a.eta_ip + ec * 27 + q) : T(1); eov = &etaov; }
            QpMat<T> mt;
            interp_material(mt, uniform, p0, PH, m1, m2, qz, plastic, eov);
            if (!act) mt.eta = T(1);
            T Pq = T(0), Pfq = T(0), muq = T(0);
#pragma unroll
            for (int p = 0; p < 4; ++p) { Pq += NPq[qz][p] * Pl[p]; Pfq += NPq[qz][p] * Pfl[p]; muq += NPq[qz][p] * mu[p]; }
            const T Peq = a.Pf ? Pq - Pfq : Pq;
            const T etave = T(1) / (T(1) / mt.eta + mt.invG / dt);
            const T twoe = T(2) * etave;
            const T inv2Gdt = mt.invG / (T(2) * dt);
            T told[6];
#pragma unroll
            for (int c = 0; c < 6; ++c) told[c] = (act && a.told[c]) ? ld(a.told[c] + ec * 27 + q) : T(0);
            const T tr = (gq[0][0] + gq[1][1] + gq[2][2]) / T(3);
            const T ed[6] = {gq[0][0] - tr, gq[1][1] - tr, gq[2][2] - tr, (gq[0][1] + gq[1][0]) / T(2),
                             (gq[0][2] + gq[2][0]) / T(2), (gq[1][2] + gq[2][1]) / T(2)};
            T ttr[6];
#pragma unroll
            for (int c = 0; c < 6; ++c) ttr[c] = twoe * (ed[c] + told[c] * inv2Gdt);
            // cotangent of τ from λ's gradient: Gλ:σ = Σ ḡ_i τ_i
            const T gb[6] = {G[0][0], G[1][1], G[2][2], G[0][1] + G[1][0], G[0][2] + G[2][0], G[1][2] + G[2][1]};
            T tbar[6];
            T Pbar_eq = T(0);
            const T cC = mt.cphi * mt.C;
            const T rest = mt.ereg + mt.Kb * dt * (-mt.spsi) * (-mt.sphi);
            bool yielded = false;
            if (plastic) {
                const T tII = sqrt((ttr[0] * ttr[0] + ttr[1] * ttr[1] + ttr[2] * ttr[2]) / T(2) + ttr[3] * ttr[3] +
                                   ttr[4] * ttr[4] + ttr[5] * ttr[5] + EPS2);
                const T tIIs = tII + EPS2;
                const T Fy = tII - cC - mt.sphi * Peq;
                if (Fy > T(0)) {
                    // τ_i = τtr_i (1 − f m_i / tIIs), f = 2ηve·F/den, m = (½,½,½,1,1,1)
                    yielded = true;
                    const T den = etave + rest;
                    const T f = twoe * (Fy / den);
                    const T mm[6] = {T(0.5), T(0.5), T(0.5), T(1), T(1), T(1)};
                    T A = T(0);
#pragma unroll
                    for (int i = 0; i < 6; ++i) A += gb[i] * mm[i] * ttr[i];
                    // ∂(f/tIIs)/∂tII = (2ηve/den)(ε² + C cosϕ + sinϕ Peq)/tIIs²
                    const T dftII = (twoe / den) * (EPS2 + cC + mt.sphi * Peq) / (tIIs * tIIs);
#pragma unroll
                    for (int i = 0; i < 6; ++i) tbar[i] = gb[i] * (T(1) - f * mm[i] / tIIs) - A * dftII * mm[i] * ttr[i] / tII;
                    Pbar_eq = A * twoe * mt.sphi / (den * tIIs);
                }
            }
            if (!yielded) {
#pragma unroll
                for (int i = 0; i < 6; ++i) tbar[i] = gb[i];
            }
            // through the Maxwell trial stress and the deviatoric strain rate
            T eb[6];
#pragma unroll
            for (int i = 0; i < 6; ++i) eb[i] = twoe * tbar[i];
            const T str = (eb[0] + eb[1] + eb[2]) / T(3);
            const T Gb[3][3] = {{eb[0] - str, eb[3] / T(2), eb[4] / T(2)},
                                {eb[3] / T(2), eb[1] - str, eb[5] / T(2)},
                                {eb[4] / T(2), eb[5] / T(2), eb[2] - str}};
            // reference-frame fluxes, with (∂RP/∂v)ᵀμ as a pressure-like term −μ·I
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    Fb[c][d][qz] = act ? dO * (J[d] * Gb[c][0] + J[d + 3] * Gb[c][1] + J[d + 6] * Gb[c][2]) -
                                             dOP * muq * J[d + 3 * c]
                                       : T(0);
            // pressure cotangent: −∇·λv (σ ∋ −P·I), the yield function's pressure, the
            // EOS density ρ0·β·P in the body force, and (∂RP/∂P)ᵀμ (storage)
            const T divl = G[0][0] + G[1][1] + G[2][2];
            T pb = dO * (Pbar_eq - divl);
            const T gl_dot = gvec[0] * lval[0][qz] + gvec[1] * lval[1][qz] + gvec[2] * lval[2][qz];
            pb -= dO * mt.rho0 * mt.beta * gl_dot;
            if (!bulk_inf) {
                T ebq = T(0);
#pragma unroll
                for (int p = 0; p < 4; ++p) ebq += NPq[qz][p] * (T)c_mat.bulk[php[p]];
                pb -= dOP * muq / (ebq * dt);
            }
            if (!act) pb = T(0);
#pragma unroll
            for (int p = 0; p < 4; ++p) dPp[p] += NPq[qz][p] * pb;
            // sensitivity to the viscosity of this point: dΩ·Σ ḡ_i ∂τ_i/∂η
            if (a.out_eta && act) {
                D1<T> td[6];
                stress_eta<T>(ed, told, mt.eta, mt.invG, dt, plastic, cC, mt.sphi, rest, Peq, EPS2, td);
                T sens = T(0);
#pragma unroll
                for (int i = 0; i < 6; ++i) sens += gb[i] * td[i].d;
                a.out_eta[ec * 27 + q] = dO * sens;
            }
        }
        // ---- pressure cotangent: element sum over the 27 points ----
#pragma unroll
        for (int p = 0; p < 4; ++p) RPs[m * 4 + p] = dPp[p];
        __syncwarp();
        if (act && m < 4) {
            T acc = T(0);
#pragma unroll
            for (int t = 0; t < 9; ++t) acc += RPs[t * 4 + m];
            if (a.out_dP) a.out_dP[dof[m]] = acc;
        }
        __syncwarp();
        if (!a.out_dv[0]) continue;
        T R[3][3];
        h27_transpose<T, true, LY>(tb, Fb, zero3, gvec, E, m1, m2, R);
        if (act) {
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int i = 0; i < 3; ++i) atomic_add(a.out_dv[c] + node[i], R[c][i]);
        }
    }
}

template <class T>
cudaError_t launch_hex27_adjoint(const AdjArgs<T>& args, int num_sms, cudaStream_t st) {
    const int wpb = H27_THREADS / 32;
    const size_t smem = (size_t)wpb * 4 * H27Layout<T>::SLOT * sizeof(T) + (size_t)wpb * 4 * 28 * sizeof(int);
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(hex27_adjoint_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    const int64_t groups = (args.nels + 2) / 3;
    int64_t blocks = (groups + wpb - 1) / wpb;
    const int64_t cap = (int64_t)num_sms * 16;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    count_launch();
    hex27_adjoint_kernel<T><<<(unsigned)blocks, H27_THREADS, smem, st>>>(args);
    return cudaGetLastError();
}

template cudaError_t launch_hex27_adjoint<double>(const AdjArgs<double>&, int, cudaStream_t);

}  // namespace femb
