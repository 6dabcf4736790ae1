// stokes3d.cu — Hex27/P1-disc Stokes element sweeps for sm_100a.
//
// One kernel evaluates, per element and in one pass over the element's data:
//   the pressure residual  RP  (integrate_PH_pressure_residual,
//                               src/stokes/assemblers/pressure_residual.jl:132-158),
//   Pnum = γP·RP/M_P       (element-local, src/stokes/solvers/DR.jl:674),
//   the momentum residual  Rv  with the visco-elasto-plastic stress
//                               (momentum_residuals.jl:209-258, rheology.jl:413-472),
// optionally storing the integration-point stress (update_stokes_current_stress!,
// DR.jl:820) or the shear dissipation (shear_heating.jl:47-103) instead.
// The nodal residual is scattered with FP64/FP32 atomics into a zeroed Rv.
#include "kernels.cuh"
#include "hex27.cuh"

namespace femb {

template <class T, class TG>
__global__ void __launch_bounds__(H27_THREADS) hex27_residual_kernel(H27Args<T, TG> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const bool lane_ok = lane < 27;
    // lanes 27..31 carry no element; they work in a private scratch slot (3) so
    // their (discarded) stage writes never touch an element's shared memory.
    using LY = H27Layout<T>;   // stage layout (bank-conflict-free in FP64)
    const int s = lane_ok ? lane / 9 : 3, m = lane_ok ? lane % 9 : LY::IDLE_M, m1 = m % 3, m2 = m / 3;
    T* E = reinterpret_cast<T*>(smem_raw) + ((size_t)warp * 4 + s) * LY::SLOT;
    int* PH = reinterpret_cast<int*>(reinterpret_cast<T*>(smem_raw) + (size_t)wpb * 4 * LY::SLOT) + (warp * 4 + s) * 28;

    Tab1D<T> tb; tb.load();
    const T dt = a.dt;
    const T gvec[3] = {(T)c_mat.g[0], (T)c_mat.g[1], (T)c_mat.g[2]};
    const bool plastic = c_mat.plastic != 0;
    const T EPS2 = eps2<T>();

    const int64_t stride = (int64_t)gridDim.x * wpb * 3;
    for (int64_t base = ((int64_t)blockIdx.x * wpb + warp) * 3; base < a.nels; base += stride) {
        const int64_t e = base + (lane_ok ? s : 0);
        const bool act = lane_ok && e < a.nels;
        const int64_t ec = act ? e : 0;   // clamped element for address formation

        // ---- gather: x-line nodes (·, m1, m2) of v ----
        int node[3];
        T v[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            node[i] = act ? __ldg(a.el2n + 27 * ec + c_tab.tn3[tidx(i, m1, m2)]) - 1 : 0;
#pragma unroll
            for (int c = 0; c < 3; ++c) v[c][i] = act ? ld(a.v[c] + node[i]) : T(0);
        }
        // element phases
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

        // ---- element pressure data (element-private DoFs) ----
        int dof[4];
        T Pl[4], P0l[4], Tl[4], T0l[4], Ql[4], Pfl[4], gam[4], MPl[4];
        int php[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            dof[p] = act ? __ldg(a.dofsP + 4 * ec + p) - 1 : 0;
            Pl[p] = act ? ld(a.P + dof[p]) : T(0);
            P0l[p] = (act && a.P0) ? ld(a.P0 + dof[p]) : T(0);
            Tl[p] = (act && a.temp) ? ld(a.temp + dof[p]) : T(0);
            T0l[p] = (act && a.temp0) ? ld(a.temp0 + dof[p]) : T(0);
            Ql[p] = (act && a.Q) ? ld(a.Q + dof[p]) : T(0);
            Pfl[p] = (act && a.Pf) ? ld(a.Pf + dof[p]) : T(0);
            gam[p] = (act && a.gammaP) ? ld(a.gammaP + dof[p]) : T(0);
            MPl[p] = (act && a.MP) ? ld(a.MP + dof[p]) : T(1);
            php[p] = act ? phase_of(a.php, a.php_layout, (int64_t)dof[p] + 1, p, ec, 4) : 0;
        }

        // ---- reference gradients at the owned quadrature points ----
        T g[3][3][3];
        h27_gradient<T, LY>(tb, v, E, m1, m2, g);

        // physical gradients and geometry at the three owned points
        T gp[3][3][3];   // gp[qz][c][k] = ∂v_c/∂x_k
        T dO[3], dOP[3];
#pragma unroll
        for (int qz = 0; qz < 3; ++qz) {
            const int q = tidx(m1, m2, qz);
            const TG* G = a.geo_v + ((int64_t)ec * 27 + q) * 10;
            T Ji[9];
#pragma unroll
            for (int r = 0; r < 9; ++r) Ji[r] = act ? (T)ld(G + r) : T(0);
            dO[qz] = act ? (T)ld(G + 9) : T(0);
            dOP[qz] = act ? (T)ld(a.geo_P + (int64_t)ec * 27 + q) : T(0);
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    gp[qz][c][k] = g[c][0][qz] * Ji[0 + 3 * k] + g[c][1][qz] * Ji[1 + 3 * k] + g[c][2][qz] * Ji[2 + 3 * k];
        }

        // ---- pressure residual (element-local reduction over the 27 points) ----
        T NPq[3][4];
        T rp[4] = {T(0), T(0), T(0), T(0)};
        const bool bulk_inf = c_mat.all_bulk_inf != 0;
#pragma unroll
        for (int qz = 0; qz < 3; ++qz) {
            const T xi = (T)c_tab.qx[m1], et = (T)c_tab.qx[m2], ze = (T)c_tab.qx[qz];
            NPq[qz][0] = T(1) - xi - et - ze; NPq[qz][1] = xi; NPq[qz][2] = et; NPq[qz][3] = ze;
            T ebq = T(0), aq = T(0);
            if (!bulk_inf) for (int p = 0; p < 4; ++p) ebq += NPq[qz][p] * (T)c_mat.bulk[php[p]];
            for (int p = 0; p < 4; ++p) aq += NPq[qz][p] * (T)c_mat.alpha[php[p]];
            T dPinc = T(0);
            if (a.P_old_ip) {
                for (int p = 0; p < 4; ++p) dPinc += NPq[qz][p] * Pl[p];
                dPinc -= act ? ld(a.P_old_ip + ec * 27 + tidx(m1, m2, qz)) : T(0);
            } else {
                for (int p = 0; p < 4; ++p) dPinc += NPq[qz][p] * (Pl[p] - P0l[p]);
            }
            const T dPdt = bulk_inf ? T(0) : dPinc / (ebq * dt);
            T dT = T(0), Qq = T(0);
            for (int p = 0; p < 4; ++p) { dT += NPq[qz][p] * (Tl[p] - T0l[p]); Qq += NPq[qz][p] * Ql[p]; }
            const T dTdt = aq * dT / dt;
            const T div = gp[qz][0][0] + gp[qz][1][1] + gp[qz][2][2];
            const T f = (-div - dPdt + dTdt + Qq) * dOP[qz];
#pragma unroll
            for (int p = 0; p < 4; ++p) rp[p] += NPq[qz][p] * f;
        }
        T* RPs = E + 6 * LY::K1 + 9 * LY::K2;   // after the gradient's stages
        static_assert(6 * LY::K1 + 9 * LY::K2 + 36 <= LY::SLOT, "mode reduction scratch");
#pragma unroll
        for (int p = 0; p < 4; ++p) RPs[m * 4 + p] = rp[p];
        __syncwarp();
        T RPe[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            T acc = T(0);
#pragma unroll
            for (int t = 0; t < 9; ++t) acc += RPs[t * 4 + p];
            RPe[p] = acc;
        }
        __syncwarp();
        if (act && a.write_RP && m < 4) a.RP[dof[m]] = RPe[m];
        T Pn[4];
#pragma unroll
        for (int p = 0; p < 4; ++p)
            Pn[p] = !a.with_pnum ? T(0) : (a.Pnum_in ? (act ? ld(a.Pnum_in + dof[p]) : T(0)) : gam[p] * RPe[p] / MPl[p]);
        if (act && a.Pnum_out && a.with_pnum && m < 4) a.Pnum_out[dof[m]] = Pn[m];

        if (!a.do_momentum && !a.phi) continue;

        // ---- stress and fluxes at the owned points ----
        T F[3][3][3];   // F[c][d][qz]
        T beta_q[3];
#pragma unroll
        for (int qz = 0; qz < 3; ++qz) {
            const int q = tidx(m1, m2, qz);
            const TG* G = a.geo_v + ((int64_t)ec * 27 + q) * 10;
            T Ji[9];
#pragma unroll
            for (int r = 0; r < 9; ++r) Ji[r] = act ? (T)ld(G + r) : T(0);
            T etaov;
            const T* eov = nullptr;
            if (a.eta_ip) { etaov = act ? ld(a.eta_ip + ec * 27 + q) : T(1); eov = &etaov; }
            QpMat<T> mt;
            interp_material(mt, uniform, p0, PH, m1, m2, qz, plastic, eov);
            if (!act) { mt.eta = T(1); }
            T Pq = T(0), Pfq = T(0), Pnq = T(0), Tq = T(0);
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                Pq += NPq[qz][p] * Pl[p]; Pfq += NPq[qz][p] * Pfl[p];
                Pnq += NPq[qz][p] * Pn[p]; Tq += NPq[qz][p] * Tl[p];
            }
            const T Peq = a.Pf ? Pq - Pfq : Pq;
            // Maxwell coefficients (rheology.jl:35-42)
            const T etave = T(1) / (T(1) / mt.eta + mt.invG / dt);
            const T inv2Gdt = mt.invG / (T(2) * dt);
            T told[6];
#pragma unroll
            for (int c = 0; c < 6; ++c) told[c] = (act && a.told[c]) ? ld(a.told[c] + ec * 27 + q) : T(0);
            const T (&gq)[3][3] = gp[qz];
            const T tr = (gq[0][0] + gq[1][1] + gq[2][2]) / T(3);
            const T eps_[6] = {gq[0][0] - tr, gq[1][1] - tr, gq[2][2] - tr, (gq[0][1] + gq[1][0]) / T(2),
                               (gq[0][2] + gq[2][0]) / T(2), (gq[1][2] + gq[2][1]) / T(2)};
            T tau[6];
#pragma unroll
            for (int c = 0; c < 6; ++c) tau[c] = (T(2) * etave) * (eps_[c] + told[c] * inv2Gdt);
            if (plastic) {
                // Drucker–Prager radial return (rheology.jl:441-472)
                const T tII = sqrt((tau[0] * tau[0] + tau[1] * tau[1] + tau[2] * tau[2]) / T(2) + tau[3] * tau[3] +
                                   tau[4] * tau[4] + tau[5] * tau[5] + EPS2);
                const T tIIs = tII + EPS2;
                const T Fy = tII - mt.cphi * mt.C - mt.sphi * Peq;
                const T lam = Fy > T(0) ? Fy / (etave + mt.ereg + mt.Kb * dt * (-mt.spsi) * (-mt.sphi)) : T(0);
                if (lam > T(0)) {
                    const T f = T(2) * etave * lam;
                    tau[0] -= f * (tau[0] / (T(2) * tIIs)); tau[1] -= f * (tau[1] / (T(2) * tIIs));
                    tau[2] -= f * (tau[2] / (T(2) * tIIs));
                    tau[3] -= f * (tau[3] / tIIs); tau[4] -= f * (tau[4] / tIIs); tau[5] -= f * (tau[5] / tIIs);
                }
            }
            if (act && a.tau_store[0]) {
#pragma unroll
                for (int c = 0; c < 6; ++c) a.tau_store[c][ec * 27 + q] = tau[c];
            }
            if (act && a.phi) {
                // shear_dissipation 3-D (shear_heating.jl:91-103)
                const T power = tau[0] * gq[0][0] + tau[1] * gq[1][1] + tau[2] * gq[2][2] + tau[3] * (gq[0][1] + gq[1][0]) +
                                tau[4] * (gq[0][2] + gq[2][0]) + tau[5] * (gq[1][2] + gq[2][1]);
                const T el = (tau[0] * (tau[0] - told[0]) + tau[1] * (tau[1] - told[1]) + tau[2] * (tau[2] - told[2]) +
                              T(2) * (tau[3] * (tau[3] - told[3]) + tau[4] * (tau[4] - told[4]) + tau[5] * (tau[5] - told[5]))) *
                             inv2Gdt;
                a.phi[ec * 27 + q] = power - el;
            }
            const T Ptot = (a.Pf ? Peq + Pfq : Pq) + Pnq;
            const T rhoq = mt.rho0 * (T(1) - mt.alpha * (Tq - (T)c_mat.Tref) + mt.beta * Pq);
            beta_q[qz] = act ? rhoq * dO[qz] : T(0);
            // σ = τ − Ptot·I; reference-frame flux F_cd = dΩ Σ_j J⁻¹(d, j) σ(j, c)
            const T sg[3][3] = {{tau[0] - Ptot, tau[3], tau[4]}, {tau[3], tau[1] - Ptot, tau[5]}, {tau[4], tau[5], tau[2] - Ptot}};
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    F[c][d][qz] = act ? dO[qz] * (Ji[d + 0] * sg[0][c] + Ji[d + 3] * sg[1][c] + Ji[d + 6] * sg[2][c]) : T(0);
        }
        if (!a.do_momentum) continue;

        T R[3][3];
        h27_transpose<T, true, LY>(tb, F, beta_q, gvec, E, m1, m2, R);
        if (act) {
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int i = 0; i < 3; ++i) atomic_add(a.Rv[c] + node[i], R[c][i]);
        }
    }
}

template <class T, class TG>
cudaError_t launch_hex27_residual(const H27Args<T, TG>& args, int num_sms, cudaStream_t st) {
    const int wpb = H27_THREADS / 32;
    const size_t smem = (size_t)wpb * 4 * H27Layout<T>::SLOT * sizeof(T) + (size_t)wpb * 4 * 28 * sizeof(int);
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(hex27_residual_kernel<T, TG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        configured = true;
    }
    const int64_t groups = (args.nels + 2) / 3;
    int64_t blocks = (groups + wpb - 1) / wpb;
    const int64_t cap = (int64_t)num_sms * 16;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    count_launch();
    hex27_residual_kernel<T, TG><<<(unsigned)blocks, H27_THREADS, smem, st>>>(args);
    return cudaGetLastError();
}

template cudaError_t launch_hex27_residual<double, double>(const H27Args<double, double>&, int, cudaStream_t);
template cudaError_t launch_hex27_residual<float, float>(const H27Args<float, float>&, int, cudaStream_t);
template cudaError_t launch_hex27_residual<double, float>(const H27Args<double, float>&, int, cudaStream_t);
template cudaError_t launch_hex27_residual<float, double>(const H27Args<float, double>&, int, cudaStream_t);

}  // namespace femb
