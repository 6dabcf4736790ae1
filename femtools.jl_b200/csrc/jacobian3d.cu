// jacobian3d.cu — augmented momentum-Jacobian diagnostics for Hex27/P1-disc.
//
// Restates assemble_augmented_momentum_jacobian_matrices_atomix!
// (src/stokes/assemblers/momentum_residuals.jl:998-1117): per element, the
// Jacobian of the momentum residual with Pnum = γP·RP(v)/M_P formed inline,
// evaluated with the element-max viscosity η_pc; its L1 row sums over all
// direction blocks go to dRdv and the |diagonal| of the same-direction block to
// PC. The reference differentiates with ForwardDiff; here each of the 81 columns
// is the exact directional derivative of the same expressions (the linearised
// Maxwell stress and Drucker–Prager return, rheology.jl:441-472), pushed through
// the sum-factorised transposed contraction. Line threads own fixed rows, so the
// row sums accumulate in registers without cross-thread reduction.
#include <algorithm>
#include "kernels.cuh"
#include "hex27.cuh"

namespace femb {

constexpr int JAC_THREADS = 64;                // 2 warps, 6 elements per block
constexpr int JAC_GEO = 27 * 11;               // J⁻¹ (9), dΩ, dΩ_P per point
constexpr int JAC_BP = 4 * 81;                 // ∂RP_p/∂v_(b,j)
// Shared memory per element slot (3 elements and an idle-lane slot per warp). The
// column loop's transposed contraction stores its two intermediate stages with the
// strided layouts LA(i,j,k) = 3i + 9j + 10k and LB(i,j,k) = 9i + 10j + 3k (45 words
// per component block); with slots 1025 ≡ 1 (mod 32) words apart and the idle lanes
// on m = 8, every stage access of the warp hits 28 distinct banks. The geometry
// slots, 306 ≡ 18 (mod 32) words apart, are conflict-free for the same lane map.
// FP64 uses the bank-conflict-free h27 stage buffers (H27Fp64Banked) for the gradient
// and the column loop's transposes, with element slots 859 ≡ 539 (mod 16) words apart,
// geometry slots 307 ≡ 3 (mod 16) apart and the idle lanes on m = 2: 480 shared
// wavefronts per gradient + transpose instead of the compact layout's 1 152 in 864-word
// slots, and two per geometry read instead of four.
constexpr int JAC_LA = 9 * 45;                 // stage-1 scratch: 9 blocks
template <class T>
struct JacSmem {
    static constexpr bool strided = sizeof(T) == 4;
    using LY = std::conditional_t<strided, H27Compact, H27Fp64Banked>;   // h27 stage buffers
    static constexpr int stage = strided ? JAC_LA + 6 * 45 : h27_stage_words<H27Fp64Banked>();   // BP follows
    static constexpr int e_stride = strided ? 1025 : 859;
    static constexpr int g_stride = strided ? 306 : 307;
    static constexpr int idle_m = strided ? 8 : H27Fp64Banked::IDLE_M;
    static_assert(stage + JAC_BP <= e_stride && stage >= h27_stage_words<LY>() && g_stride >= JAC_GEO, "slot layout");
    static_assert(strided ? (e_stride % 32 == 1 && g_stride % 32 == 18)
                          : (e_stride % 16 == H27Fp64Banked::SLOT % 16 && g_stride % 16 == 3), "bank layout");
};

FEMB_D int jla(int i, int j, int k) { return 3 * i + 9 * j + 10 * k; }
FEMB_D int jlb(int i, int j, int k) { return 9 * i + 10 * j + 3 * k; }

// h27_transpose without body force, with the conflict-free stage layouts above.
template <class T>
FEMB_D void jac_transpose(const Tab1D<T>& t, const T F[3][3][3], T* E, int m1, int m2, T R[3][3]) {
    // Z^T: thread owns z-line (qx = m1, qy = m2)
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int iz = 0; iz < 3; ++iz) {
            E[(c * 3 + 0) * 45 + jla(m1, m2, iz)] = t.B[0][iz] * F[c][0][0] + t.B[1][iz] * F[c][0][1] + t.B[2][iz] * F[c][0][2];
            E[(c * 3 + 1) * 45 + jla(m1, m2, iz)] = t.B[0][iz] * F[c][1][0] + t.B[1][iz] * F[c][1][1] + t.B[2][iz] * F[c][1][2];
            E[(c * 3 + 2) * 45 + jla(m1, m2, iz)] = t.Dd[0][iz] * F[c][2][0] + t.Dd[1][iz] * F[c][2][1] + t.Dd[2][iz] * F[c][2][2];
        }
    __syncwarp();
    // Y^T: thread owns y-line (qx = m1, ·, iz = m2)
    T* E1 = E + JAC_LA;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        T TA[3], TB[3], TC[3];
#pragma unroll
        for (int qy = 0; qy < 3; ++qy) {
            TA[qy] = E[(c * 3 + 0) * 45 + jla(m1, qy, m2)];
            TB[qy] = E[(c * 3 + 1) * 45 + jla(m1, qy, m2)];
            TC[qy] = E[(c * 3 + 2) * 45 + jla(m1, qy, m2)];
        }
#pragma unroll
        for (int iy = 0; iy < 3; ++iy) {
            E1[(c * 2 + 0) * 45 + jlb(m1, iy, m2)] = t.B[0][iy] * TA[0] + t.B[1][iy] * TA[1] + t.B[2][iy] * TA[2];
            E1[(c * 2 + 1) * 45 + jlb(m1, iy, m2)] = (t.Dd[0][iy] * TB[0] + t.Dd[1][iy] * TB[1] + t.Dd[2][iy] * TB[2]) +
                                                      (t.B[0][iy] * TC[0] + t.B[1][iy] * TC[1] + t.B[2][iy] * TC[2]);
        }
    }
    __syncwarp();
    // X^T: thread owns x-line (·, iy = m1, iz = m2)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        T UA[3], UB[3];
#pragma unroll
        for (int qx = 0; qx < 3; ++qx) { UA[qx] = E1[(c * 2 + 0) * 45 + jlb(qx, m1, m2)]; UB[qx] = E1[(c * 2 + 1) * 45 + jlb(qx, m1, m2)]; }
#pragma unroll
        for (int ix = 0; ix < 3; ++ix)
            R[c][ix] = (t.Dd[0][ix] * UA[0] + t.Dd[1][ix] * UA[1] + t.Dd[2][ix] * UA[2]) +
                       (t.B[0][ix] * UB[0] + t.B[1][ix] * UB[1] + t.B[2][ix] * UB[2]);
    }
    __syncwarp();
}

// Input match of an element against its phase's shared Jacobian (FP32 diagnostics of the
// mixed-precision solve): within 4e-7 of `scale` (about 3 ulp; structured generators form
// J = Σ dN_a·x_a, whose last bits vary with the element's position, and the FP32 assembly
// carries rounding of that order anyway). `scale` is the entry itself, or for J⁻¹ entries
// the largest |J⁻¹| of the point (its off-diagonals carry rounding residues near zero on
// axis-aligned cells).
FEMB_D bool same_input(float g, float t, float scale) { return fabsf(g - t) <= 4e-7f * scale; }
FEMB_D bool same_input(double g, double t, double) { return g == t; }

// DIAG: every J⁻¹ is diagonal (axis-aligned boxes); the gradient and flux transforms
// are one product per entry.
template <class T, class TG, bool DIAG>
__global__ void __launch_bounds__(JAC_THREADS) hex27_jacobian_kernel(H27JacArgs<T, TG> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const bool lane_ok = lane < 27;
    // lanes 27..31 carry no element; they work in a private scratch slot (3) so
    // their (discarded) stage writes never touch an element's shared memory.
    using L = JacSmem<T>;
    const int s = lane_ok ? lane / 9 : 3, m = lane_ok ? lane % 9 : L::idle_m, m1 = m % 3, m2 = m / 3;
    T* E = reinterpret_cast<T*>(smem_raw) + ((size_t)warp * 4 + s) * L::e_stride;
    T* GEO = reinterpret_cast<T*>(smem_raw) + (size_t)wpb * 4 * L::e_stride + ((size_t)warp * 4 + s) * L::g_stride;
    T* BP = E + L::stage;
    int* PH = reinterpret_cast<int*>(reinterpret_cast<T*>(smem_raw) + (size_t)wpb * 4 * (L::e_stride + L::g_stride)) +
              (warp * 4 + s) * 28;

    Tab1D<T> tb; tb.load();
    const T dt = a.dt;
    const bool plastic = c_mat.plastic != 0;
    const T EPS2 = eps2<T>();
    const T zero3[3] = {T(0), T(0), T(0)};

    // the shared element Jacobians exist in the FP32 diagnostics (the mixed-precision solve)
    constexpr bool SHARE = sizeof(T) == 4;
    const bool build = SHARE && a.tmpl_mode == JAC_TMPL_BUILD;
    // work item gk is group gk (three elements), or the gk-th group of the launch's list
    const bool listed = a.group_list != nullptr && !build;
    const int64_t gstride = (int64_t)gridDim.x * wpb;
    const int64_t ngroups = listed ? a.group_count : (a.nels + 2) / 3;
    for (int64_t gk = (int64_t)blockIdx.x * wpb + warp; gk < ngroups; gk += gstride) {
        const int64_t base = listed ? 3 * (int64_t)__ldg(a.group_list + gk) : 3 * gk;
        // building templates, slot k of the loop is phase k and its element pick[k]
        const int64_t k = base + (lane_ok ? s : 0);
        const bool picked = build && k < MAXPH && a.pick[k] >= 0 && a.pick[k] < a.pick_nels;
        const int64_t e = build ? (picked ? (int64_t)a.pick[k] : 0) : k;
        const bool act = lane_ok && (build ? picked : e < a.nels);
        const int64_t ec = act ? e : 0;

        int node[3];
        T v[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            node[i] = act ? __ldg(a.el2n + 27 * ec + c_tab.tn3[tidx(i, m1, m2)]) - 1 : 0;
#pragma unroll
            for (int c = 0; c < 3; ++c) v[c][i] = act ? ld(a.v[c] + node[i]) : T(0);
        }
        // phases: always staged so that the element maximum can be formed
        int p0 = 0;
        bool uniform = true;
        if (a.phv_layout == FEMB200_PHASE_CELL || !a.phv) {
            p0 = a.phv ? (act ? __ldg(a.phv + ec) - 1 : 0) : 0;
#pragma unroll
            for (int i = 0; i < 3; ++i) PH[tidx(i, m1, m2)] = p0;
            __syncwarp();
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
        int dof[4];
        T Pl[4], Pfl[4], gam[4], MPl[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            dof[p] = act ? __ldg(a.dofsP + 4 * ec + p) - 1 : 0;
            Pl[p] = act ? ld(a.P + dof[p]) : T(0);
            Pfl[p] = (act && a.Pf) ? ld(a.Pf + dof[p]) : T(0);
            gam[p] = (act && a.gammaP) ? ld(a.gammaP + dof[p]) : T(0);
            MPl[p] = (act && a.MP) ? ld(a.MP + dof[p]) : T(1);
        }
        // geometry of all 27 points of the element into shared memory
#pragma unroll
        for (int qz = 0; qz < 3; ++qz) {
            const int q = tidx(m1, m2, qz);
            const TG* G = a.geo_v + ((int64_t)ec * 27 + q) * 10;
#pragma unroll
            for (int r = 0; r < 10; ++r) GEO[q * 11 + r] = act ? (T)ld(G + r) : T(0);
            GEO[q * 11 + 10] = act ? (T)ld(a.geo_P + (int64_t)ec * 27 + q) : T(0);
        }
        // element-max viscosity η_pc (_element_max_phase_property, momentum_residuals.jl:36-44)
        T eta_pc;
        bool eta_scalar = false;
        if (a.eta_ip) {
            T mx = T(-INFINITY);
#pragma unroll
            for (int qz = 0; qz < 3; ++qz) mx = fmax(mx, act ? ld(a.eta_ip + ec * 27 + tidx(m1, m2, qz)) : T(-INFINITY));
            E[460 + m] = mx;
            __syncwarp();
            mx = E[460];
            for (int t = 1; t < 9; ++t) mx = fmax(mx, E[460 + t]);
            __syncwarp();
            eta_pc = mx;
            eta_scalar = true;
        } else {
            T mx = (T)c_mat.eta[PH[0]];
            for (int t = 1; t < 27; ++t) mx = fmax(mx, (T)c_mat.eta[PH[t]]);
            eta_pc = mx;
        }

        T g[3][3][3];
        h27_gradient<T, typename L::LY>(tb, v, E, m1, m2, g);

        // primal state at the owned points with η_pc
        // per point: ηve, λ, the trial stress and the reciprocals the 81 columns use
        T pe[3], plam[3], ptt[3][6], pitII[3], pitIIs[3], piden[3];
#pragma unroll
        for (int qz = 0; qz < 3; ++qz) {
            const int q = tidx(m1, m2, qz);
            const T* Ji = GEO + q * 11;
            T gq[3][3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    gq[c][k] = DIAG ? g[c][k][qz] * Ji[4 * k]
                                    : g[c][0][qz] * Ji[0 + 3 * k] + g[c][1][qz] * Ji[1 + 3 * k] + g[c][2][qz] * Ji[2 + 3 * k];
            const T sN = (T)c_tab.sumN3[q];
            T invG, cphi = 0, sphi = 0, spsi = 0, C = 0, ereg = 0, Kb = 0;
            if (uniform) {
                invG = (T)c_mat.invG[p0] * sN;
                if (plastic) {
                    cphi = (T)c_mat.cos_phi[p0] * sN; sphi = (T)c_mat.sin_phi[p0] * sN; spsi = (T)c_mat.sin_psi[p0] * sN;
                    C = (T)c_mat.C[p0] * sN; ereg = (T)c_mat.eta_reg[p0] * sN; Kb = (T)c_mat.Kb[p0] * sN;
                }
            } else {
                invG = T(0);
                for (int kk = 0; kk < 3; ++kk)
                    for (int jj = 0; jj < 3; ++jj)
                        for (int ii = 0; ii < 3; ++ii) {
                            const T N = tb.B[m1][ii] * tb.B[m2][jj] * tb.B[qz][kk];
                            const int p = PH[tidx(ii, jj, kk)];
                            invG += N * (T)c_mat.invG[p];
                            if (plastic) {
                                cphi += N * (T)c_mat.cos_phi[p]; sphi += N * (T)c_mat.sin_phi[p];
                                spsi += N * (T)c_mat.sin_psi[p]; C += N * (T)c_mat.C[p];
                                ereg += N * (T)c_mat.eta_reg[p]; Kb += N * (T)c_mat.Kb[p];
                            }
                        }
            }
            const T etaq = eta_scalar ? eta_pc : eta_pc * sN;
            const T etave = T(1) / (T(1) / etaq + invG / dt);
            const T inv2Gdt = invG / (T(2) * dt);
            const T tr = (gq[0][0] + gq[1][1] + gq[2][2]) / T(3);
            const T eps_[6] = {gq[0][0] - tr, gq[1][1] - tr, gq[2][2] - tr, (gq[0][1] + gq[1][0]) / T(2),
                               (gq[0][2] + gq[2][0]) / T(2), (gq[1][2] + gq[2][1]) / T(2)};
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                const T to = (act && a.told[c]) ? ld(a.told[c] + ec * 27 + q) : T(0);
                ptt[qz][c] = (T(2) * etave) * (eps_[c] + to * inv2Gdt);
            }
            pe[qz] = etave;
            plam[qz] = T(0);
            pitII[qz] = T(1); pitIIs[qz] = T(1); piden[qz] = T(1);
            if (plastic) {
                T Pq = T(0), Pfq = T(0);
#pragma unroll
                for (int p = 0; p < 4; ++p) {
                    const T xi = (T)c_tab.qx[m1], et = (T)c_tab.qx[m2], ze = (T)c_tab.qx[qz];
                    const T NP = p == 0 ? T(1) - xi - et - ze : (p == 1 ? xi : (p == 2 ? et : ze));
                    Pq += NP * Pl[p]; Pfq += NP * Pfl[p];
                }
                const T Peq = a.Pf ? Pq - Pfq : Pq;
                const T* t = ptt[qz];
                const T tII = sqrt((t[0] * t[0] + t[1] * t[1] + t[2] * t[2]) / T(2) + t[3] * t[3] + t[4] * t[4] + t[5] * t[5] + EPS2);
                const T Fy = tII - cphi * C - sphi * Peq;
                const T den = etave + ereg + Kb * dt * (-spsi) * (-sphi);
                const T lam = Fy > T(0) && !build ? Fy / den : T(0);
                plam[qz] = lam; pitII[qz] = T(1) / tII; pitIIs[qz] = T(1) / (tII + EPS2); piden[qz] = T(1) / den;
            }
        }

        // a warp whose three elements are elastic here and carry their phase template's
        // inputs bit for bit takes the template's rows (computed by this code on those inputs)
        bool shared = false;
        if (SHARE && a.tmpl_mode == JAC_TMPL_USE) {
            bool mine = !act;
            if (act && uniform && p0 >= 0 && p0 < MAXPH) {
                const JacTemplate<T>& tm = a.tmpl[p0];
                bool ok = tm.valid != 0 && plam[0] == T(0) && plam[1] == T(0) && plam[2] == T(0) &&
                          same_input(eta_pc, tm.eta_pc, fabs(tm.eta_pc));
#pragma unroll
                for (int p = 0; p < 4; ++p)
                    ok = ok && same_input(gam[p], tm.gam[p], fabs(tm.gam[p])) && same_input(MPl[p], tm.MP[p], fabs(tm.MP[p]));
#pragma unroll
                for (int qz = 0; qz < 3; ++qz) {
                    const int q = tidx(m1, m2, qz);
                    T jmax = T(0);
                    if constexpr (sizeof(T) == 4) {
#pragma unroll
                        for (int r = 0; r < 9; ++r) jmax = fmax(jmax, fabs(tm.geo[q * 11 + r]));
                    }
#pragma unroll
                    for (int r = 0; r < 11; ++r)
                        ok = ok && same_input(GEO[q * 11 + r], tm.geo[q * 11 + r],
                                              sizeof(T) == 4 && r < 9 ? jmax : fabs(tm.geo[q * 11 + r]));
                }
                mine = ok;
            }
            shared = __all_sync(0xffffffffu, mine || !lane_ok);
            if (shared && a.shared_count) {
                const unsigned n = __popc(__ballot_sync(0xffffffffu, act && m == 0));
                if (lane == 0 && n) atomicAdd(a.shared_count, (unsigned long long)n);
            }
        }
        T rows[3][3], diag[3][3];
        if (SHARE && shared) {
            if (act) {
                const JacTemplate<T>& tm = a.tmpl[p0];
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        rows[c][i] = tm.rows[tidx(i, m1, m2) * 3 + c];
                        diag[c][i] = tm.diag[tidx(i, m1, m2) * 3 + c];
                    }
            }
        } else {

        // ∂RP_p/∂v_(b,j) = −Σ_q NP_p(q) ∂_j N_b(q) dΩ_P(q) for every column, via the
        // transposed contraction with a unit "pressure" flux per p.
#pragma unroll 1
        for (int p = 0; p < 4; ++p) {
            T Fp[3][3][3];
#pragma unroll
            for (int qz = 0; qz < 3; ++qz) {
                const int q = tidx(m1, m2, qz);
                const T* Ji = GEO + q * 11;
                const T xi = (T)c_tab.qx[m1], et = (T)c_tab.qx[m2], ze = (T)c_tab.qx[qz];
                const T NP = p == 0 ? T(1) - xi - et - ze : (p == 1 ? xi : (p == 2 ? et : ze));
                const T w = -NP * Ji[10];
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int d = 0; d < 3; ++d) Fp[c][d][qz] = DIAG ? (c == d ? w * Ji[4 * c] : T(0)) : w * Ji[d + 3 * c];
            }
            T Rp[3][3];
            if constexpr (L::strided) jac_transpose<T>(tb, Fp, E, m1, m2, Rp);
            else h27_transpose<T, false, typename L::LY>(tb, Fp, zero3, zero3, E, m1, m2, Rp);
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int i = 0; i < 3; ++i) BP[p * 81 + tidx(i, m1, m2) * 3 + c] = Rp[c][i] * gam[p] / MPl[p];
        }
        __syncwarp();

#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int i = 0; i < 3; ++i) { rows[c][i] = T(0); diag[c][i] = T(0); }

#pragma unroll 1
        for (int b = 0; b < 27; ++b) {
            const int bx = b % 3, by = (b / 3) % 3, bz = b / 9;
            // physical gradient of N_b at the owned points, shared by the three columns of node b
            T dnb[3][3];
#pragma unroll
            for (int qz = 0; qz < 3; ++qz) {
                const T* Ji = GEO + tidx(m1, m2, qz) * 11;
                const T rx = tb.Dd[m1][bx] * tb.B[m2][by] * tb.B[qz][bz];
                const T ry = tb.B[m1][bx] * tb.Dd[m2][by] * tb.B[qz][bz];
                const T rz = tb.B[m1][bx] * tb.B[m2][by] * tb.Dd[qz][bz];
                if (DIAG) {
                    dnb[qz][0] = rx * Ji[0]; dnb[qz][1] = ry * Ji[4]; dnb[qz][2] = rz * Ji[8];
                } else {
#pragma unroll
                    for (int k = 0; k < 3; ++k) dnb[qz][k] = rx * Ji[0 + 3 * k] + ry * Ji[1 + 3 * k] + rz * Ji[2 + 3 * k];
                }
            }
#pragma unroll 1
            for (int j = 0; j < 3; ++j) {
                const int col = b * 3 + j;
                const T dPn0 = BP[0 * 81 + col], dPn1 = BP[1 * 81 + col], dPn2 = BP[2 * 81 + col], dPn3 = BP[3 * 81 + col];
                T Fd[3][3][3];
#pragma unroll
                for (int qz = 0; qz < 3; ++qz) {
                    const int q = tidx(m1, m2, qz);
                    const T* Ji = GEO + q * 11;
                    const T (&dn)[3] = dnb[qz];
                    // δg[i][k] = δ_ij dn[k]
                    T dg[3][3];
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int k = 0; k < 3; ++k) dg[i][k] = (i == j) ? dn[k] : T(0);
                    const T tr = (dg[0][0] + dg[1][1] + dg[2][2]) * T(1.0 / 3.0);
                    const T de[6] = {dg[0][0] - tr, dg[1][1] - tr, dg[2][2] - tr, (dg[0][1] + dg[1][0]) * T(0.5),
                                     (dg[0][2] + dg[2][0]) * T(0.5), (dg[1][2] + dg[2][1]) * T(0.5)};
                    const T two_e = T(2) * pe[qz];
                    T dt_[6];
#pragma unroll
                    for (int c = 0; c < 6; ++c) dt_[c] = two_e * de[c];
                    T dtau[6];
                    if (plam[qz] > T(0)) {
                        // linearised radial return (rheology.jl:441-472) with the reciprocals
                        // of τII, τII + ε² and the plastic denominator formed once per point
                        const T* t = ptt[qz];
                        const T itII = pitII[qz], itIIs = pitIIs[qz];
                        const T dtII = ((t[0] * dt_[0] + t[1] * dt_[1] + t[2] * dt_[2]) * T(0.5) +
                                        (t[3] * dt_[3] + t[4] * dt_[4] + t[5] * dt_[5])) * itII;
                        const T dlam = dtII * piden[qz];
                        const T lam = plam[qz];
#pragma unroll
                        for (int c = 0; c < 6; ++c) {
                            const T ifac = c < 3 ? T(0.5) * itIIs : itIIs;
                            const T mq = t[c] * ifac;
                            const T dm = (dt_[c] - t[c] * dtII * itIIs) * ifac;
                            dtau[c] = dt_[c] - two_e * (dlam * mq + lam * dm);
                        }
                    } else {
#pragma unroll
                        for (int c = 0; c < 6; ++c) dtau[c] = dt_[c];
                    }
                    const T xi = (T)c_tab.qx[m1], et = (T)c_tab.qx[m2], ze = (T)c_tab.qx[qz];
                    const T dPn = (T(1) - xi - et - ze) * dPn0 + xi * dPn1 + et * dPn2 + ze * dPn3;
                    const T sg[3][3] = {{dtau[0] - dPn, dtau[3], dtau[4]}, {dtau[3], dtau[1] - dPn, dtau[5]},
                                        {dtau[4], dtau[5], dtau[2] - dPn}};
                    const T dOq = Ji[9];
#pragma unroll
                    for (int c = 0; c < 3; ++c)
#pragma unroll
                        for (int d = 0; d < 3; ++d)
                            Fd[c][d][qz] = DIAG ? dOq * Ji[4 * d] * sg[d][c]
                                                : dOq * (Ji[d + 0] * sg[0][c] + Ji[d + 3] * sg[1][c] + Ji[d + 6] * sg[2][c]);
                }
                T dR[3][3];
                if constexpr (L::strided) jac_transpose<T>(tb, Fd, E, m1, m2, dR);
                else h27_transpose<T, false, typename L::LY>(tb, Fd, zero3, zero3, E, m1, m2, dR);
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        rows[c][i] += fabs(dR[c][i]);
                        if (c == j && tidx(i, m1, m2) == b) diag[c][i] = fabs(dR[c][i]);
                    }
            }
        }
        }
        if (SHARE && act && build) {
            JacTemplate<T>& tm = a.tmpl[k];
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    tm.rows[tidx(i, m1, m2) * 3 + c] = rows[c][i];
                    tm.diag[tidx(i, m1, m2) * 3 + c] = diag[c][i];
                }
#pragma unroll
            for (int qz = 0; qz < 3; ++qz) {
                const int q = tidx(m1, m2, qz);
#pragma unroll
                for (int r = 0; r < 11; ++r) tm.geo[q * 11 + r] = GEO[q * 11 + r];
            }
            if (m == 0) {
#pragma unroll
                for (int p = 0; p < 4; ++p) { tm.gam[p] = gam[p]; tm.MP[p] = MPl[p]; }
                tm.eta_pc = eta_pc;
                // only a one-phase element is a template; the flag is read by a later launch
                tm.valid = uniform ? 1 : 0;
            }
        } else {
            // ordered scatter: each node of the group receives one addition (hex27.cuh)
            bool folded = false;
            if (listed) {
                folded = fold_next_element(node, act, s, rows);
                fold_next_element(node, act, s, diag);
            }
            if (act) {
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int i = 0; i < 3; ++i)
                        if (i > 0 || !folded) {
                            atomic_add(a.dRdv[c] + node[i], rows[c][i]);
                            atomic_add(a.PC[c] + node[i], diag[c][i]);
                        }
            }
        }
        __syncwarp();
    }
}

namespace {
// Sets *flag when any integration point's J⁻¹ has an off-diagonal entry above 1e-13 of
// its diagonal's magnitude. Axis-aligned cells have mathematically zero off-diagonals;
// the geometry computed from their coordinates carries rounding residues of order 1e-17
// there, which the diagonal kernel drops (an error far below the FP64 arithmetic's own).
template <class TG>
__global__ void geo_offdiag_kernel(const TG* geo_v, int64_t npts, int* flag) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npts; i += (int64_t)gridDim.x * blockDim.x) {
        const TG* g = geo_v + i * 10;
        const double dsum = fabs((double)g[0]) + fabs((double)g[4]) + fabs((double)g[8]);
        double off = 0;
        for (int r : {1, 2, 3, 5, 6, 7}) off = fmax(off, fabs((double)g[r]));
        if (!(off <= 1e-13 * dsum)) *flag = 1;
    }
}
}  // namespace

namespace {
__global__ void jac_pick_kernel(const int32_t* phv, int64_t nels, int32_t* pick) {
    // the block's lowest element per phase in shared memory, then one global atomic per
    // phase and block (all elements of a phase contend on one word otherwise)
    __shared__ int32_t smin[MAXPH];
    for (int t = threadIdx.x; t < MAXPH; t += blockDim.x) smin[t] = JAC_NO_PICK;
    __syncthreads();
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nels; e += (int64_t)gridDim.x * blockDim.x) {
        const int p = phv ? phv[e] - 1 : 0;
        if (p >= 0 && p < MAXPH && e < JAC_NO_PICK) atomicMin(smin + p, (int32_t)e);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < MAXPH; t += blockDim.x)
        if (smin[t] != JAC_NO_PICK) atomicMin(pick + t, smin[t]);
}
}  // namespace

cudaError_t launch_jac_pick(const int32_t* phv, int64_t nels, int32_t* pick, cudaStream_t st) {
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((nels + 255) / 256, 148 * 8));
    count_launch();
    jac_pick_kernel<<<(unsigned)blocks, 256, 0, st>>>(phv, nels, pick);
    return cudaGetLastError();
}

template <class TG>
cudaError_t launch_geo_offdiag(const TG* geo_v, int64_t nels, int* flag, cudaStream_t st) {
    const int64_t n = nels * 27;
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16));
    count_launch();
    geo_offdiag_kernel<TG><<<(unsigned)blocks, 256, 0, st>>>(geo_v, n, flag);
    return cudaGetLastError();
}
template cudaError_t launch_geo_offdiag<double>(const double*, int64_t, int*, cudaStream_t);
template cudaError_t launch_geo_offdiag<float>(const float*, int64_t, int*, cudaStream_t);

template <class T, class TG>
cudaError_t launch_hex27_jacobian(const H27JacArgs<T, TG>& args, int num_sms, cudaStream_t st) {
    const int wpb = JAC_THREADS / 32;
    const size_t smem = (size_t)wpb * 4 * (JacSmem<T>::e_stride + JacSmem<T>::g_stride) * sizeof(T) +
                        (size_t)wpb * 4 * 28 * sizeof(int);
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(hex27_jacobian_kernel<T, TG, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(hex27_jacobian_kernel<T, TG, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        configured = true;
    }
    const int64_t groups = (args.group_list && args.tmpl_mode != JAC_TMPL_BUILD) ? args.group_count : (args.nels + 2) / 3;
    if (groups < 1) return cudaSuccess;
    int64_t blocks = (groups + wpb - 1) / wpb;
    const int64_t cap = (int64_t)num_sms * 32;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    count_launch();
    if (args.diag_geometry) hex27_jacobian_kernel<T, TG, true><<<(unsigned)blocks, JAC_THREADS, smem, st>>>(args);
    else hex27_jacobian_kernel<T, TG, false><<<(unsigned)blocks, JAC_THREADS, smem, st>>>(args);
    return cudaGetLastError();
}

template cudaError_t launch_hex27_jacobian<double, double>(const H27JacArgs<double, double>&, int, cudaStream_t);
template cudaError_t launch_hex27_jacobian<float, float>(const H27JacArgs<float, float>&, int, cudaStream_t);
template cudaError_t launch_hex27_jacobian<double, float>(const H27JacArgs<double, float>&, int, cudaStream_t);
template cudaError_t launch_hex27_jacobian<float, double>(const H27JacArgs<float, double>&, int, cudaStream_t);

}  // namespace femb
