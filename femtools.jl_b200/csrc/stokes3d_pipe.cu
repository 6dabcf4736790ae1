// stokes3d_pipe.cu — software-pipelined Hex27/P1-disc residual sweep for affine meshes.
//
// Same arithmetic as stokes3d.cu (pressure residual, element-local Pnum, visco-
// elasto-plastic momentum residual), restructured for HBM bandwidth:
//   * geometry: on meshes whose elements are affine (the structured generators'
//     boxes and any parallelepiped cells) the per-point J⁻¹ and |det J|·ω of the
//     reference layout collapse to one J⁻¹ and |det J| per element, built once per
//     solve by compress_geometry (80 B per element instead of 2376 B);
//   * each warp keeps three elements in flight; as soon as the quadrature loop
//     of the current group has consumed its shared-memory buffer, the warp issues
//     the next group's stress history, geometry and pressure-DoF loads (cp.async)
//     into that buffer and its velocity gather into registers, so the loads
//     overlap the transposed contraction, the scatter and the next gradient;
//   * one buffer per element slot (not two) keeps shared memory at 17 KB per warp
//     (FP64) and 8.5 KB (FP32), so FP32 runs 16 resident warps per SM;
//   * elements whose 27 nodes share a phase use per-phase constants prepared on
//     the host (ηve, 2ηve, C·cosϕ, the reciprocal plastic denominator).
#include "kernels.cuh"
#include "hex27.cuh"
#include "rheology.cuh"

namespace femb {

// Threads per block (one block per SM): 8 warps in FP64 (more would spill the
// 27-value gradient/flux lines of each thread), 16 in FP32.
template <class T> struct PipeThreads { static constexpr int value = 256; };
template <> struct PipeThreads<float> { static constexpr int value = 512; };
// Stage scratch per element slot and the layout of its buffers: FP64 uses the
// bank-conflict-free H27Fp64Banked buffers with slots 523 words apart and the idle lanes
// reading along line m = 0 of slot 2 (480 shared wavefronts per gradient + transpose in
// place of 750); FP32 keeps i + 3j + 9k in 500-word slots.
template <class T> struct PipeStage {
    using LY = H27Compact;
    static constexpr int WORDS = 500, IDLE_S = 0, IDLE_M = 0;
};
template <> struct PipeStage<double> {
    using LY = H27Fp64Banked;
    static constexpr int WORDS = 523, IDLE_S = 2, IDLE_M = 0;
};
static_assert(h27_stage_words<H27Compact>() <= PipeStage<float>::WORDS &&
              h27_stage_words<H27Fp64Banked>() <= PipeStage<double>::WORDS, "pipe stage scratch");
// Load buffer of one element slot: per-point fields (τ_old, 6 × 27; or, in the
// incremental sweep, the base trial stress and yield value, 7 × 27), the affine
// geometry (10) and the pressure-DoF data (32).
template <bool INCR> struct PipeLayout {
    static constexpr int NT = INCR ? 7 : 6;
    static constexpr int GEO = NT * 27;
    static constexpr int DOF = GEO + 10;
    static constexpr int BUF = INCR ? 232 : 208;
};
// Words between the load buffers of consecutive element slots: the buffer rounded up to
// 9 modulo the bank count (16 eight-byte banks per half-warp in FP64, 32 four-byte banks
// in FP32), so that the three slots' point reads (offsets m1 + 3m2 of each slot) and
// their geometry broadcasts fall in distinct banks.
template <class T, bool INCR> constexpr int pipe_buf() {
    constexpr int banks = sizeof(T) == 8 ? 16 : 32;
    constexpr int b = PipeLayout<INCR>::BUF;
    return b + ((9 - b % banks) % banks + banks) % banks;
}
static_assert(pipe_buf<double, false>() % 16 == 9 && pipe_buf<double, true>() % 16 == 9 &&
              pipe_buf<float, false>() % 32 == 9 && pipe_buf<float, true>() % 32 == 9 &&
              pipe_buf<double, false>() >= PipeLayout<false>::BUF && pipe_buf<float, true>() >= PipeLayout<true>::BUF,
              "load-buffer stride");
enum { PT_TWOE, PT_TWOE_EL, PT_RHO0, PT_ALPHA, PT_BETA, PT_CC, PT_SPHI, PT_INVDEN, PT_INVBULKDT, PT_BULK, PT_FIELDS };

namespace {

FEMB_D void cp_async(double* dst, const double* src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(src) : "memory");
}
FEMB_D void cp_async(float* dst, const float* src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(src) : "memory");
}
FEMB_D void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
FEMB_D void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Identifiers of one element group as seen by one lane.
struct GroupIds {
    int node[3];    // 0-based nodes of the lane's x-line
    int dof;        // 0-based pressure DoF m (lanes m < 4)
    int phase;      // cell phase (0-based) or 0
    bool act;
};

template <class T>
FEMB_D GroupIds load_ids(const H27Args<T, T>& a, int64_t base, int s, int m, const int tn_own[3], bool lane_ok) {
    GroupIds g;
    const int64_t e = base + s;
    g.act = lane_ok && base >= 0 && e < a.nels;
    const int64_t ec = g.act ? e : 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) g.node[i] = g.act ? __ldg(a.el2n + 27 * ec + tn_own[i]) - 1 : 0;
    g.dof = (g.act && m < 4) ? __ldg(a.dofsP + 4 * ec + m) - 1 : 0;
    g.phase = (g.act && a.phv && a.phv_layout == FEMB200_PHASE_CELL) ? __ldg(a.phv + ec) - 1 : 0;
    return g;
}

// Issue the prefetch of one group: velocity gather into registers, stress history,
// geometry and pressure-DoF data into the shared-memory buffer.
template <class T, bool INCR>
FEMB_D void issue_prefetch(const H27Args<T, T>& a, const T* geo_c, const GroupIds& id, int64_t base, int s, int m,
                           int m1, int m2, T* buf, T vn[3][3]) {
    using L = PipeLayout<INCR>;
    if (!id.act) return;
    const int64_t e = base + s;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c) vn[c][i] = ld(a.v[c] + id.node[i]);
    T* B = buf + s * pipe_buf<T, INCR>();
    if constexpr (INCR) {
#pragma unroll
        for (int c = 0; c < 7; ++c)
#pragma unroll
            for (int qz = 0; qz < 3; ++qz) {
                const int q = tidx(m1, m2, qz);
                cp_async(B + c * 27 + q, a.base_in + base_index(e, q, c));
            }
    } else if (a.told[0]) {
#pragma unroll
        for (int c = 0; c < 6; ++c)
#pragma unroll
            for (int qz = 0; qz < 3; ++qz) {
                const int q = tidx(m1, m2, qz);
                cp_async(B + c * 27 + q, a.told[c] + e * 27 + q);
            }
    }
    cp_async(B + L::GEO + m, geo_c + e * 10 + m);
    if (m == 0) cp_async(B + L::GEO + 9, geo_c + e * 10 + 9);
    if (m < 4) {
        T* D = B + L::DOF;
        cp_async(D + 0 * 4 + m, a.P + id.dof);
        if constexpr (INCR) cp_async(D + 1 * 4 + m, a.RP_base + id.dof);
        if (a.P0) cp_async(D + 1 * 4 + m, a.P0 + id.dof);
        if (a.gammaP) cp_async(D + 2 * 4 + m, a.gammaP + id.dof);
        if (a.MP) cp_async(D + 3 * 4 + m, a.MP + id.dof);
        if (a.temp) cp_async(D + 4 * 4 + m, a.temp + id.dof);
        if (a.temp0) cp_async(D + 5 * 4 + m, a.temp0 + id.dof);
        if (a.Q) cp_async(D + 6 * 4 + m, a.Q + id.dof);
        if (a.Pf) cp_async(D + 7 * 4 + m, a.Pf + id.dof);
    }
}

}  // namespace

template <class T, bool INCR>
__global__ void __launch_bounds__(PipeThreads<T>::value, 1) hex27_residual_pipe_kernel(H27Args<T, T> a, const T* __restrict__ geo_c) {
    static_assert(!INCR || sizeof(T) == 4, "the incremental sweep runs in FP32");
    using L = PipeLayout<INCR>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const bool lane_ok = lane < 27;
    // lanes 27..31 carry no element: they follow one slot's reads but never write
    using PS = PipeStage<T>;
    using LY = typename PS::LY;
    constexpr int PL_STAGE = PS::WORDS;
    const int s = lane_ok ? lane / 9 : PS::IDLE_S, m = lane_ok ? lane % 9 : PS::IDLE_M, m1 = m % 3, m2 = m / 3;
    constexpr int SB = pipe_buf<T, INCR>();
    T* base_w = reinterpret_cast<T*>(smem_raw) + (size_t)warp * (3 * PL_STAGE + 3 * SB);
    T* E = base_w + s * PL_STAGE;
    T* BUF = base_w + 3 * PL_STAGE;
    int* PH = reinterpret_cast<int*>(reinterpret_cast<T*>(smem_raw) + (size_t)wpb * (3 * PL_STAGE + 3 * SB)) +
              (warp * 3 + s) * 28;
    const int sl = s;

    Tab1D<T> tb; tb.load();
    const T dt = a.dt;
    const T gvec[3] = {(T)c_mat.g[0], (T)c_mat.g[1], (T)c_mat.g[2]};
    const bool plastic = c_mat.plastic != 0;
    const bool consts_ok = c_mat.dt_consts == (double)a.dt || (T)c_mat.dt_consts == a.dt;
    // lane-dependent table entries hoisted out of the element loop (constant-memory
    // reads with lane-dependent indices serialise across the warp)
    int tn_own[3];
    T w_own[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) { tn_own[i] = c_tab.tn3[tidx(i, m1, m2)]; w_own[i] = (T)c_tab.w3[tidx(m1, m2, i)]; }
    const T xi = (T)c_tab.qx[m1], et = (T)c_tab.qx[m2];
    // per-phase constants in shared memory: the three elements of a warp may sit in
    // different phases, and shared-memory reads of distinct words do not serialise
    __shared__ T PT[PT_FIELDS][MAXPH];
    for (int t = threadIdx.x; t < PT_FIELDS * MAXPH; t += blockDim.x) {
        const int f = t / MAXPH, ph = t % MAXPH;
        double val = 0;
        switch (f) {
            case PT_TWOE: val = c_mat.u_twoe[ph]; break;
            case PT_TWOE_EL: val = c_mat.u_twoe_el[ph]; break;
            case PT_RHO0: val = c_mat.rho0[ph]; break;
            case PT_ALPHA: val = c_mat.alpha[ph]; break;
            case PT_BETA: val = c_mat.beta[ph]; break;
            case PT_CC: val = c_mat.u_cC[ph]; break;
            case PT_SPHI: val = c_mat.sin_phi[ph]; break;
            case PT_INVDEN: val = c_mat.u_inv_den[ph]; break;
            case PT_INVBULKDT: val = c_mat.u_inv_bulkdt[ph]; break;
            default: val = c_mat.bulk[ph]; break;
        }
        PT[f][ph] = (T)val;
    }
    __syncthreads();
    const bool bulk_inf = c_mat.all_bulk_inf != 0;
    // the incremental sweep models the FP64 problem: its ε² is FP64's
    const T EPS2 = INCR ? (T)eps2<double>() : eps2<T>();
    const bool nodal_phases = a.phv && a.phv_layout != FEMB200_PHASE_CELL;

    // work item gk is group gk, or the gk-th group of the launch's list; its first element
    // (a.nels past the end, which load_ids marks inactive)
    const int64_t gstride = (int64_t)gridDim.x * wpb;
    const int64_t ngroups = a.group_list ? a.group_count : (a.nels + 2) / 3;
    auto group_base = [&](int64_t g) -> int64_t {
        return g >= ngroups ? a.nels : a.group_list ? 3 * (int64_t)__ldg(a.group_list + g) : 3 * g;
    };
    int64_t gk = (int64_t)blockIdx.x * wpb + warp;
    int64_t base = group_base(gk);

    // prologue: ids of the first two groups, loads of the first
    GroupIds id_cur = load_ids(a, base, s, m, tn_own, lane_ok);
    GroupIds id_next = load_ids(a, group_base(gk + gstride), s, m, tn_own, lane_ok);
    T vn[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int i = 0; i < 3; ++i) vn[c][i] = T(0);
    issue_prefetch<T, INCR>(a, geo_c, id_cur, base, s, m, m1, m2, BUF, vn);
    cp_commit();
    const bool do_qp = a.do_momentum || a.phi;

    for (; gk < ngroups; gk += gstride, base = group_base(gk)) {
        cp_wait_all();
        __syncwarp();
        T v[3][3];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int i = 0; i < 3; ++i) v[c][i] = vn[c][i];
        const GroupIds id = id_cur;
        const bool act = id.act;
        const int64_t ec = act ? base + s : 0;

        const T* B = BUF + sl * SB;
        // ---- phases ----
        int p0 = id.phase;
        bool uniform = true;
        if (nodal_phases) {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int ph = act ? phase_of(a.phv, a.phv_layout, (int64_t)id.node[i] + 1, tn_own[i], ec, 27) : 0;
                if (lane_ok) PH[tidx(i, m1, m2)] = ph;
            }
            __syncwarp();
            p0 = PH[0];
            const bool same = PH[tidx(0, m1, m2)] == p0 && PH[tidx(1, m1, m2)] == p0 && PH[tidx(2, m1, m2)] == p0;
            const unsigned bal = __ballot_sync(0xffffffffu, same || !lane_ok);
            uniform = ((bal >> (s * 9)) & 0x1ffu) == 0x1ffu;
        }
        int php[4] = {0, 0, 0, 0};
        if (a.php) {
            if (a.php_layout == FEMB200_PHASE_CELL) {
                const int cp_ = act ? __ldg(a.php + ec) - 1 : 0;
#pragma unroll
                for (int p = 0; p < 4; ++p) php[p] = cp_;
            } else {
                // pressure-DoF phases of the other layouts (the DoFs of lanes 0..3)
                const int mine = (act && m < 4) ? phase_of(a.php, a.php_layout, (int64_t)id.dof + 1, m, ec, 4) : 0;
#pragma unroll
                for (int p = 0; p < 4; ++p) php[p] = __shfl_sync(0xffffffffu, mine, (lane_ok ? s * 9 : 0) + p);
            }
        }

        // ---- geometry of the element (affine: constant J⁻¹ and |det J|) ----
        T Ji[9];
#pragma unroll
        for (int r = 0; r < 9; ++r) Ji[r] = B[L::GEO + r];
        const T detJ = B[L::GEO + 9];
        const T* D = B + L::DOF;

        T g[3][3][3];
        h27_gradient<T, LY>(tb, v, E, m1, m2, g, lane_ok);

        // ---- pressure residual ----
        T rp[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
        for (int qz = 0; qz < 3; ++qz) {
            const int q = tidx(m1, m2, qz);
            const T dO = act ? detJ * w_own[qz] : T(0);
            const T ze = (T)c_tab.qx[qz];
            const T NP[4] = {T(1) - xi - et - ze, xi, et, ze};
            // physical gradient ∂v_c/∂x_k, kept in g for the momentum loop
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const T r0 = g[c][0][qz], r1 = g[c][1][qz], r2 = g[c][2][qz];
#pragma unroll
                for (int k = 0; k < 3; ++k) g[c][k][qz] = r0 * Ji[0 + 3 * k] + r1 * Ji[1 + 3 * k] + r2 * Ji[2 + 3 * k];
            }
            const T div = g[0][0][qz] + g[1][1][qz] + g[2][2][qz];
            T dPdt = T(0);
            if (!bulk_inf) {
                T dPinc = T(0);
                if (a.P_old_ip) {
#pragma unroll
                    for (int p = 0; p < 4; ++p) dPinc += NP[p] * D[p];
                    dPinc -= act ? ld(a.P_old_ip + ec * 27 + q) : T(0);
                } else {
#pragma unroll
                    for (int p = 0; p < 4; ++p) dPinc += NP[p] * (D[p] - (a.P0 ? D[4 + p] : T(0)));
                }
                if (uniform && consts_ok && php[0] == p0 && php[1] == p0 && php[2] == p0 && php[3] == p0) {
                    dPdt = dPinc * PT[PT_INVBULKDT][p0];
                } else {
                    T ebq = T(0);
#pragma unroll
                    for (int p = 0; p < 4; ++p) ebq += NP[p] * PT[PT_BULK][php[p]];
                    dPdt = dPinc / (ebq * dt);
                }
            }
            T dTdt = T(0), Qq = T(0);
            if (a.temp) {
                T aq = T(0), dT = T(0);
#pragma unroll
                for (int p = 0; p < 4; ++p) { aq += NP[p] * PT[PT_ALPHA][php[p]]; dT += NP[p] * (D[16 + p] - (a.temp0 ? D[20 + p] : T(0))); }
                dTdt = aq * dT / dt;
            }
            if (a.Q) {
#pragma unroll
                for (int p = 0; p < 4; ++p) Qq += NP[p] * D[24 + p];
            }
            const T f = (-div - dPdt + dTdt + Qq) * dO;
#pragma unroll
            for (int p = 0; p < 4; ++p) rp[p] += NP[p] * f;
        }
        // element sums of RP: lane m < 4 of each element sums component m, computes
        // its Pnum = γP·RP/M_P and shares it with the element's other lanes
        T* RPs = E + 6 * LY::K1 + 9 * LY::K2;   // after the gradient's stages
        static_assert(6 * LY::K1 + 9 * LY::K2 + 36 <= PL_STAGE, "RP scratch");
        if (lane_ok) {
#pragma unroll
            for (int p = 0; p < 4; ++p) RPs[m * 4 + p] = rp[p];
        }
        __syncwarp();
        T pn_own = T(0);
        if (m < 4) {
            T acc = T(0);
#pragma unroll
            for (int t = 0; t < 9; ++t) acc += RPs[t * 4 + m];
            if (act && a.write_RP) a.RP[id.dof] = INCR ? D[4 + m] + acc : acc;
            const T gam = a.gammaP ? D[8 + m] : T(0);
            const T mp = a.MP ? D[12 + m] : T(1);
            pn_own = a.with_pnum ? gam * acc / mp : T(0);
            if (act && a.Pnum_out && a.with_pnum) a.Pnum_out[id.dof] = pn_own;
        }
        T Pn[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) Pn[p] = __shfl_sync(0xffffffffu, pn_own, (lane_ok ? s * 9 : 0) + p);

        T beta_q[3] = {T(0), T(0), T(0)};
        if (do_qp) {
            // ---- stress and reference-frame fluxes; F overwrites g point by point ----
#pragma unroll
            for (int qz = 0; qz < 3; ++qz) {
                const int q = tidx(m1, m2, qz);
                const T dO = act ? detJ * w_own[qz] : T(0);
                const T ze = (T)c_tab.qx[qz];
                const T NP[4] = {T(1) - xi - et - ze, xi, et, ze};
                T gq[3][3];
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int k = 0; k < 3; ++k) gq[c][k] = g[c][k][qz];
                T Pq = T(0), Pfq = T(0), Pnq = T(0), Tq = T(0);
#pragma unroll
                for (int p = 0; p < 4; ++p) {
                    Pq += NP[p] * D[p];
                    Pnq += NP[p] * Pn[p];
                    if (a.Pf) Pfq += NP[p] * D[28 + p];
                    if (a.temp) Tq += NP[p] * D[16 + p];
                }
                const T Peq = a.Pf ? Pq - Pfq : Pq;
                T twoe, twoe_el, rho0, alpha, beta, cC = T(0), sphi = T(0), inv_den = T(0), etave;
                const bool fast = uniform && consts_ok && !a.eta_ip;
                if (fast) {
                    twoe = PT[PT_TWOE][p0];
                    twoe_el = PT[PT_TWOE_EL][p0];
                    etave = T(0.5) * twoe;
                    rho0 = PT[PT_RHO0][p0]; alpha = PT[PT_ALPHA][p0]; beta = PT[PT_BETA][p0];
                    if (plastic) { cC = PT[PT_CC][p0]; sphi = PT[PT_SPHI][p0]; inv_den = PT[PT_INVDEN][p0]; }
                } else {
                    T eta = T(0), invG = T(0), cphi = T(0), C = T(0), spsi = T(0), ereg = T(0), Kb = T(0);
                    rho0 = alpha = beta = T(0);
                    for (int k = 0; k < 3; ++k)
                        for (int j = 0; j < 3; ++j)
                            for (int i = 0; i < 3; ++i) {
                                const T N = tb.B[m1][i] * tb.B[m2][j] * tb.B[qz][k];
                                const int p = uniform ? p0 : PH[tidx(i, j, k)];
                                eta += N * (T)c_mat.eta[p]; invG += N * (T)c_mat.invG[p];
                                rho0 += N * (T)c_mat.rho0[p]; alpha += N * (T)c_mat.alpha[p]; beta += N * (T)c_mat.beta[p];
                                if (plastic) {
                                    cphi += N * (T)c_mat.cos_phi[p]; sphi += N * (T)c_mat.sin_phi[p];
                                    spsi += N * (T)c_mat.sin_psi[p]; C += N * (T)c_mat.C[p];
                                    ereg += N * (T)c_mat.eta_reg[p]; Kb += N * (T)c_mat.Kb[p];
                                }
                            }
                    if (a.eta_ip) eta = act ? ld(a.eta_ip + ec * 27 + q) : T(1);
                    if (!act) eta = T(1);
                    etave = T(1) / (T(1) / eta + invG / dt);
                    twoe = T(2) * etave;
                    twoe_el = twoe * (invG / (T(2) * dt));
                    cC = cphi * C;
                    inv_den = T(1) / (etave + ereg + Kb * dt * (-spsi) * (-sphi));
                }
                const T tr = (gq[0][0] + gq[1][1] + gq[2][2]) * T(1.0 / 3.0);
                const T eps_[6] = {gq[0][0] - tr, gq[1][1] - tr, gq[2][2] - tr, T(0.5) * (gq[0][1] + gq[1][0]),
                                   T(0.5) * (gq[0][2] + gq[2][0]), T(0.5) * (gq[1][2] + gq[2][1])};
                T tau[6];
            if constexpr (INCR) {
                // τ(base + δ) − τ(base): the trial stress is affine in the strain rate
                T tb[6], dtt[6];
#pragma unroll
                for (int c = 0; c < 6; ++c) { tb[c] = B[c * 27 + q]; dtt[c] = twoe * eps_[c]; }
                if (plastic) {
                    const T Fk = B[6 * 27 + q];
                    const T Jk = T(0.5) * (tb[0] * tb[0] + tb[1] * tb[1] + tb[2] * tb[2]) + tb[3] * tb[3] + tb[4] * tb[4] + tb[5] * tb[5];
                    if (Jk < T(1e-6) * cC * cC) {
                        // within 1e-3·C·cosϕ of the yield-surface apex: the return direction
                        // is ill-conditioned, so this point's increment is formed in FP64
                        double tbd[6], dtd[6], outd[6];
#pragma unroll
                        for (int c = 0; c < 6; ++c) { tbd[c] = tb[c]; dtd[c] = dtt[c]; }
                        dp_increment<double>(tbd, (double)Fk, dtd, (double)Peq, (double)twoe, (double)sphi, (double)inv_den,
                                             eps2<double>(), outd);
#pragma unroll
                        for (int c = 0; c < 6; ++c) tau[c] = (T)outd[c];
                    } else {
                        dp_increment<T>(tb, Fk, dtt, Peq, twoe, sphi, inv_den, EPS2, tau);
                    }
                } else {
#pragma unroll
                    for (int c = 0; c < 6; ++c) tau[c] = dtt[c];
                }
            } else {
                T told[6];
#pragma unroll
                for (int c = 0; c < 6; ++c) {
                    told[c] = a.told[0] ? B[c * 27 + q] : T(0);
                    tau[c] = twoe * eps_[c] + twoe_el * told[c];
                }
                if (act && a.base_out) {
#pragma unroll
                    for (int c = 0; c < 6; ++c) a.base_out[base_index(ec, q, c)] = (float)tau[c];
                }
                if (plastic) {
                    const T tII = sqrt(T(0.5) * (tau[0] * tau[0] + tau[1] * tau[1] + tau[2] * tau[2]) + tau[3] * tau[3] +
                                       tau[4] * tau[4] + tau[5] * tau[5] + EPS2);
                    const T Fy = tII - cC - sphi * Peq;
                    if (act && a.base_out) a.base_out[base_index(ec, q, 6)] = (float)Fy;
                    if (Fy > T(0)) {
                        const T lam = Fy * inv_den;
                        const T f = twoe * lam / (tII + EPS2);
                        tau[0] -= T(0.5) * f * tau[0]; tau[1] -= T(0.5) * f * tau[1]; tau[2] -= T(0.5) * f * tau[2];
                        tau[3] -= f * tau[3]; tau[4] -= f * tau[4]; tau[5] -= f * tau[5];
                    }
                }
                if (act && a.tau_store[0]) {
#pragma unroll
                    for (int c = 0; c < 6; ++c) a.tau_store[c][ec * 27 + q] = tau[c];
                }
                if (act && a.phi) {
                    const T inv2Gdt = twoe_el / twoe;
                    const T power = tau[0] * gq[0][0] + tau[1] * gq[1][1] + tau[2] * gq[2][2] + tau[3] * (gq[0][1] + gq[1][0]) +
                                    tau[4] * (gq[0][2] + gq[2][0]) + tau[5] * (gq[1][2] + gq[2][1]);
                    const T el = (tau[0] * (tau[0] - told[0]) + tau[1] * (tau[1] - told[1]) + tau[2] * (tau[2] - told[2]) +
                                  T(2) * (tau[3] * (tau[3] - told[3]) + tau[4] * (tau[4] - told[4]) + tau[5] * (tau[5] - told[5]))) *
                                 inv2Gdt;
                    a.phi[ec * 27 + q] = power - el;
                }
            }
            const T Ptot = (a.Pf ? Peq + Pfq : Pq) + Pnq;
                // EOS density (momentum_residuals.jl:11-16); its increment is ρ0·β·δP
            const T rhoq = INCR ? rho0 * beta * Pq : rho0 * (T(1) - alpha * (Tq - (T)c_mat.Tref) + beta * Pq);
                beta_q[qz] = act ? rhoq * dO : T(0);
                const T sg[3][3] = {{tau[0] - Ptot, tau[3], tau[4]}, {tau[3], tau[1] - Ptot, tau[5]}, {tau[4], tau[5], tau[2] - Ptot}};
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        g[c][d][qz] = dO * (Ji[d + 0] * sg[0][c] + Ji[d + 3] * sg[1][c] + Ji[d + 6] * sg[2][c]);
            }
        }
        // every lane is done with this group's buffer: load the next group into it
        __syncwarp();
        issue_prefetch<T, INCR>(a, geo_c, id_next, group_base(gk + gstride), s, m, m1, m2, BUF, vn);
        cp_commit();
        id_cur = id_next;
        id_next = load_ids(a, group_base(gk + 2 * gstride), s, m, tn_own, lane_ok);
        if (!a.do_momentum) continue;
        T R[3][3];
        h27_transpose<T, true, LY>(tb, g, beta_q, gvec, E, m1, m2, R, lane_ok);
        // ordered scatter: the next element's ξ = −1 node of this line, when it is this
        // element's ξ = +1 node, is added here, so a group adds to each node once
        const bool folded = a.group_list ? fold_next_element(id.node, act, s, R) : false;
        if (act) {
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    if (i > 0 || !folded) atomic_add(a.Rv[c] + id.node[i], R[c][i]);
        }
    }
    cp_wait_all();
}

// One J⁻¹ and |det J| per element when every quadrature point of the reference
// layout carries the same J⁻¹ and |det J|·ω/ω, and geo_P equals the velocity
// weights (Hex27 MixedMeshCache, src/mesh/mixed_mesh.jl:375-392).
template <class TG, class TC>
__global__ void compress_geometry_kernel(const TG* geo_v, const TG* geo_P, int64_t nels, TC* out, int* not_affine) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nels) return;
    const TG* G = geo_v + e * 270;
    const int qc = 13;
    double Jc[9], sc = 0;
    for (int r = 0; r < 9; ++r) { Jc[r] = (double)G[qc * 10 + r]; sc = fmax(sc, fabs(Jc[r])); }
    const double dc = (double)G[qc * 10 + 9] / c_tab.w3[qc];
    const double tol = sizeof(TG) == 8 ? 1e-12 : 1e-5;
    bool ok = true;
    for (int q = 0; q < 27; ++q) {
        for (int r = 0; r < 9; ++r) ok = ok && fabs((double)G[q * 10 + r] - Jc[r]) <= tol * sc;
        const double dq = (double)G[q * 10 + 9];
        ok = ok && fabs(dq / c_tab.w3[q] - dc) <= tol * fabs(dc);
        ok = ok && fabs((double)geo_P[e * 27 + q] - dq) <= tol * fabs(dq);
    }
    if (!ok) atomicOr(not_affine, 1);
    for (int r = 0; r < 9; ++r) out[e * 10 + r] = (TC)Jc[r];
    out[e * 10 + 9] = (TC)dc;
}

template <class TG, class TC>
cudaError_t launch_compress_geometry(const TG* geo_v, const TG* geo_P, int64_t nels, TC* out, int* not_affine,
                                     cudaStream_t st) {
    count_launch();
    compress_geometry_kernel<TG, TC><<<(unsigned)((nels + 127) / 128), 128, 0, st>>>(geo_v, geo_P, nels, out, not_affine);
    return cudaGetLastError();
}

template <class T, bool INCR>
size_t pipe_smem_bytes() {
    const int wpb = PipeThreads<T>::value / 32;
    return (size_t)wpb * (3 * PipeStage<T>::WORDS + 3 * pipe_buf<T, INCR>()) * sizeof(T) +
           (size_t)wpb * 3 * 28 * sizeof(int);
}

template <class T, bool INCR>
cudaError_t launch_pipe(const H27Args<T, T>& args, const T* geo_c, int num_sms, cudaStream_t st) {
    const size_t smem = pipe_smem_bytes<T, INCR>();
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(hex27_residual_pipe_kernel<T, INCR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    int per_sm = 1;
    constexpr int threads = PipeThreads<T>::value;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hex27_residual_pipe_kernel<T, INCR>, threads, smem);
    if (per_sm < 1) per_sm = 1;
    const int64_t groups = args.group_list ? args.group_count : (args.nels + 2) / 3;
    if (groups < 1) return cudaSuccess;
    int64_t blocks = (groups + threads / 32 - 1) / (threads / 32);
    const int64_t cap = (int64_t)num_sms * per_sm;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    count_launch();
    hex27_residual_pipe_kernel<T, INCR><<<(unsigned)blocks, threads, smem, st>>>(args, geo_c);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_hex27_residual_pipe(const H27Args<T, T>& args, const T* geo_c, int num_sms, cudaStream_t st) {
    return launch_pipe<T, false>(args, geo_c, num_sms, st);
}

cudaError_t launch_hex27_residual_incr(const H27Args<float, float>& args, const float* geo_c, int num_sms, cudaStream_t st) {
    return launch_pipe<float, true>(args, geo_c, num_sms, st);
}

template cudaError_t launch_hex27_residual_pipe<double>(const H27Args<double, double>&, const double*, int, cudaStream_t);
template cudaError_t launch_hex27_residual_pipe<float>(const H27Args<float, float>&, const float*, int, cudaStream_t);
template cudaError_t launch_compress_geometry<double, double>(const double*, const double*, int64_t, double*, int*, cudaStream_t);
template cudaError_t launch_compress_geometry<float, float>(const float*, const float*, int64_t, float*, int*, cudaStream_t);
template cudaError_t launch_compress_geometry<double, float>(const double*, const double*, int64_t, float*, int*, cudaStream_t);
template cudaError_t launch_compress_geometry<float, double>(const float*, const float*, int64_t, double*, int*, cudaStream_t);

}  // namespace femb
