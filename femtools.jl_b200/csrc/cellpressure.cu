// cellpressure.cu — the viscous Hex27 Stokes operator with four cell-local pressure
// modes (1, ξ, η, ζ) (CellPressureStokesDR): preconditioner and pressure mass
// (stokes_preconditioner_3d!, src/stokes/assemblers/momentum_residuals.jl:703-745),
// pressure residual (assemble_stokes_pressure_residual_3d!, pressure_residual.jl:330-364),
// momentum residual (assemble_stokes_momentum_residual_3d!, momentum_residuals.jl:644-700)
// and the node/cell updates of the Arrow–Hurwicz relaxation (DR.jl:1004-1057).
//
// The residuals, evaluated every iteration, use the sum-factorised line-thread stages
// of the StokesDR sweeps (three elements per warp). The preconditioner, once per solve,
// is one warp per element: lane a < 27 owns node a and lane q < 27 point q, with the
// Hex27 tables staged once per block in shared memory because the lanes index them by
// their own point or node.
#include <algorithm>
#include "kernels.cuh"
#include "hex27.cuh"

namespace femb {
namespace {

constexpr int CP_WARPS = 4;
constexpr int CP_THREADS = CP_WARPS * 32;
constexpr int CPS_THREADS = 128;   // sum-factorised residuals: 4 warps × 3 elements

struct CpTabs {
    double dN[27][27][3];   // ∂N_a/∂ξ_j at q
    double N[27][27];       // N_a at q
    double sumN[27];
    double x[27][3];        // reference coordinates of q (the pressure modes ξ, η, ζ)
};

FEMB_D void stage_tables(CpTabs& T) {
    for (int i = threadIdx.x; i < 27 * 27 * 3; i += blockDim.x) (&T.dN[0][0][0])[i] = (&c_tab.dN3[0][0][0])[i];
    for (int i = threadIdx.x; i < 27 * 27; i += blockDim.x) (&T.N[0][0])[i] = (&c_tab.N3[0][0])[i];
    for (int q = threadIdx.x; q < 27; q += blockDim.x) {
        T.sumN[q] = c_tab.sumN3[q];
        T.x[q][0] = c_tab.qx[q % 3];
        T.x[q][1] = c_tab.qx[(q / 3) % 3];
        T.x[q][2] = c_tab.qx[q / 9];
    }
    __syncthreads();
}

FEMB_D double warp_sum_d(double x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// Sum-factorised residuals (the line-thread stages of hex27.cuh): a warp holds three
// elements, nine lanes per element, each owning one tensor line of the 3×3×3 node and
// point grids. PRES: RP(m, e) = −Σ_q mode_m ∇·v dΩ, reduced over the element's lanes
// through shared memory; MOM: the viscous stress 2ηε̇′ − P·I and the body force −ρg at
// the owned points, pushed back to the nodes by the transposed contraction and
// scattered with FP64 atomics.
// AFF: every cell is affine and a.geo_c holds one J⁻¹ and |det J| per cell (dΩ_q =
// |det J|·ω_q), read once per element instead of at every point.
template <bool MOM, bool AFF>
__global__ void __launch_bounds__(CPS_THREADS, AFF ? 3 : 2) cp_residual_sf_kernel(const CpArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const bool lane_ok = lane < 27;
    // lanes 27..31 carry no element; they work in a private scratch slot (3) on the line
    // the bank-conflict-free stage layout leaves them
    using LY = H27Fp64Banked;
    const int s = lane_ok ? lane / 9 : 3, m = lane_ok ? lane % 9 : LY::IDLE_M, m1 = m % 3, m2 = m / 3;
    double* E = reinterpret_cast<double*>(smem_raw) + ((size_t)warp * 4 + s) * LY::SLOT;
    Tab1D<double> tb; tb.load();
    const double gvec[3] = {a.g[0], a.g[1], a.g[2]};
    const double xi = c_tab.qx[m1], et = c_tab.qx[m2];
    const int64_t stride = (int64_t)gridDim.x * wpb * 3;
    for (int64_t base = ((int64_t)blockIdx.x * wpb + warp) * 3; base < a.nels; base += stride) {
        const int64_t e = base + (lane_ok ? s : 0);
        const bool act = lane_ok && e < a.nels;
        const int64_t ec = act ? e : 0;
        int node[3];
        double v[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            node[i] = act ? __ldg(a.el2n + 27 * ec + c_tab.tn3[tidx(i, m1, m2)]) - 1 : 0;
#pragma unroll
            for (int c = 0; c < 3; ++c) v[c][i] = act ? a.v[c][node[i]] : 0.0;
        }
        double g[3][3][3];
        h27_gradient<double, LY>(tb, v, E, m1, m2, g);
        if constexpr (!MOM) {
            double rp[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int qz = 0; qz < 3; ++qz) {
                const int q = tidx(m1, m2, qz);
                const double* G = AFF ? a.geo_c + ec * 10 : a.geo_v + (ec * 27 + q) * 10;
                double div = 0.0;
#pragma unroll
                for (int c = 0; c < 3; ++c) div += g[c][0][qz] * __ldg(G + 3 * c) + g[c][1][qz] * __ldg(G + 1 + 3 * c) +
                                                   g[c][2][qz] * __ldg(G + 2 + 3 * c);
                const double dOq = AFF ? __ldg(G + 9) * c_tab.w3[q] : __ldg(G + 9);
                const double f = act ? -div * dOq : 0.0;
                const double ze = c_tab.qx[qz];
                rp[0] += f; rp[1] += xi * f; rp[2] += et * f; rp[3] += ze * f;
            }
            double* RPs = E + 6 * LY::K1 + 9 * LY::K2;   // after the gradient's stages
            static_assert(6 * LY::K1 + 9 * LY::K2 + 36 <= LY::SLOT, "mode reduction scratch");
#pragma unroll
            for (int p = 0; p < 4; ++p) RPs[m * 4 + p] = rp[p];
            __syncwarp();
            if (act && m < 4) {
                double acc = 0.0;
#pragma unroll
                for (int t = 0; t < 9; ++t) acc += RPs[t * 4 + m];
                a.RP[4 * e + m] = acc;
            }
            __syncwarp();
        } else {
            const int ph = act ? __ldg(a.phases + ec) - 1 : 0;
            double Pl[4];
#pragma unroll
            for (int p = 0; p < 4; ++p) Pl[p] = act ? a.P[4 * ec + p] : 0.0;
            double F[3][3][3], beta_q[3];
#pragma unroll
            for (int qz = 0; qz < 3; ++qz) {
                const int q = tidx(m1, m2, qz);
                const double* G = AFF ? a.geo_c + ec * 10 : a.geo_v + (ec * 27 + q) * 10;
                double Ji[9];
#pragma unroll
                for (int r = 0; r < 9; ++r) Ji[r] = act ? __ldg(G + r) : 0.0;
                const double dO = act ? (AFF ? __ldg(G + 9) * c_tab.w3[q] : __ldg(G + 9)) : 0.0;
                double gq[3][3];
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int k = 0; k < 3; ++k)
                        gq[c][k] = g[c][0][qz] * Ji[3 * k] + g[c][1][qz] * Ji[1 + 3 * k] + g[c][2][qz] * Ji[2 + 3 * k];
                // η and ρ interpolated over the cell's single phase (interp2ip_phase)
                const double sN = c_tab.sumN3[q];
                const double eta_q = a.eta[ph] * sN;
                const double tr = (gq[0][0] + gq[1][1] + gq[2][2]) / 3.0;
                const double Pq = Pl[0] + Pl[1] * xi + Pl[2] * et + Pl[3] * c_tab.qx[qz];
                double sg[3][3];
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j)
                        sg[i][j] = 2.0 * eta_q * (0.5 * (gq[i][j] + gq[j][i]) - (i == j ? tr : 0.0)) - (i == j ? Pq : 0.0);
                beta_q[qz] = a.rho[ph] * sN * dO;
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int d = 0; d < 3; ++d) F[c][d][qz] = dO * (Ji[d] * sg[0][c] + Ji[d + 3] * sg[1][c] + Ji[d + 6] * sg[2][c]);
            }
            double R[3][3];
            h27_transpose<double, true, LY>(tb, F, beta_q, gvec, E, m1, m2, R);
            if (act) {
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int i = 0; i < 3; ++i) atomicAdd(a.Rv[c] + node[i], R[c][i]);
            }
        }
    }
}

__global__ void __launch_bounds__(CP_THREADS) cp_preconditioner_kernel(const CpArgs a) {
    __shared__ CpTabs T;
    stage_tables(T);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int64_t e = (int64_t)blockIdx.x * CP_WARPS + w; e < a.nels; e += (int64_t)gridDim.x * CP_WARPS) {
        const int ph = __ldg(a.phases + e) - 1;
        const double eta = a.eta[ph];
        double m[4] = {0, 0, 0, 0};
        if (lane < 27) {
            const int an = lane;
            const int node = __ldg(a.el2n + e * 27 + an) - 1;
            double dg[3] = {0, 0, 0};
            for (int q = 0; q < 27; ++q) {
                const double* g = a.geo_v + (e * 27 + q) * 10;
                double gN[3];
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    gN[k] = T.dN[q][an][0] * __ldg(g + 3 * k) + T.dN[q][an][1] * __ldg(g + 1 + 3 * k) +
                            T.dN[q][an][2] * __ldg(g + 2 + 3 * k);
                const double dO = __ldg(g + 9);
                const double n2 = gN[0] * gN[0] + gN[1] * gN[1] + gN[2] * gN[2];
#pragma unroll
                for (int c = 0; c < 3; ++c) dg[c] += eta * (n2 + gN[c] * gN[c] / 3.0) * dO;
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) atomicAdd(a.diagonal[c] + node, dg[c]);
            // pressure mass: lane = point
            const int q = lane;
            const double dO = __ldg(a.geo_v + (e * 27 + q) * 10 + 9);
            m[0] = dO;
            m[1] = T.x[q][0] * T.x[q][0] * dO;
            m[2] = T.x[q][1] * T.x[q][1] * dO;
            m[3] = T.x[q][2] * T.x[q][2] * dO;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) m[k] = warp_sum_d(m[k]);
        if (lane < 4) a.pressure_mass[4 * e + lane] = lane == 0 ? m[0] : lane == 1 ? m[1] : lane == 2 ? m[2] : m[3];
    }
}

// P += step·RP/M over 4·nels entries; block partials of Σ P(1,e)·M(1,e) and Σ M(1,e)
// (after the update) into partials[2·block + {0, 1}].
__global__ void __launch_bounds__(256) cp_pressure_update_kernel(double* P, const double* RP, const double* M,
                                                                 int64_t nels, double step, double* partials) {
    __shared__ double red[8][2];
    double s0 = 0, s1 = 0;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nels; e += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const int64_t i = 4 * e + m;
            const double p = P[i] + step * RP[i] / M[i];
            P[i] = p;
            if (m == 0) { s0 += p * M[i]; s1 += M[i]; }
        }
    }
    s0 = warp_sum_d(s0);
    s1 = warp_sum_d(s1);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { red[w][0] = s0; red[w][1] = s1; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0, t1 = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { t0 += red[k][0]; t1 += red[k][1]; }
        partials[2 * blockIdx.x] = t0;
        partials[2 * blockIdx.x + 1] = t1;
    }
}

// P(1, e) −= Σ P·M / Σ M, every block reducing the nb partials in the same order.
__global__ void __launch_bounds__(256) cp_pressure_mean_kernel(double* P, int64_t nels, const double* partials, int nb) {
    __shared__ double red[8][2];
    __shared__ double mean;
    // every block reduces the partials itself (in a fixed order), all threads at once
    double t0 = 0, t1 = 0;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) { t0 += partials[2 * k]; t1 += partials[2 * k + 1]; }
    t0 = warp_sum_d(t0);
    t1 = warp_sum_d(t1);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { red[w][0] = t0; red[w][1] = t1; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0, s1 = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { s0 += red[k][0]; s1 += red[k][1]; }
        mean = s0 / s1;
    }
    __syncthreads();
    const double pm = mean;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nels; e += (int64_t)gridDim.x * blockDim.x)
        P[4 * e] -= pm;
}

__global__ void cp_velocity_step_kernel(const CpVelArgs a) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
        const unsigned m = a.mask[i];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double r = a.Rv[c][i];
            if (a.load[c]) r -= __ldg(a.load[c] + i);
            if ((m >> c) & 1u) r = 0.0;
            else a.v[c][i] -= a.step * r / __ldg(a.diag[c] + i);
            a.Rv[c][i] = a.zero ? 0.0 : r;
        }
    }
}

// Connectivity in 1..nnodes and phases in 1..nphases, before any kernel gathers by them.
__global__ void cp_validate_kernel(const int32_t* el2n, const int32_t* phases, int64_t nels, int64_t nnodes, int nphases,
                                   int* bad) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nels * 27; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t n = el2n[i];
        if (n < 1 || n > nnodes) atomicOr(bad, 1);
        if (i % 27 == 0) {
            const int32_t ph = phases[i / 27];
            if (ph < 1 || ph > nphases) atomicOr(bad, 2);
        }
    }
}

inline unsigned grid_for(int64_t n, int t, int cap) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + t - 1) / t, cap));
}

}  // namespace

namespace {
size_t cps_smem() { return (size_t)(CPS_THREADS / 32) * 4 * H27Fp64Banked::SLOT * sizeof(double); }

template <bool MOM, bool AFF>
cudaError_t launch_cp_sf(const CpArgs& a, int num_sms, cudaStream_t st) {
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(cp_residual_sf_kernel<MOM, AFF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)cps_smem());
        if (e != cudaSuccess) return e;
        configured = true;
    }
    const int wpb = CPS_THREADS / 32;
    const int64_t groups = (a.nels + 2) / 3;
    const unsigned blocks = grid_for(groups, wpb, num_sms * 16);
    count_launch();
    cp_residual_sf_kernel<MOM, AFF><<<blocks, CPS_THREADS, cps_smem(), st>>>(a);
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_cp_pressure_residual(const CpArgs& a, int num_sms, cudaStream_t st) {
    return a.geo_c ? launch_cp_sf<false, true>(a, num_sms, st) : launch_cp_sf<false, false>(a, num_sms, st);
}

cudaError_t launch_cp_momentum_residual(const CpArgs& a, int num_sms, cudaStream_t st) {
    return a.geo_c ? launch_cp_sf<true, true>(a, num_sms, st) : launch_cp_sf<true, false>(a, num_sms, st);
}

namespace {
// One J⁻¹ and |det J| = dΩ_q/ω_q per cell from its centre point; *not_affine is set when
// any point of a cell differs from them by more than 1e-12 of their scale.
__global__ void cp_compress_geometry_kernel(const double* geo_v, int64_t nels, double* out, int* not_affine) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nels) return;
    const double* G = geo_v + e * 270;
    double Jc[9], sc = 0;
    for (int r = 0; r < 9; ++r) { Jc[r] = G[13 * 10 + r]; sc = fmax(sc, fabs(Jc[r])); }
    const double dc = G[13 * 10 + 9] / c_tab.w3[13];
    bool ok = true;
    for (int q = 0; q < 27; ++q) {
        for (int r = 0; r < 9; ++r) ok = ok && fabs(G[q * 10 + r] - Jc[r]) <= 1e-12 * sc;
        ok = ok && fabs(G[q * 10 + 9] / c_tab.w3[q] - dc) <= 1e-12 * fabs(dc);
    }
    if (!ok) atomicOr(not_affine, 1);
    for (int r = 0; r < 9; ++r) out[e * 10 + r] = Jc[r];
    out[e * 10 + 9] = dc;
}
}  // namespace

cudaError_t launch_cp_compress_geometry(const double* geo_v, int64_t nels, double* out, int* not_affine, cudaStream_t st) {
    count_launch();
    cp_compress_geometry_kernel<<<grid_for(nels, 128, 1 << 30), 128, 0, st>>>(geo_v, nels, out, not_affine);
    return cudaGetLastError();
}

cudaError_t launch_cp_preconditioner(const CpArgs& a, int num_sms, cudaStream_t st) {
    count_launch();
    cp_preconditioner_kernel<<<grid_for(a.nels, CP_WARPS, num_sms * 8), CP_THREADS, 0, st>>>(a);
    return cudaGetLastError();
}

int cp_mean_blocks(int num_sms) { return num_sms * 2; }

cudaError_t launch_cp_validate(const int32_t* el2n, const int32_t* phases, int64_t nels, int64_t nnodes, int nphases,
                               int* bad, cudaStream_t st) {
    count_launch();
    cp_validate_kernel<<<grid_for(nels * 27, 256, 148 * 8), 256, 0, st>>>(el2n, phases, nels, nnodes, nphases, bad);
    return cudaGetLastError();
}

cudaError_t launch_cp_pressure_update(double* P, const double* RP, const double* M, int64_t nels, double step,
                                      double* partials, int nb, cudaStream_t st) {
    count_launch();
    cp_pressure_update_kernel<<<nb, 256, 0, st>>>(P, RP, M, nels, step, partials);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    count_launch();
    cp_pressure_mean_kernel<<<grid_for(nels, 256, 148 * 4), 256, 0, st>>>(P, nels, partials, nb);
    return cudaGetLastError();
}

cudaError_t launch_cp_velocity_step(const CpVelArgs& a, cudaStream_t st) {
    count_launch();
    cp_velocity_step_kernel<<<grid_for(a.n, 256, 148 * 8), 256, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace femb
