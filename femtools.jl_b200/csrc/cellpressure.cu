// cellpressure.cu — the viscous Hex27 Stokes operator with four cell-local pressure
// modes (1, ξ, η, ζ) (CellPressureStokesDR): preconditioner and pressure mass
// (stokes_preconditioner_3d!, src/stokes/assemblers/momentum_residuals.jl:703-745),
// pressure residual (assemble_stokes_pressure_residual_3d!, pressure_residual.jl:330-364),
// momentum residual (assemble_stokes_momentum_residual_3d!, momentum_residuals.jl:644-700)
// and the node/cell updates of the Arrow–Hurwicz relaxation (DR.jl:1004-1057).
//
// One warp per element: lane q < 27 evaluates integration point q, lane a < 27 owns node
// a, and the element's velocities and per-point fluxes pass through the warp's shared
// memory. The Hex27 tables are staged once per block in shared memory, because the
// lanes index them by their own point or node.
#include <algorithm>
#include "kernels.cuh"

namespace femb {
namespace {

constexpr int CP_WARPS = 4;
constexpr int CP_THREADS = CP_WARPS * 32;

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

// Velocity gradient ∂v_c/∂x_k at point q from the element's staged velocities V[c·27 + a].
FEMB_D void grad_at(const CpTabs& T, const double* V, int q, const double* Ji, double gv[3][3]) {
    double gr[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int a = 0; a < 27; ++a) {
        const double d0 = T.dN[q][a][0], d1 = T.dN[q][a][1], d2 = T.dN[q][a][2];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double va = V[c * 27 + a];
            gr[c][0] = fma(va, d0, gr[c][0]);
            gr[c][1] = fma(va, d1, gr[c][1]);
            gr[c][2] = fma(va, d2, gr[c][2]);
        }
    }
    // ∂v_c/∂x_k = Σ_j gr[c][j] J⁻¹[j][k], J⁻¹ column-major: (j, k) at j + 3k
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int k = 0; k < 3; ++k) gv[c][k] = gr[c][0] * Ji[3 * k] + gr[c][1] * Ji[1 + 3 * k] + gr[c][2] * Ji[2 + 3 * k];
}

FEMB_D void stage_velocity(const CpArgs& a, int64_t e, int lane, double* V, int& node) {
    node = lane < 27 ? __ldg(a.el2n + e * 27 + lane) - 1 : 0;
    if (lane < 27) {
#pragma unroll
        for (int c = 0; c < 3; ++c) V[c * 27 + lane] = a.v[c][node];
    }
    __syncwarp();
}

__global__ void __launch_bounds__(CP_THREADS) cp_pressure_residual_kernel(const CpArgs a) {
    __shared__ CpTabs T;
    __shared__ double Vs[CP_WARPS][81];
    stage_tables(T);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int64_t e = (int64_t)blockIdx.x * CP_WARPS + w; e < a.nels; e += (int64_t)gridDim.x * CP_WARPS) {
        int node;
        stage_velocity(a, e, lane, Vs[w], node);
        double r[4] = {0, 0, 0, 0};
        if (lane < 27) {
            const int q = lane;
            const double* g = a.geo_v + (e * 27 + q) * 10;
            double Ji[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) Ji[i] = __ldg(g + i);
            double gv[3][3];
            grad_at(T, Vs[w], q, Ji, gv);
            const double f = (gv[0][0] + gv[1][1] + gv[2][2]) * __ldg(g + 9);
            r[0] = f; r[1] = T.x[q][0] * f; r[2] = T.x[q][1] * f; r[3] = T.x[q][2] * f;
        }
#pragma unroll
        for (int m = 0; m < 4; ++m) r[m] = warp_sum_d(r[m]);
        if (lane < 4) a.RP[4 * e + lane] = -(lane == 0 ? r[0] : lane == 1 ? r[1] : lane == 2 ? r[2] : r[3]);
        __syncwarp();
    }
}

__global__ void __launch_bounds__(CP_THREADS) cp_momentum_residual_kernel(const CpArgs a) {
    __shared__ CpTabs T;
    __shared__ double Vs[CP_WARPS][81];
    __shared__ double Fs[CP_WARPS][27][10];
    stage_tables(T);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int64_t e = (int64_t)blockIdx.x * CP_WARPS + w; e < a.nels; e += (int64_t)gridDim.x * CP_WARPS) {
        int node;
        stage_velocity(a, e, lane, Vs[w], node);
        const int ph = __ldg(a.phases + e) - 1;
        if (lane < 27) {
            const int q = lane;
            const double* g = a.geo_v + (e * 27 + q) * 10;
            double Ji[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) Ji[i] = __ldg(g + i);
            const double dO = __ldg(g + 9);
            double gv[3][3];
            grad_at(T, Vs[w], q, Ji, gv);
            // deviatoric strain rate and the viscous stress 2ηε̇′ (η interpolated over the cell)
            const double tr = (gv[0][0] + gv[1][1] + gv[2][2]) / 3.0;
            const double eta_q = a.eta[ph] * T.sumN[q];
            double s[3][3];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) s[i][j] = 2.0 * eta_q * (0.5 * (gv[i][j] + gv[j][i]) - (i == j ? tr : 0.0));
            const double* P = a.P + 4 * e;
            const double Pq = P[0] + P[1] * T.x[q][0] + P[2] * T.x[q][1] + P[3] * T.x[q][2];
#pragma unroll
            for (int i = 0; i < 3; ++i) s[i][i] -= Pq;
            // reference-frame flux F[c][d] = dΩ Σ_k J⁻¹[d][k] σ[k][c]
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    Fs[w][q][c * 3 + d] = dO * (Ji[d] * s[0][c] + Ji[d + 3] * s[1][c] + Ji[d + 6] * s[2][c]);
            Fs[w][q][9] = a.rho[ph] * T.sumN[q] * dO;
        }
        __syncwarp();
        if (lane < 27) {
            const int an = lane;
            double R[3] = {0, 0, 0}, B = 0;
            for (int q = 0; q < 27; ++q) {
                const double d0 = T.dN[q][an][0], d1 = T.dN[q][an][1], d2 = T.dN[q][an][2];
                const double* F = Fs[w][q];
#pragma unroll
                for (int c = 0; c < 3; ++c) R[c] += d0 * F[c * 3] + d1 * F[c * 3 + 1] + d2 * F[c * 3 + 2];
                B += T.N[q][an] * F[9];
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) atomicAdd(a.Rv[c] + node, R[c] - a.g[c] * B);
        }
        __syncwarp();
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
    __shared__ double mean;
    if (threadIdx.x == 0) {
        double t0 = 0, t1 = 0;
        for (int k = 0; k < nb; ++k) { t0 += partials[2 * k]; t1 += partials[2 * k + 1]; }
        mean = t0 / t1;
    }
    __syncthreads();
    const double pm = mean;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nels; e += (int64_t)gridDim.x * blockDim.x)
        P[4 * e] -= pm;
}

__global__ void cp_velocity_update_kernel(double* v, const double* R, const double* diag, int64_t n, double step) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v[i] -= step * R[i] / diag[i];
}

__global__ void cp_subtract_kernel(double* R, const double* load, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        R[i] -= load[i];
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

cudaError_t launch_cp_pressure_residual(const CpArgs& a, int num_sms, cudaStream_t st) {
    count_launch();
    cp_pressure_residual_kernel<<<grid_for(a.nels, CP_WARPS, num_sms * 8), CP_THREADS, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_cp_momentum_residual(const CpArgs& a, int num_sms, cudaStream_t st) {
    count_launch();
    cp_momentum_residual_kernel<<<grid_for(a.nels, CP_WARPS, num_sms * 8), CP_THREADS, 0, st>>>(a);
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

cudaError_t launch_cp_velocity_update(double* v, const double* R, const double* diag, int64_t n, double step,
                                      cudaStream_t st) {
    count_launch();
    cp_velocity_update_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(v, R, diag, n, step);
    return cudaGetLastError();
}

cudaError_t launch_cp_subtract(double* R, const double* load, int64_t n, cudaStream_t st) {
    count_launch();
    cp_subtract_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(R, load, n);
    return cudaGetLastError();
}

}  // namespace femb
