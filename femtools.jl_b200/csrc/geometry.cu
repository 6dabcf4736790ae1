// geometry.cu — per-integration-point element geometry from the node coordinates:
// precompute_geometry_kernel! (src/mesh/mesh.jl:674-682) with the stored entry of
// _geometry_entry (mesh.jl:550-553), for Hex27 (3-D) and Q9 (2-D). Used at setup and
// by update_geometry! (mesh.jl:640-650, mixed_mesh.jl:337-345) after the nodes move.
#include <algorithm>
#include "kernels.cuh"

namespace femb {
namespace {

template <int DIM> struct GeoTabs;
template <> struct GeoTabs<3> {
    static constexpr int NV = 27;
    FEMB_D static double dN(int q, int a, int j) { return c_tab.dN3[q][a][j]; }
    FEMB_D static double w(int q) { return c_tab.w3[q]; }
};
template <> struct GeoTabs<2> {
    static constexpr int NV = 9;
    FEMB_D static double dN(int q, int a, int j) { return c_tab.dN2[q][a][j]; }
    FEMB_D static double w(int q) { return c_tab.w2[q]; }
};

// One thread per (element, integration point): J = Σ_a x_a ⊗ ∂N_a/∂ξ in FP64
// (J[i][j] = ∂x_i/∂ξ_j), the cofactor inverse and determinant, rounded once on store
// to TG. A connectivity entry outside [1, nnodes] sets *bad and the point's entries to
// NaN (no out-of-range read).
template <int DIM, class TG>
__global__ void geometry_kernel(const double* __restrict__ coords, const int32_t* __restrict__ el2n, int64_t nels,
                                int64_t nnodes, TG* geo_v, TG* geo_P, int* bad) {
    using G = GeoTabs<DIM>;
    constexpr int NV = G::NV, NQ = G::NV, NG = DIM * DIM + 1;
    const int64_t n = nels * NQ;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = idx / NQ;
        const int q = (int)(idx - e * NQ);
        double J[DIM][DIM];
#pragma unroll
        for (int i = 0; i < DIM; ++i)
#pragma unroll
            for (int j = 0; j < DIM; ++j) J[i][j] = 0.0;
        bool ok = true;
        for (int a = 0; a < NV; ++a) {
            const int64_t node = __ldg(el2n + e * NV + a);
            if (node < 1 || node > nnodes) { ok = false; break; }
            const double* x = coords + (node - 1) * DIM;
            double xa[DIM];
#pragma unroll
            for (int i = 0; i < DIM; ++i) xa[i] = __ldg(x + i);
#pragma unroll
            for (int j = 0; j < DIM; ++j) {
                const double d = G::dN(q, a, j);
#pragma unroll
                for (int i = 0; i < DIM; ++i) J[i][j] = fma(xa[i], d, J[i][j]);
            }
        }
        double inv[DIM][DIM], det;
        if constexpr (DIM == 3) {
            const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
            const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
            const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
            det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
            const double r = 1.0 / det;
            inv[0][0] = c00 * r;
            inv[1][0] = c01 * r;
            inv[2][0] = c02 * r;
            inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * r;
            inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * r;
            inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * r;
            inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * r;
            inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * r;
            inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * r;
        } else {
            det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
            const double r = 1.0 / det;
            inv[0][0] = J[1][1] * r;
            inv[0][1] = -J[0][1] * r;
            inv[1][0] = -J[1][0] * r;
            inv[1][1] = J[0][0] * r;
        }
        const double dO = fabs(det) * G::w(q);
        TG* g = geo_v + idx * NG;
        if (!ok) {
            atomicOr(bad, 1);
            for (int k = 0; k < NG; ++k) g[k] = (TG)NAN;
            if (geo_P) geo_P[idx] = (TG)NAN;
            continue;
        }
        // J⁻¹ column-major: entry (r, c) at r + DIM·c
#pragma unroll
        for (int c = 0; c < DIM; ++c)
#pragma unroll
            for (int r = 0; r < DIM; ++r) g[r + DIM * c] = (TG)inv[r][c];
        g[DIM * DIM] = (TG)dO;
        if (geo_P) geo_P[idx] = (TG)dO;
    }
}

}  // namespace

template <class TG>
cudaError_t launch_geometry(int dim, const double* coords, const int32_t* el2n, int64_t nels, int64_t nnodes, TG* geo_v,
                            TG* geo_P, int* bad, cudaStream_t st) {
    const int64_t n = nels * (dim == 3 ? 27 : 9);
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16));
    count_launch();
    if (dim == 3) geometry_kernel<3, TG><<<(unsigned)blocks, 256, 0, st>>>(coords, el2n, nels, nnodes, geo_v, geo_P, bad);
    else geometry_kernel<2, TG><<<(unsigned)blocks, 256, 0, st>>>(coords, el2n, nels, nnodes, geo_v, geo_P, bad);
    return cudaGetLastError();
}
template cudaError_t launch_geometry<double>(int, const double*, const int32_t*, int64_t, int64_t, double*, double*,
                                             int*, cudaStream_t);
template cudaError_t launch_geometry<float>(int, const double*, const int32_t*, int64_t, int64_t, float*, float*, int*,
                                            cudaStream_t);

}  // namespace femb
