// postprocess.cu — element-averaged strain-rate and deviatoric-stress diagnostics
// (compute_strain_rate_stress_postprocess, src/postprocess/postprocess.jl:17-79 in 2-D
// and :168-215 in 3-D, from integration-point stresses): every field is integrated
// against dΩ over the element and divided by the element volume. One thread per
// element; the element's velocities stay in registers, the geometry is read once.
#include <algorithm>
#include "kernels.cuh"

namespace femb {
namespace {

template <int DIM> struct PpTabs;
template <> struct PpTabs<3> {
    static constexpr int NV = 27, NF = 14;
    FEMB_D static double dN(int q, int a, int j) { return c_tab.dN3[q][a][j]; }
};
template <> struct PpTabs<2> {
    static constexpr int NV = 9, NF = 10;
    FEMB_D static double dN(int q, int a, int j) { return c_tab.dN2[q][a][j]; }
};

// Output order (3-D): εxx, εyy, εzz, εxy, εxz, εyz, εII, τxx, τyy, τzz, τxy, τxz, τyz, τII;
// (2-D): εxx, εyy, εzz, εxy, εII, τxx, τyy, τzz, τxy, τII.
template <int DIM, class T, class TG>
__global__ void strain_rate_stress_kernel(PostArgs<T, TG> a) {
    using P = PpTabs<DIM>;
    constexpr int NV = P::NV, NQ = P::NV, NG = DIM * DIM + 1;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < a.nels; e += (int64_t)gridDim.x * blockDim.x) {
        T vl[DIM][NV];
#pragma unroll
        for (int n = 0; n < NV; ++n) {
            const int64_t node = __ldg(a.el2n + e * NV + n) - 1;
#pragma unroll
            for (int c = 0; c < DIM; ++c) vl[c][n] = a.v[c][node];
        }
        T tot[P::NF];
#pragma unroll
        for (int f = 0; f < P::NF; ++f) tot[f] = T(0);
        T vol = T(0);
        for (int q = 0; q < NQ; ++q) {
            const TG* g = a.geo_v + (e * NQ + q) * NG;
            // reference gradient gr[c][j] = Σ_a v_c(a) ∂N_a/∂ξ_j, then ∂v_c/∂x_k = Σ_j gr[c][j] J⁻¹[j][k]
            T gr[DIM][DIM];
#pragma unroll
            for (int c = 0; c < DIM; ++c)
#pragma unroll
                for (int j = 0; j < DIM; ++j) gr[c][j] = T(0);
#pragma unroll
            for (int n = 0; n < NV; ++n)
#pragma unroll
                for (int j = 0; j < DIM; ++j) {
                    const T d = (T)P::dN(q, n, j);
#pragma unroll
                    for (int c = 0; c < DIM; ++c) gr[c][j] += vl[c][n] * d;
                }
            T gv[DIM][DIM];
#pragma unroll
            for (int c = 0; c < DIM; ++c)
#pragma unroll
                for (int k = 0; k < DIM; ++k) {
                    T s = T(0);
#pragma unroll
                    for (int j = 0; j < DIM; ++j) s += gr[c][j] * (T)g[j + DIM * k];
                    gv[c][k] = s;
                }
            const T dO = (T)g[DIM * DIM];
            const int64_t iq = e * NQ + q;
            T f[P::NF];
            if constexpr (DIM == 3) {
                const T ex = gv[0][0], ey = gv[1][1], ez = gv[2][2];
                const T exy = (gv[0][1] + gv[1][0]) / T(2), exz = (gv[0][2] + gv[2][0]) / T(2),
                        eyz = (gv[1][2] + gv[2][1]) / T(2);
                const T tr = (ex + ey + ez) / T(3);
                const T dx = ex - tr, dy = ey - tr, dz = ez - tr;
                // second_invariant of a 6-tuple with the eps² floor (rheology.jl:395-400)
                const T eII = sqrt((dx * dx + dy * dy + dz * dz) / T(2) + exy * exy + exz * exz + eyz * eyz + eps2<T>());
                T t[6];
#pragma unroll
                for (int c = 0; c < 6; ++c) t[c] = a.tau[c][iq];
                const T tII = sqrt((t[0] * t[0] + t[1] * t[1] + t[2] * t[2]) / T(2) + t[3] * t[3] + t[4] * t[4] +
                                   t[5] * t[5] + eps2<T>());
                f[0] = ex; f[1] = ey; f[2] = ez; f[3] = exy; f[4] = exz; f[5] = eyz; f[6] = eII;
#pragma unroll
                for (int c = 0; c < 6; ++c) f[7 + c] = t[c];
                f[13] = tII;
            } else {
                const T ex = gv[0][0], ey = gv[1][1], ez = T(0), exy = (gv[0][1] + gv[1][0]) / T(2);
                const T tr = (ex + ey + ez) / T(3);
                const T dx = ex - tr, dy = ey - tr, dz = ez - tr;
                const T eII = sqrt((dx * dx + dy * dy + dz * dz) / T(2) + exy * exy);
                const T txx = a.tau[0][iq], tyy = a.tau[1][iq], txy = a.tau[2][iq];
                const T tzz = -(txx + tyy);
                const T tII = sqrt((txx * txx + tyy * tyy + tzz * tzz) / T(2) + txy * txy);
                f[0] = ex; f[1] = ey; f[2] = ez; f[3] = exy; f[4] = eII;
                f[5] = txx; f[6] = tyy; f[7] = tzz; f[8] = txy; f[9] = tII;
            }
#pragma unroll
            for (int k = 0; k < P::NF; ++k) tot[k] += f[k] * dO;
            vol += dO;
        }
#pragma unroll
        for (int k = 0; k < P::NF; ++k) a.out[k][e] = tot[k] / vol;
    }
}

}  // namespace

template <class T, class TG>
cudaError_t launch_strain_rate_stress(int dim, const PostArgs<T, TG>& a, cudaStream_t st) {
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((a.nels + 127) / 128, 148 * 16));
    count_launch();
    if (dim == 3) strain_rate_stress_kernel<3, T, TG><<<(unsigned)blocks, 128, 0, st>>>(a);
    else strain_rate_stress_kernel<2, T, TG><<<(unsigned)blocks, 128, 0, st>>>(a);
    return cudaGetLastError();
}
template cudaError_t launch_strain_rate_stress<double, double>(int, const PostArgs<double, double>&, cudaStream_t);
template cudaError_t launch_strain_rate_stress<double, float>(int, const PostArgs<double, float>&, cudaStream_t);
template cudaError_t launch_strain_rate_stress<float, float>(int, const PostArgs<float, float>&, cudaStream_t);
template cudaError_t launch_strain_rate_stress<float, double>(int, const PostArgs<float, double>&, cudaStream_t);

}  // namespace femb
