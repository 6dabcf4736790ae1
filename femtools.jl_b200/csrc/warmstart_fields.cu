// warmstart_fields.cu — the learned warm start's view of a structured 2-D Q9/P1-disc
// state: converged fields on the (2n+1)² node grid (vx, vy, P evaluated from the
// element's linear pressure, ε̇II by central differences), the network input of two
// consecutive steps, the training target (the next step's correction to linear
// extrapolation) and the initial guess the solver starts from. No reference
// counterpart (the reference has no learned component).
#include <cuda_bf16.h>
#include <algorithm>
#include "kernels.cuh"

namespace femb {
namespace {

inline unsigned blk(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16)); }

template <class T>
__global__ void grid_fields_kernel(const T* __restrict__ vx, const T* __restrict__ vy, const T* __restrict__ P,
                                   const int32_t* __restrict__ dofsP, const int32_t* __restrict__ node_elem,
                                   const int8_t* __restrict__ node_xi, const int8_t* __restrict__ node_eta, int nx,
                                   int ny, float dx, float dy, float* out) {
    const int64_t n = (int64_t)nx * ny;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int ix = (int)(i % nx), iy = (int)(i / nx);
        const int e = node_elem[i];
        const float xi = node_xi[i], et = node_eta[i];
        const float P0 = (float)P[dofsP[3 * e] - 1], P1 = (float)P[dofsP[3 * e + 1] - 1], P2 = (float)P[dofsP[3 * e + 2] - 1];
        const int xl = max(ix - 1, 0), xr = min(ix + 1, nx - 1), yl = max(iy - 1, 0), yr = min(iy + 1, ny - 1);
        const float ddx = dx * (float)(xr - xl), ddy = dy * (float)(yr - yl);
        const float dvxdx = (float)(vx[(int64_t)iy * nx + xr] - vx[(int64_t)iy * nx + xl]) / ddx;
        const float dvydx = (float)(vy[(int64_t)iy * nx + xr] - vy[(int64_t)iy * nx + xl]) / ddx;
        const float dvxdy = (float)(vx[(int64_t)yr * nx + ix] - vx[(int64_t)yl * nx + ix]) / ddy;
        const float dvydy = (float)(vy[(int64_t)yr * nx + ix] - vy[(int64_t)yl * nx + ix]) / ddy;
        // plane-strain deviatoric strain rate and its second invariant
        const float tr = (dvxdx + dvydy) / 3.0f;
        const float exx = dvxdx - tr, eyy = dvydy - tr, ezz = -tr, exy = 0.5f * (dvxdy + dvydx);
        out[4 * i + 0] = (float)vx[i];
        out[4 * i + 1] = (float)vy[i];
        out[4 * i + 2] = P0 * (1.0f - xi - et) + P1 * xi + P2 * et;
        out[4 * i + 3] = sqrtf(0.5f * (exx * exx + eyy * eyy + ezz * ezz) + exy * exy);
    }
}

// X[p][c] = F_cur[p][c]/s[c] (c < 4), (F_cur − F_prev)[p][c−4]/s[c] (4 ≤ c < 8), 0 (8 ≤ c < 16)
__global__ void net_input_kernel(const float* __restrict__ Fp, const float* __restrict__ Fc, const float* __restrict__ s,
                                 __nv_bfloat16* X, int64_t npix) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npix * 16; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = i / 16;
        const int c = (int)(i % 16);
        float v = 0.0f;
        if (c < 4) v = Fc[4 * p + c] / s[c];
        else if (c < 8) v = (Fc[4 * p + c - 4] - Fp[4 * p + c - 4]) / s[c];
        X[i] = __float2bfloat16(v);
    }
}

// target[p][c] = (F_next − (2 F_cur − F_prev))[p][c] / s[c], c = vx, vy, P
__global__ void net_target_kernel(const float* __restrict__ Fp, const float* __restrict__ Fc, const float* __restrict__ Fn,
                                  const float* __restrict__ s, float* tgt, int64_t npix) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npix * 3; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = i / 3;
        const int c = (int)(i % 3);
        tgt[i] = (Fn[4 * p + c] - (2.0f * Fc[4 * p + c] - Fp[4 * p + c])) / s[c];
    }
}

// Initial guess: v = 2 v_cur − v_prev + s·Δv on unconstrained nodes (mask bit c), and
// per element P_p = 2 P_cur − P_prev + s·ΔP at the node of DoF p (centre, ξ = 1, η = 1).
template <class T>
__global__ void apply_guess_v_kernel(const T* __restrict__ vprev, const T* __restrict__ vcur, const float* __restrict__ out,
                                     int co, int comp, float s, const uint8_t* __restrict__ mask, T* v, int64_t nnodes) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nnodes; i += (int64_t)gridDim.x * blockDim.x) {
        if (mask && ((mask[i] >> comp) & 1u)) continue;
        const float d = out ? out[(int64_t)co * i + comp] * s : 0.0f;
        v[i] = (T)(2.0 * (double)vcur[i] - (double)vprev[i] + (double)d);
    }
}

template <class T>
__global__ void apply_guess_P_kernel(const T* __restrict__ Pprev, const T* __restrict__ Pcur, const float* __restrict__ out,
                                     int co, float s, const int32_t* __restrict__ dofsP, const int32_t* __restrict__ el2n,
                                     T* P, int64_t nels) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nels; e += (int64_t)gridDim.x * blockDim.x) {
        // Q9 local nodes of the P1-disc DoFs: centre (8), (ξ, η) = (1, 0) (5), (0, 1) (6)
        const int loc[3] = {8, 5, 6};
        for (int p = 0; p < 3; ++p) {
            const int d = dofsP[3 * e + p] - 1;
            const int64_t node = el2n[9 * e + loc[p]] - 1;
            // the grid value at a DoF's node is P0(1−ξ−η) + P1ξ + P2η; ΔP_p follows from the three nodes
            float dp = 0.0f;
            if (out) {
                const float c0 = out[(int64_t)co * (el2n[9 * e + 8] - 1) + 2];
                const float cn = out[(int64_t)co * node + 2];
                dp = (p == 0 ? c0 : cn) * s;
            }
            P[d] = (T)(2.0 * (double)Pcur[d] - (double)Pprev[d] + (double)dp);
        }
    }
}

}  // namespace

template <class T>
cudaError_t launch_grid_fields(const T* vx, const T* vy, const T* P, const int32_t* dofsP, const int32_t* node_elem,
                               const int8_t* node_xi, const int8_t* node_eta, int nx, int ny, float dx, float dy,
                               float* out, cudaStream_t st) {
    count_launch();
    grid_fields_kernel<T><<<blk((int64_t)nx * ny), 256, 0, st>>>(vx, vy, P, dofsP, node_elem, node_xi, node_eta, nx, ny,
                                                                 dx, dy, out);
    return cudaGetLastError();
}
template cudaError_t launch_grid_fields<double>(const double*, const double*, const double*, const int32_t*,
                                                const int32_t*, const int8_t*, const int8_t*, int, int, float, float,
                                                float*, cudaStream_t);

cudaError_t launch_net_input(const float* Fp, const float* Fc, const float* s, void* X, int64_t npix, cudaStream_t st) {
    count_launch();
    net_input_kernel<<<blk(npix * 16), 256, 0, st>>>(Fp, Fc, s, static_cast<__nv_bfloat16*>(X), npix);
    return cudaGetLastError();
}

cudaError_t launch_net_target(const float* Fp, const float* Fc, const float* Fn, const float* s, float* tgt, int64_t npix,
                              cudaStream_t st) {
    count_launch();
    net_target_kernel<<<blk(npix * 3), 256, 0, st>>>(Fp, Fc, Fn, s, tgt, npix);
    return cudaGetLastError();
}

template <class T>
__global__ void extrapolate_kernel(const T* __restrict__ prev, const T* __restrict__ cur, T* x, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = (T)(2.0 * (double)cur[i] - (double)prev[i]);
}

template <class T>
cudaError_t launch_extrapolate_guess(int dim, const T* const* vprev, const T* const* vcur, const T* Pprev,
                                     const T* Pcur, const uint8_t* mask, T* const* v, T* P, int64_t nnodes,
                                     int64_t nP, cudaStream_t st) {
    for (int c = 0; c < dim; ++c) {
        count_launch();
        apply_guess_v_kernel<T><<<blk(nnodes), 256, 0, st>>>(vprev[c], vcur[c], nullptr, 0, c, 0.0f, mask, v[c], nnodes);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    count_launch();
    extrapolate_kernel<T><<<blk(nP), 256, 0, st>>>(Pprev, Pcur, P, nP);
    return cudaGetLastError();
}
template cudaError_t launch_extrapolate_guess<double>(int, const double* const*, const double* const*, const double*,
                                                      const double*, const uint8_t*, double* const*, double*, int64_t,
                                                      int64_t, cudaStream_t);

template <class T>
cudaError_t launch_apply_guess(const T* vprev[2], const T* vcur[2], const T* Pprev, const T* Pcur, const float* out, int co,
                               const float* s, const uint8_t* mask, T* v[2], T* P, const int32_t* dofsP,
                               const int32_t* el2n, int64_t nnodes, int64_t nels, cudaStream_t st) {
    for (int c = 0; c < 2; ++c) {
        count_launch();
        apply_guess_v_kernel<T><<<blk(nnodes), 256, 0, st>>>(vprev[c], vcur[c], out, co, c, s ? s[c] : 0.0f, mask, v[c],
                                                            nnodes);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    count_launch();
    apply_guess_P_kernel<T><<<blk(nels), 256, 0, st>>>(Pprev, Pcur, out, co, s ? s[2] : 0.0f, dofsP, el2n, P, nels);
    return cudaGetLastError();
}
template cudaError_t launch_apply_guess<double>(const double* [2], const double* [2], const double*, const double*,
                                                const float*, int, const float*, const uint8_t*, double* [2], double*,
                                                const int32_t*, const int32_t*, int64_t, int64_t, cudaStream_t);

}  // namespace femb
