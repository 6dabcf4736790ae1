// node.cu — node-wise DR kernels: the fused Chebyshev velocity update with its
// check-iteration reductions, Dirichlet pins, the Powell–Hestenes pressure
// update, spectral-bound reductions and the temperature transfer.
#include <type_traits>
#include "kernels.cuh"

namespace femb {

namespace {

FEMB_D double warp_sum(double x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// Deterministic block reduction of `n` slots; thread 0 writes the block partials.
template <int NS>
FEMB_D void block_reduce_store(double (&acc)[NS], double* out) {
    __shared__ double red[NODE_THREADS / 32][NS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        double x = warp_sum(acc[s]);
        if (lane == 0) red[w][s] = x;
    }
    __syncthreads();
    if (threadIdx.x < NS) {
        double t = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k][threadIdx.x];
        out[(size_t)blockIdx.x * RED_SLOTS + threadIdx.x] = t;
    }
}

// update_stokes_velocity! (helpers.jl:31-41) with the Dirichlet pins of the
// residual and the rate folded in (DR.jl:687-688): constrained entries get R = 0
// and rate = 0. On check iterations the same pass accumulates Σ R², Σ (αr)² and
// Σ (αr)(R − R0)/PC per component (DR.jl:700, :722-724, _stokes_λmin :32-37).
template <class T>
__global__ void __launch_bounds__(NODE_THREADS) node_update_kernel(NodeArgs<T> a) {
    double acc[RED_SLOTS];
#pragma unroll
    for (int s = 0; s < RED_SLOTS; ++s) acc[s] = 0.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        const unsigned msk = a.mask ? a.mask[i] : 0u;
        // all loads of the node first: the stores below may alias them as far as the
        // compiler knows, and would otherwise serialise the components' round trips
        T R[3], rt[3], pc[3], vv[3], r0[3], rf[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (c < a.dim) {
                R[c] = a.Rv[c][i]; rt[c] = a.rate[c][i]; pc[c] = a.PC[c][i]; vv[c] = a.v[c][i];
                r0[c] = a.reduce ? a.Rv0[c][i] : T(0);
                rf[c] = (a.fill && a.Rfill[c]) ? a.Rfill[c][i] : T(0);
            }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (c >= a.dim) break;
            T r;
            if ((msk >> c) & 1u) {
                R[c] = T(0);
                if (!a.fill) a.Rv[c][i] = T(0);
                r = T(0);
                a.rate[c][i] = T(0);
            } else {
                r = (T)a.beta[c] * rt[c] + R[c] / pc[c];
                a.rate[c][i] = r;
                a.v[c][i] = vv[c] + (T)a.alpha[c] * r;
            }
            if (a.save_R0) a.Rv0[c][i] = R[c];
            if (a.fill) a.Rv[c][i] = rf[c];
            if (a.reduce) {
                const double Rd = (double)R[c];
                const double sr = a.lam_step[c] * (double)r;
                acc[c * 3 + 0] += Rd * Rd;
                acc[c * 3 + 1] += sr * sr;
                acc[c * 3 + 2] += sr * ((Rd - (double)r0[c]) / (double)pc[c]);
            }
        }
    }
    if (a.reduce) block_reduce_store<RED_SLOTS>(acc, a.partials);
}

// One component of one node of node_update_kernel, on values already loaded:
// returns the new rate and velocity and the values Rv0 and Rv take.
struct NodeOut {
    float rate, v, R0, Rv;
};
template <bool REDUCE>
FEMB_D NodeOut node_comp(const NodeArgs<float>& a, int c, bool masked, float R, float rt, float pc, float vv, float r0,
                         float rf, double* acc) {
    NodeOut o;
    float r;
    if (masked) {
        R = 0.0f;
        r = 0.0f;
        o.v = vv;
    } else {
        r = (float)a.beta[c] * rt + R / pc;
        o.v = vv + (float)a.alpha[c] * r;
    }
    o.rate = r;
    o.R0 = R;
    o.Rv = a.fill ? rf : R;
    if (REDUCE) {
        const double Rd = (double)R;
        const double sr = a.lam_step[c] * (double)r;
        acc[c * 3 + 0] += Rd * Rd;
        acc[c * 3 + 1] += sr * sr;
        acc[c * 3 + 2] += sr * ((Rd - (double)r0) / (double)pc);
    }
    return o;
}

// node_update_kernel for FP32 state, four nodes per thread with 128-bit accesses
// (every array 16-byte aligned); the n mod 4 last nodes go one per thread.
// REDUCE (check iterations only) carries the FP64 partial sums; without it the
// kernel needs no FP64 registers.
template <bool REDUCE>
__global__ void __launch_bounds__(NODE_THREADS, 2) node_update_f32x4_kernel(NodeArgs<float> a) {
    pdl_enter();
    double acc[RED_SLOTS];
#pragma unroll
    for (int s = 0; s < RED_SLOTS; ++s) acc[s] = 0.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n4 = a.n >> 2;
    for (int64_t g = tid; g < n4; g += stride) {
        const uint32_t m4 = a.mask ? __ldg(reinterpret_cast<const uint32_t*>(a.mask) + g) : 0u;
        float4 R[3], rt[3], pc[3], vv[3], r0[3], rf[3];
        const float4 z4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (c < a.dim) {
                R[c] = reinterpret_cast<const float4*>(a.Rv[c])[g];
                rt[c] = reinterpret_cast<const float4*>(a.rate[c])[g];
                pc[c] = __ldg(reinterpret_cast<const float4*>(a.PC[c]) + g);
                vv[c] = reinterpret_cast<const float4*>(a.v[c])[g];
                r0[c] = REDUCE ? reinterpret_cast<const float4*>(a.Rv0[c])[g] : z4;
                rf[c] = (a.fill && a.Rfill[c]) ? __ldg(reinterpret_cast<const float4*>(a.Rfill[c]) + g) : z4;
            }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (c >= a.dim) break;
            const float* Rj = &R[c].x; const float* tj = &rt[c].x; const float* pj = &pc[c].x;
            const float* vj = &vv[c].x; const float* r0j = &r0[c].x; const float* rfj = &rf[c].x;
            float4 orate, ov, oR0, oRv;
            float* pr = &orate.x; float* pv = &ov.x; float* p0 = &oR0.x; float* pR = &oRv.x;
            bool any_masked = false;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const bool masked = (m4 >> (8 * j + c)) & 1u;
                any_masked |= masked;
                const NodeOut o = node_comp<REDUCE>(a, c, masked, Rj[j], tj[j], pj[j], vj[j], r0j[j], rfj[j], acc);
                pr[j] = o.rate; pv[j] = o.v; p0[j] = o.R0; pR[j] = o.Rv;
            }
            reinterpret_cast<float4*>(a.rate[c])[g] = orate;
            reinterpret_cast<float4*>(a.v[c])[g] = ov;
            if (a.save_R0) reinterpret_cast<float4*>(a.Rv0[c])[g] = oR0;
            if (a.fill || any_masked) reinterpret_cast<float4*>(a.Rv[c])[g] = oRv;
        }
    }
    for (int64_t i = 4 * n4 + tid; i < a.n; i += stride) {
        const unsigned msk = a.mask ? a.mask[i] : 0u;
        for (int c = 0; c < a.dim; ++c) {
            const bool masked = (msk >> c) & 1u;
            const NodeOut o = node_comp<REDUCE>(a, c, masked, a.Rv[c][i], a.rate[c][i], a.PC[c][i], a.v[c][i],
                                        REDUCE ? a.Rv0[c][i] : 0.0f, (a.fill && a.Rfill[c]) ? a.Rfill[c][i] : 0.0f, acc);
            a.rate[c][i] = o.rate;
            a.v[c][i] = o.v;
            if (a.save_R0) a.Rv0[c][i] = o.R0;
            if (a.fill || masked) a.Rv[c][i] = o.Rv;
        }
    }
    if (REDUCE) block_reduce_store<RED_SLOTS>(acc, a.partials);
}

template <class T>
__global__ void dirichlet_kernel(T* x, const int32_t* dofs, const T* vals, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[dofs[i] - 1] = vals ? vals[i] : T(0);
}

__global__ void mask_kernel(uint8_t* mask, const int32_t* dofs, int64_t n, int comp) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        uint8_t* m = mask + (dofs[i] - 1);
        *m = (uint8_t)(*m | (1u << comp));
    }
}

template <class T>
__global__ void __launch_bounds__(NODE_THREADS) sumsq_kernel(const T* x, const T* div, int64_t n, double* partials) {
    double acc[1] = {0.0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double r = div ? (double)(x[i] / div[i]) : (double)x[i];
        acc[0] += r * r;
    }
    block_reduce_store<1>(acc, partials);
}

template <class T>
__global__ void __launch_bounds__(NODE_THREADS) ratio_max_kernel(const T* J, const T* PC, int64_t n, double* partials) {
    __shared__ double red[NODE_THREADS / 32][2];
    double mx = -INFINITY, nan = 0.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double r = (double)(J[i] / PC[i]);
        if (r != r) nan = 1.0; else mx = fmax(mx, r);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        nan = fmax(nan, __shfl_xor_sync(0xffffffffu, nan, o));
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { red[w][0] = mx; red[w][1] = nan; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = -INFINITY, f = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { m = fmax(m, red[k][0]); f = fmax(f, red[k][1]); }
        partials[(size_t)blockIdx.x * RED_SLOTS + 0] = m;
        partials[(size_t)blockIdx.x * RED_SLOTS + 1] = f;
    }
}

template <class T>
__global__ void pressure_update_kernel(T* P, const T* gP, const T* RP, const T* MP, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) P[i] += gP[i] * RP[i] / MP[i];
}

template <class T>
__global__ void pnum_kernel(T* Pn, const T* gP, const T* RP, const T* MP, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) Pn[i] = gP[i] * RP[i] / MP[i];
}

template <class T>
__global__ void sub_kernel(T* x, const T* y, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] -= y[i];
}

template <class T>
__global__ void copy_kernel(T* d, const T* s, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) d[i] = s[i];
}

template <class T>
__global__ void transfer_kernel(T* TP, const T* Tn, const int32_t* dofsP, const int32_t* el2nP, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) TP[dofsP[i] - 1] = Tn[el2nP[i] - 1];
}

// update_rate_kernel! / update_variable_kernel! (dynamic_relaxation/solver.jl:182-198)
// with the Dirichlet pins of R and the rate folded in.
template <class T>
__global__ void thermal_update_kernel(T* Tn, T* rate, T* R, const T* PC, const uint8_t* mask, int64_t n, double alpha,
                                      double beta) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (mask && mask[i]) {
        R[i] = T(0);
        rate[i] = T(0);
        return;
    }
    const T r = R[i] / PC[i] + (T)beta * rate[i];
    rate[i] = r;
    Tn[i] += (T)alpha * r;
}

template <class T>
__global__ void __launch_bounds__(NODE_THREADS) lmin_kernel(const T* rate, const T* R, const T* R0, const T* PC,
                                                            int64_t n, double step, double* partials) {
    double acc[3] = {0.0, 0.0, 0.0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double sr = step * (double)rate[i];
        acc[0] += sr * sr;
        acc[1] += sr * (((double)R[i] - (double)R0[i]) / (double)PC[i]);
        acc[2] += (double)R[i] * (double)R[i];
    }
    block_reduce_store<3>(acc, partials);
}

inline unsigned nblk(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

}  // namespace

namespace {
bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }
}  // namespace

template <class T>
cudaError_t launch_node_update(const NodeArgs<T>& a, int blocks, cudaStream_t st, bool pdl) {
    count_launch();
    if constexpr (std::is_same<T, float>::value) {
        bool ok = aligned16(a.mask);
        for (int c = 0; c < a.dim; ++c)
            ok = ok && aligned16(a.v[c]) && aligned16(a.rate[c]) && aligned16(a.Rv[c]) && aligned16(a.PC[c]) &&
                 aligned16(a.Rv0[c]) && aligned16(a.Rfill[c]);
        if (ok) {
            return launch_pdl(pdl, a.reduce ? node_update_f32x4_kernel<true> : node_update_f32x4_kernel<false>,
                              dim3((unsigned)blocks), dim3(NODE_THREADS), 0, st, a);
        }
    }
    node_update_kernel<T><<<blocks, NODE_THREADS, 0, st>>>(a);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_dirichlet(T* x, const int32_t* dofs, const T* vals, int64_t n, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    count_launch();
    dirichlet_kernel<T><<<nblk(n), 256, 0, st>>>(x, dofs, vals, n);
    return cudaGetLastError();
}

cudaError_t launch_build_mask(uint8_t* mask, const int32_t* dofs, int64_t n, int comp, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    count_launch();
    mask_kernel<<<nblk(n), 256, 0, st>>>(mask, dofs, n, comp);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_sumsq(const T* x, const T* div, int64_t n, double* partials, int blocks, cudaStream_t st) {
    count_launch();
    sumsq_kernel<T><<<blocks, NODE_THREADS, 0, st>>>(x, div, n, partials);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_ratio_max(const T* J, const T* PC, int64_t n, double* partials, int blocks, cudaStream_t st) {
    count_launch();
    ratio_max_kernel<T><<<blocks, NODE_THREADS, 0, st>>>(J, PC, n, partials);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_pressure_update(T* P, const T* gP, const T* RP, const T* MP, int64_t n, cudaStream_t st) {
    count_launch();
    pressure_update_kernel<T><<<nblk(n), 256, 0, st>>>(P, gP, RP, MP, n);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_pnum(T* Pn, const T* gP, const T* RP, const T* MP, int64_t n, cudaStream_t st) {
    count_launch();
    pnum_kernel<T><<<nblk(n), 256, 0, st>>>(Pn, gP, RP, MP, n);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_sub(T* x, const T* y, int64_t n, cudaStream_t st) {
    count_launch();
    sub_kernel<T><<<nblk(n), 256, 0, st>>>(x, y, n);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_copy(T* d, const T* s, int64_t n, cudaStream_t st) {
    count_launch();
    copy_kernel<T><<<nblk(n), 256, 0, st>>>(d, s, n);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_transfer_temperature(T* TP, const T* Tn, const int32_t* dofsP, const int32_t* el2nP, int64_t n,
                                        cudaStream_t st) {
    count_launch();
    transfer_kernel<T><<<nblk(n), 256, 0, st>>>(TP, Tn, dofsP, el2nP, n);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_thermal_update(T* Tn, T* rate, T* R, const T* PC, const uint8_t* mask, int64_t n, double alpha,
                                  double beta, cudaStream_t st) {
    count_launch();
    thermal_update_kernel<T><<<nblk(n), 256, 0, st>>>(Tn, rate, R, PC, mask, n, alpha, beta);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_lmin_sums(const T* rate, const T* R, const T* R0, const T* PC, int64_t n, double step,
                             double* partials, int blocks, cudaStream_t st) {
    count_launch();
    lmin_kernel<T><<<blocks, NODE_THREADS, 0, st>>>(rate, R, R0, PC, n, step, partials);
    return cudaGetLastError();
}

#define FEMB_INST(T)                                                                                                  \
    template cudaError_t launch_node_update<T>(const NodeArgs<T>&, int, cudaStream_t, bool);                               \
    template cudaError_t launch_dirichlet<T>(T*, const int32_t*, const T*, int64_t, cudaStream_t);                   \
    template cudaError_t launch_sumsq<T>(const T*, const T*, int64_t, double*, int, cudaStream_t);                   \
    template cudaError_t launch_ratio_max<T>(const T*, const T*, int64_t, double*, int, cudaStream_t);               \
    template cudaError_t launch_pressure_update<T>(T*, const T*, const T*, const T*, int64_t, cudaStream_t);         \
    template cudaError_t launch_pnum<T>(T*, const T*, const T*, const T*, int64_t, cudaStream_t);                    \
    template cudaError_t launch_sub<T>(T*, const T*, int64_t, cudaStream_t);                                         \
    template cudaError_t launch_copy<T>(T*, const T*, int64_t, cudaStream_t);                                        \
    template cudaError_t launch_transfer_temperature<T>(T*, const T*, const int32_t*, const int32_t*, int64_t,       \
                                                        cudaStream_t);                                               \
    template cudaError_t launch_thermal_update<T>(T*, T*, T*, const T*, const uint8_t*, int64_t, double, double,     \
                                                  cudaStream_t);                                                     \
    template cudaError_t launch_lmin_sums<T>(const T*, const T*, const T*, const T*, int64_t, double, double*, int, \
                                             cudaStream_t);
FEMB_INST(double)
FEMB_INST(float)
#undef FEMB_INST


// Mixed precision: fold the FP32 increment into the FP64 state (x += δ, δ = 0),
// and FP32 images of FP64 arrays (y = x, or y = x + δ).
__global__ void fold_kernel(double* x, float* d, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { x[i] += (double)d[i]; d[i] = 0.0f; }
}
__global__ void round_kernel(float* y, const double* x, const float* d, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = d ? (float)(x[i] + (double)d[i]) : (float)x[i];
}

cudaError_t launch_fold(double* x, float* d, int64_t n, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    count_launch();
    fold_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(x, d, n);
    return cudaGetLastError();
}
cudaError_t launch_round(float* y, const double* x, const float* d, int64_t n, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    count_launch();
    round_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(y, x, d, n);
    return cudaGetLastError();
}

}  // namespace femb
