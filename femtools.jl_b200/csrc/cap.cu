// cap.cu — batched tensile-cap local updates (cap_return_map / cap_local_update,
// src/stokes/assemblers/rheology.jl:640-724): one thread per point, FP64.
#include <algorithm>
#include "kernels.cuh"
#include "cap.cuh"

namespace femb {
namespace {

constexpr int CAP_THREADS = 128;

template <int NC>
__global__ void __launch_bounds__(CAP_THREADS) cap_update_kernel(const femb200_cap_problem p) {
    constexpr int nc = NC;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += (int64_t)gridDim.x * blockDim.x) {
        double tt[NC > 0 ? NC : 1];
        double st;
        if (nc > 0) {
#pragma unroll
            for (int j = 0; j < nc; ++j) tt[j] = __ldg(p.tau_trial + i * nc + j);
            st = cap_second_invariant(tt, nc);
        } else {
            st = __ldg(p.s_trial + i);
        }
        const double Pt = __ldg(p.P_trial + i), eve = __ldg(p.eta_ve + i), Kdt = __ldg(p.K_dt + i);
        const CapReturn<double> r = cap_return_map(st, Pt, eve, Kdt, __ldg(p.k + i), __ldg(p.kq + i), __ldg(p.c + i),
                                                   __ldg(p.pT + i), __ldg(p.eta_reg + i), p.maxiter);
        // cap_local_update (rheology.jl:700-724): a failed solve gives NaN rates
        const double lam = r.converged ? r.lam : __longlong_as_double(0x7ff8000000000000ll);
        const double gdot = lam * r.At, tdot = lam * r.Ap;
        if (p.tau && nc > 0)
#pragma unroll
            for (int j = 0; j < nc; ++j) p.tau[i * nc + j] = tt[j] - 2.0 * eve * gdot * tt[j] / st;
        if (p.tau_II) p.tau_II[i] = r.s;
        if (p.P) p.P[i] = nc > 0 ? Pt + Kdt * tdot : r.p;
        if (p.lambda) p.lambda[i] = r.lam;
        if (p.A_tau) p.A_tau[i] = r.At;
        if (p.A_p) p.A_p[i] = r.Ap;
        if (p.gamma_dot) p.gamma_dot[i] = gdot;
        if (p.theta_dot) p.theta_dot[i] = tdot;
        if (p.converged) p.converged[i] = r.converged ? 1 : 0;
    }
}

}  // namespace

cudaError_t launch_cap_update(const femb200_cap_problem& p, int num_sms, cudaStream_t st) {
    if (p.n <= 0) return cudaSuccess;
    count_launch();
    const int64_t want = (p.n + CAP_THREADS - 1) / CAP_THREADS;
    const int blocks = (int)std::min<int64_t>(want, (int64_t)num_sms * 16);
    if (p.ncomp == 6) cap_update_kernel<6><<<blocks, CAP_THREADS, 0, st>>>(p);
    else if (p.ncomp == 3) cap_update_kernel<3><<<blocks, CAP_THREADS, 0, st>>>(p);
    else cap_update_kernel<0><<<blocks, CAP_THREADS, 0, st>>>(p);
    return cudaGetLastError();
}

}  // namespace femb
