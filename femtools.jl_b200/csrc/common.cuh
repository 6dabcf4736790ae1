// common.cuh — device-side constants and helpers shared by the libfemtools_b200 kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/femtools_b200.h"

#define FEMB_HD __host__ __device__ __forceinline__
#define FEMB_D __device__ __forceinline__

namespace femb {

constexpr int MAXPH = FEMB200_MAX_PHASES;

// Material of one solve in constant memory, always in double; kernels convert to
// their arithmetic type once per use. Mirrors femb200_stokes_material with the
// reciprocals the residuals need (1/G interpolated as compliance, 1/K as β).
struct DevStokesMaterial {
    int nphases;
    int plastic;
    int all_bulk_inf;          // every storage modulus infinite (pressure_residual.jl:143)
    double eta[MAXPH];         // viscosity used by the residual
    double eta_scaling[MAXPH]; // viscosity of the pressure scaling
    double invG[MAXPH];
    double alpha[MAXPH];
    double rho0[MAXPH];
    double beta[MAXPH];        // 1/K (EOS compressibility)
    double bulk[MAXPH];        // ηb or K: storage modulus of the continuity residual
    double inv_Kscale[MAXPH];  // 1/(ηb or K) for the pressure scaling
    double g[3];
    double Tref;
    double cos_phi[MAXPH], sin_phi[MAXPH], sin_psi[MAXPH], C[MAXPH], eta_reg[MAXPH], Kb[MAXPH];
    // Per-phase constants of an element whose nodes all carry one phase, for the
    // Δt of the upload (valid when dt_consts == the kernel's Δt): the Maxwell
    // viscosity ηve = 1/(1/η + 1/(GΔt)), 2ηve, 2ηve/(2GΔt), C·cosϕ, the reciprocal
    // plastic denominator 1/(ηve + η_reg + Kb·Δt·sinΨ·sinϕ) and 1/(bulk·Δt).
    double dt_consts;
    double u_twoe[MAXPH], u_twoe_el[MAXPH], u_cC[MAXPH], u_inv_den[MAXPH], u_inv_bulkdt[MAXPH];
};

// Hex27 tensor tables: 1-D quadratic Lagrange values/derivatives at the 3 Gauss
// points (B[q][i], Dd[q][i]), the local node number of tensor node (i,j,k), and
// the reference coordinate of each Gauss point.
struct DevTables {
    double B[3][3];
    double Dd[3][3];
    double w1[3];
    double qx[3];
    int tn3[27];     // Hex27 local node of tensor index i + 3j + 9k
    int tn2[9];      // Q9 local node of tensor index i + 3j
    double sumN3[27];// Σ_a N_a(q), Hex27 (partition of unity up to rounding)
    double sumN2[9];
    double N2[9][9]; // Q9 N[q][a]
    double dN2[9][9][2];
    double NP2[9][3];
    double w2[9];
    double NP3[27][4];
    double w3[27];
    double N3[27][27];      // Hex27 N[q][a]
    double dN3[27][27][3];  // Hex27 ∂N_a/∂ξ_j at q
};

extern __constant__ DevStokesMaterial c_mat;
extern __constant__ DevTables c_tab;

template <class T> FEMB_D T ld(const T* p) { return __ldg(p); }

// eps(T)^2 of the reference's second-invariant floor (rheology.jl:211, :399).
template <class T> FEMB_HD T eps2();
template <> FEMB_HD double eps2<double>() { return 2.220446049250313e-16 * 2.220446049250313e-16; }
template <> FEMB_HD float eps2<float>() { return 1.1920929e-07f * 1.1920929e-07f; }

FEMB_D void atomic_add(double* p, double v) { atomicAdd(p, v); }
FEMB_D void atomic_add(float* p, float v) { atomicAdd(p, v); }

// Programmatic dependent launch (sm_90+) of the inner DR iteration's kernels: a kernel
// launched with programmatic stream serialization may be scheduled while its predecessor
// in the stream still runs. It waits here, before its first global-memory access, until
// the predecessor grid has completed and its writes are visible, then lets its own
// successor be scheduled. Without the launch attribute both are no-ops.
FEMB_D void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Phase lookup for the three layouts (src/utils.jl:70-72); returns 0-based.
FEMB_D int phase_of(const int32_t* ph, int layout, int64_t node1, int i, int64_t e, int n) {
    if (!ph) return 0;
    if (layout == FEMB200_PHASE_CELL) return __ldg(ph + e) - 1;
    if (layout == FEMB200_PHASE_ELEMENT_NODE) return __ldg(ph + (int64_t)n * e + i) - 1;
    return __ldg(ph + node1 - 1) - 1;
}

}  // namespace femb
