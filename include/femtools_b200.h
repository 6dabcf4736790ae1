/*
 * femtools_b200.h — C ABI of libfemtools_b200, the sm_100a backend for the
 * matrix-free dynamic-relaxation (DR) Stokes and thermal-diffusion solvers of
 * FEMTools.jl.
 *
 * Every entry point takes plain pointers and sizes, returns an int status
 * (FEMB200_OK on success) and never synchronises the device: work is queued on
 * the stream set with femb200_set_stream (the legacy default stream if none),
 * and a call that must read a scalar back (a convergence check) synchronises
 * that stream only.
 *
 * Conventions, identical to the Julia arrays the reference hands to its
 * KernelAbstractions kernels, so a Julia caller passes `pointer(::CuArray)`:
 *   - arrays are column-major; connectivities are 1-based int32;
 *   - `el2n` is nv × nels, `dofsP` and `el2nP` are np × nels;
 *   - `geo_v` is nels × nq × (dim·dim + 1): the inverse Jacobian (column-major)
 *     followed by |det J|·ω at each velocity quadrature point
 *     (QuadraturePointGeometry, src/mesh/mesh.jl:467); `geo_P` is nels × nq;
 *   - vector fields are separate component arrays (VectorField3D), stresses are
 *     the six assembler-order components (xx, yy, zz, xy, xz, yz)
 *     (src/stokes/types/stokes_types.jl:316-318), or (xx, yy, xy) in 2-D;
 *   - integration-point arrays (stress history, P_old, viscosity) are nq × nels.
 *
 * The library owns only scratch (reduction buffers and iteration scalars);
 * every state array belongs to the caller.
 */
#ifndef FEMTOOLS_B200_H
#define FEMTOOLS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
enum {
    FEMB200_OK = 0,
    FEMB200_EINVAL = 1,        /* bad argument (sizes, layouts, null pointers) */
    FEMB200_ECUDA = 2,         /* a CUDA runtime call failed */
    FEMB200_ENOMEM = 3,        /* scratch allocation failed */
    FEMB200_ENOTCONV = 4,      /* solve did not converge (throw_on_failure) */
    FEMB200_ENAN = 5,          /* NaN detected in a convergence check */
    FEMB200_EKABOOM = 6,       /* error above 1e10 in a convergence check */
    FEMB200_ELAMBDA = 7,       /* preconditioner produced an invalid lambda_max */
    FEMB200_EUNSUPPORTED = 8,  /* element/option combination not implemented */
    FEMB200_ENONFINITE = 9     /* non-finite thermal residual in a coupled solve */
};

/* ---- enumerations -------------------------------------------------------- */
enum { FEMB200_F64 = 0, FEMB200_F32 = 1 };

/* Phase layouts (src/utils.jl:70-74): a per-node vector indexed through the
 * connectivity, one phase per cell (a 1 × nels matrix), or one phase per
 * element-local node (an n × nels matrix). */
enum { FEMB200_PHASE_NODAL = 0, FEMB200_PHASE_CELL = 1, FEMB200_PHASE_ELEMENT_NODE = 2 };

/* Layout of an auxiliary field: absent, nq × nels at integration points, or
 * nodal (interpolated with the shape functions). */
enum { FEMB200_FIELD_NONE = 0, FEMB200_FIELD_IP = 1, FEMB200_FIELD_NODAL = 2 };

/* Arithmetic of the DR sweeps. FP64 is the reference algorithm. MIXED (3-D
 * affine Hex27, FP64 state) keeps the state in FP64 and runs the Chebyshev
 * iterations in FP32 on increments δv, δP: at every Powell–Hestenes step the
 * increments are folded into the state, the outer residual and convergence test
 * are evaluated in FP64 (as in FP64 mode), and the FP32 residual sweeps evaluate
 * R(x) + [R(x + δ) − R(x)] with the bracket formed from the increments, so FP32
 * rounding scales with δ. Norms are accumulated in FP64. */
enum { FEMB200_PRECISION_FP64 = 0, FEMB200_PRECISION_MIXED = 1 };

#define FEMB200_MAX_PHASES 16

/* ---- problem description ------------------------------------------------- */

/* Per-phase Stokes material (StokesMaterial, src/stokes/types/stokes_types.jl:19)
 * and Drucker-Prager parameters (DruckerPrager, stokes_types.jl:388). Host data. */
typedef struct femb200_stokes_material {
    int32_t nphases;
    double eta[FEMB200_MAX_PHASES];
    double eta_b[FEMB200_MAX_PHASES];
    double G[FEMB200_MAX_PHASES];
    double alpha[FEMB200_MAX_PHASES];
    double rho0[FEMB200_MAX_PHASES];
    double K[FEMB200_MAX_PHASES];
    double g[3];
    double Tref;
    int32_t plastic;                 /* 0: no yield model; 1: DruckerPrager */
    double cos_phi[FEMB200_MAX_PHASES];
    double sin_phi[FEMB200_MAX_PHASES];
    double sin_psi[FEMB200_MAX_PHASES];
    double C[FEMB200_MAX_PHASES];
    double eta_reg[FEMB200_MAX_PHASES];
    double Kb[FEMB200_MAX_PHASES];
    /* Pressure-scaling viscosity (the `scaling_viscosity` keyword of solve!,
     * src/stokes/solvers/DR.jl:309); used only when use_scaling_eta != 0. */
    int32_t use_scaling_eta;
    double scaling_eta[FEMB200_MAX_PHASES];
} femb200_stokes_material;

/* Mesh, state and boundary data of one StokesDR solve. Pointers are device
 * pointers for libfemtools_b200 (host pointers for the CPU oracle); every
 * floating-point array has the type given by `dtype` except the geometry,
 * whose type is `geo_dtype` (the reference's geometry_precision). */
typedef struct femb200_stokes_problem {
    int32_t dim;          /* 2 (plane strain, Q9/P1-disc) or 3 (Hex27/P1-disc) */
    int32_t nv, np, nq;   /* 9,3,9 or 27,4,27 */
    int32_t dtype;        /* FEMB200_F64 or FEMB200_F32 */
    int32_t geo_dtype;
    int64_t nels, nnodes, nnodesP;

    /* mesh */
    const int32_t* el2n;
    const int32_t* dofsP;
    const int32_t* el2nP;
    const void* geo_v;
    const void* geo_P;

    /* velocity-node state (dim components each, length nnodes) */
    void* v[3];
    void* rate[3];        /* ∂v∂τ */
    void* Rv[3];
    void* Rv0[3];
    void* dRdv[3];        /* ∂Rv∂v: Jacobian L1 row sums */
    void* PC[3];          /* |diag| preconditioner */

    /* pressure-DoF state (length nnodesP) */
    void* P;
    void* P0;
    void* gammaP;
    void* T;
    void* T0;
    void* Q;              /* may be NULL: no volumetric source */
    void* Pf;             /* may be NULL: zero fluid pressure */
    void* RP;
    void* M_P;
    void* Pnum;

    /* phases */
    const int32_t* phases_v;
    int32_t phases_v_layout;
    const int32_t* phases_P;
    int32_t phases_P_layout;

    /* stress history and output (3 or 6 components) */
    const void* tau_old[6];
    int32_t tau_old_layout;   /* FEMB200_FIELD_NONE / IP / NODAL */
    void* tau[6];             /* written by femb200_store_stress (IP layout) */

    /* optional overrides */
    const void* P_old;        /* NULL → P0; else nodal (nnodesP) or IP */
    int32_t P_old_layout;
    const void* viscosity_ip; /* NULL → material eta; else nq × nels */
    const void* body_force[3];/* NULL or assembled nodal loads */

    /* Dirichlet conditions, one set per velocity component */
    const int32_t* bc_dofs[3];
    const void* bc_vals[3];
    int64_t bc_n[3];

    femb200_stokes_material mat;
} femb200_stokes_problem;

/* Iteration controls of solve!/solve_stokes_dyrel! (src/stokes/solvers/DR.jl:302-387). */
typedef struct femb200_stokes_controls {
    double dt;
    double pressure_factor;   /* γfact of the pressure scaling (default 50) */
    double tolerance;         /* ϵ_tol (default 1e-6) */
    int64_t max_iterations;   /* total_iterMax (default 50 000) */
    int64_t check_interval;   /* ncheck (default 50) */
    int64_t iter_max;         /* iterMax per Powell–Hestenes step (default 50 000) */
    int64_t max_ph_iterations;/* default 1000 */
    double rel_drop0;         /* default 1e-2 */
    int32_t freeze_jacobian;  /* -1: default (plastic == 0) */
    int32_t finite_K;         /* storage modulus K instead of ηb */
    int32_t assemble_scaling; /* 1: solve! (assemble M_P, γP first); 0: solve_stokes_dyrel! */
    int32_t throw_on_failure; /* nonzero: return FEMB200_ENOTCONV when not converged */
    int32_t precision;        /* FEMB200_PRECISION_FP64 / MIXED */
    double cfl_v;             /* CFL_v (default 0.98) */
    double c_fact;            /* default 0.9 */
    /* Optional history of every convergence check, 4 + dim doubles per entry:
     * (iter, err_v, err_P, unused, err_v_components[dim]). */
    double* history;
    int64_t history_capacity;
} femb200_stokes_controls;

typedef struct femb200_stokes_stats {
    int64_t itPH;
    int64_t iter;
    double err, err_abs, err_rel, err_v, err_P;
    int32_t converged;
    int32_t reached_total_iter;
    double lambda_max;
    double lambda_max_gershgorin;
    int64_t jacobian_assemblies;
    int64_t history_len;
    double err_T;
    int64_t thermal_iterations;
    int64_t defect_corrections;   /* mixed precision: FP64 base sweeps (one per Powell–Hestenes step) */
} femb200_stokes_stats;

/* Thermal diffusion (ThermalDiffusionDR, src/heat_diffusion/types/heat_diffusion_types.jl:90). */
typedef struct femb200_thermal_problem {
    int32_t dim, nv, nq, dtype, geo_dtype;
    int64_t nels, nnodes;
    const int32_t* el2n;
    const void* geo;          /* nels × nq × (dim·dim + 1) */
    void* T; void* T0; void* rate; void* R; void* R0; void* dRdT; void* PC;
    void* P; void* source;
    const void* source_ip;    /* optional nq × nels heat source (shear heating Φ) */
    const int32_t* phases; int32_t phases_layout;
    const int32_t* bc_dofs; const void* bc_vals; int64_t bc_n;
    int32_t nphases;
    double k[FEMB200_MAX_PHASES], Cp[FEMB200_MAX_PHASES], rho0[FEMB200_MAX_PHASES];
    double alpha[FEMB200_MAX_PHASES], K[FEMB200_MAX_PHASES];
    double cfl, c_fact, eps;  /* CFL (0.98), c_fact (0.9), ϵ (1e-6) */
} femb200_thermal_problem;

typedef struct femb200_thermal_controls {
    double dt;
    double Tref;
    double tolerance;         /* relative ‖R‖/‖R⁰‖ */
    int64_t max_iterations;   /* default 10 000 */
    int64_t check_interval;   /* default 100 */
    int32_t throw_on_failure;
} femb200_thermal_controls;

typedef struct femb200_thermal_stats {
    int32_t converged;
    int64_t iterations;
    double residual;
} femb200_thermal_stats;

/* Lithostatic pressure (LithostaticPressureDR,
 * src/lithostatic_pressure/types/lithostatic_pressure_types.jl:1-104): the steady
 * Poisson problem ∫ ∇P·∇v dΩ = ∫ ρ(T, P) g·∇v dΩ for a nodal P on the velocity mesh
 * (Hex27 or Q9), ρ = ρ0(1 − α(T − Tref) + P/K); solved by the same dynamic relaxation
 * as the thermal problem. FP64 device arrays of nnodes entries. */
typedef struct femb200_lithostatic_problem {
    int32_t dim, nv, nq;      /* 3, 27, 27 or 2, 9, 9 */
    int64_t nels, nnodes;
    const int32_t* el2n;
    const double* geo;        /* nels × nq × (dim·dim + 1) */
    double* P;                /* the unknown, updated in place */
    double* rate;             /* ∂P∂τ */
    double* R; double* R0; double* dRdP; double* PC;
    const double* T;          /* temperature (EOS coefficient); NULL → 0 */
    const int32_t* phases; int32_t phases_layout;
    int32_t nphases;
    double rho0[FEMB200_MAX_PHASES], alpha[FEMB200_MAX_PHASES], K[FEMB200_MAX_PHASES];
    const int32_t* bc_dofs; const double* bc_vals; int64_t bc_n;
    double cfl, c_fact, eps;  /* CFL (0.98), c_fact (0.9), ϵ (1e-6) */
} femb200_lithostatic_problem;

typedef struct femb200_lithostatic_controls {
    double Tref;              /* 273 */
    double g[3];              /* body force; (0, −9.81) in 2-D by default */
    double tolerance;         /* relative ‖R‖/‖R⁰‖ (default ϵ) */
    int64_t max_iterations;   /* 10 000 */
    int64_t check_interval;   /* 100 */
    int32_t throw_on_failure;
} femb200_lithostatic_controls;

/* Viscous incompressible Hex27 Stokes with four cell-local pressure modes (1, ξ, η, ζ)
 * per cell (CellPressureStokesDR, src/stokes/types/stokes_types.jl:567-613). FP64
 * device arrays; P, RP and pressure_mass are 4 × nels (column-major: mode fastest). */
typedef struct femb200_cell_pressure_problem {
    int64_t nels, nnodes;
    const int32_t* el2n;          /* 27 × nels, 1-based */
    const double* geo_v;          /* nels × 27 × 10: J⁻¹ (column-major), |det J|·ω */
    const int32_t* phases;        /* one phase per cell, 1-based */
    int32_t nphases;
    double eta[FEMB200_MAX_PHASES];
    double rho[FEMB200_MAX_PHASES];
    double g[3];
    double* v[3];
    double* P;
    double* Rv[3];
    double* RP;
    double* diagonal[3];          /* Jacobi preconditioner */
    double* pressure_mass;        /* lumped mass of the pressure modes */
    const double* load[3];        /* NULL, or a momentum right-hand side subtracted from Rv */
    const int32_t* bc_dofs[3];
    const double* bc_vals[3];     /* NULL → homogeneous */
    int64_t bc_n[3];
} femb200_cell_pressure_problem;

/* Controls of solve!(dr::CellPressureStokesDR, mesh, bc_v; …) (src/stokes/solvers/DR.jl:980-1002). */
typedef struct femb200_cell_pressure_controls {
    double tolerance;             /* 1e-5 */
    int64_t max_iterations;       /* 3000 */
    int64_t check_interval;       /* 100 */
    double velocity_step;         /* 0.6 */
    double pressure_step;         /* 0.2 */
    int32_t throw_on_failure;     /* nonzero: FEMB200_ENOTCONV when not converged */
    double* history;              /* optional (iter, err_v, err_P) per check */
    int64_t history_capacity;
} femb200_cell_pressure_controls;

typedef struct femb200_cell_pressure_stats {
    int32_t converged;
    int32_t reached_total_iter;
    int64_t iterations;
    double residual, err_v, err_P;
    int64_t history_len;
} femb200_cell_pressure_stats;

/* One batch of Drucker–Prager tensile-cap local updates (DruckerPragerCap,
 * src/stokes/types/stokes_types.jl:426-545; Popov, Berlie & Kaus 2025). FP64 device
 * arrays of n points; the material arrays hold each point's parameters as the
 * reference interpolates them to the point: k = sin ϕ, kq = sin Ψ, c = C·cos ϕ (the
 * softened cohesion), pT ≤ 0 (compression-positive pressure), η_reg, and the Maxwell
 * viscosity ηve and Kb·Δt. */
typedef struct femb200_cap_problem {
    int64_t n;
    int32_t ncomp;            /* 0: cap_return_map of s_trial; 3: cap_local_update of a
                                 plane-strain (xx, yy, xy) stress; 6: of a 3-D
                                 (xx, yy, zz, xy, xz, yz) stress */
    int32_t maxiter;          /* Newton budget (40 in the reference) */
    const double* tau_trial;  /* n × ncomp, point-major (ncomp > 0) */
    const double* s_trial;    /* n (ncomp == 0) */
    const double* P_trial;
    const double* eta_ve;
    const double* K_dt;
    const double* k;
    const double* kq;
    const double* c;
    const double* pT;
    const double* eta_reg;
    /* outputs, each optional (NULL: not written) */
    double* tau;              /* n × ncomp: τ_trial − 2ηve·γdot·τ_trial/s_trial */
    double* tau_II;           /* s of the return (s_trial when elastic or failed) */
    double* P;                /* ncomp == 0: p of the return; ncomp > 0: P_trial + Kb·Δt·θdot */
    double* lambda;
    double* A_tau;            /* ½ ∂Q/∂s at the returned state */
    double* A_p;              /* −∂Q/∂p at the returned state */
    double* gamma_dot;        /* λ·A_tau (NaN when the local solve failed) */
    double* theta_dot;        /* λ·A_p (NaN when the local solve failed) */
    int32_t* converged;
} femb200_cap_problem;

/* ---- handle -------------------------------------------------------------- */
typedef struct femb200_handle femb200_handle;

/* Create a handle on the current CUDA device. Replaces the implicit backend
 * state of KA.get_backend(mesh.coords) (src/stokes/solvers/DR.jl:255). */
int femb200_create(femb200_handle** out);
int femb200_destroy(femb200_handle* h);
/* Queue all work on `stream` (a cudaStream_t; NULL = legacy default stream).
 * Replaces CUDA.stream() of the Julia CUDABackend. */
int femb200_set_stream(femb200_handle* h, void* stream);
/* Ordered scatter for mixed-precision solves on this handle (on != 0; off at creation):
 * a reproducible solve. The FP32 sweep runs once per colour of its tiles (32 consecutive
 * elements), the FP64 sweep and the Jacobian diagnostics once per colour of their warp
 * groups (3 consecutive elements); no two units of a colour share a node (greedy colours:
 * 8 tile colours and 10 group colours at 64³), and inside a unit the ξ-face node shared by
 * consecutive elements is added once. Every node then receives at most one atomic addition
 * per launch, in a fixed order of launches, so two solves of the same inputs give the same
 * iterations and fields bit for bit. Costs about a third of the solve time (64³). A solve
 * returns FEMB200_EUNSUPPORTED when a unit's elements share other nodes (tiles that span
 * several rows: fewer than 32 elements along ξ) or when the solve does not take the
 * thread-per-element FP32 sweep. No reference counterpart: the reference's GPU scatter
 * (Atomix, src/stokes/assemblers/momentum_residuals.jl:474-482) is unordered. */
int femb200_set_ordered_scatter(femb200_handle* h, int32_t on);
/* Message of the last failure on this handle (also the reference's error text). */
const char* femb200_last_error(const femb200_handle* h);
/* Build information: compiled architecture and version string. */
const char* femb200_version(void);

/* ---- Stokes element sweeps ------------------------------------------------ */

/* assemble_pressure_residual_kernel! (src/stokes/assemblers/pressure_residual.jl:256):
 * RP ← Σ_e ∫ N (−∇·v − (P−P_old)/(ηb Δt) + α(T−T0)/Δt + Q) dΩ, element-private DoFs.
 * `finite_K` selects K instead of ηb as the storage modulus. */
int femb200_pressure_residual(femb200_handle* h, const femb200_stokes_problem* p,
                              double dt, int32_t finite_K);

/* assemble_momentum_residual_kernel! (src/stokes/assemblers/momentum_residuals.jl:417):
 * Rv ← Σ_e ∫ ∇N·(τ − (P + Pnum) I) − N ρ g dΩ with the visco-elasto-plastic stress
 * of src/stokes/assemblers/rheology.jl. `with_pnum` = 0 passes Pnum = nothing. */
int femb200_momentum_residual(femb200_handle* h, const femb200_stokes_problem* p,
                              double dt, int32_t with_pnum);

/* One fused DR residual sweep: the pressure residual, Pnum = γP·RP/M_P
 * (src/stokes/solvers/DR.jl:665-684) and the momentum residual in one pass. */
int femb200_stokes_residuals(femb200_handle* h, const femb200_stokes_problem* p,
                             double dt, int32_t finite_K);

/* update_stokes_velocity! (src/stokes/helpers.jl:52): per component,
 * rate ← β·rate + Rv/PC; v ← v + alpha·rate (alpha already signed). */
int femb200_velocity_update(femb200_handle* h, const femb200_stokes_problem* p,
                            const double* beta, const double* alpha);

/* apply_dirichlet! (src/dynamic_relaxation/solver.jl:152): x[dofs[i]] ← vals[i]
 * (vals == NULL → 0). dtype as in the problem. */
int femb200_apply_dirichlet(femb200_handle* h, void* x, const int32_t* dofs,
                            const void* vals, int64_t n, int32_t dtype);

/* assemble_augmented_momentum_jacobian_matrices_atomix!
 * (src/stokes/assemblers/momentum_residuals.jl:998): L1 row sums of the augmented
 * element Jacobian into dRdv and |diagonal| of the same-direction block into PC. */
int femb200_jacobian_diagnostics(femb200_handle* h, const femb200_stokes_problem* p,
                                 double dt, int32_t finite_K);

/* assemble_viscosity_weighted_pressure_scaling! (src/stokes/assemblers/pressure_scaling.jl:118):
 * M_P = Σ N² dΩ, γP = Σ N² γ_eff dΩ / M_P. */
int femb200_pressure_scaling(femb200_handle* h, const femb200_stokes_problem* p,
                             double gamma_fact, double dt, int32_t finite_K);

/* update_stokes_current_stress! (src/stokes/solvers/DR.jl:820): integration-point
 * stresses of the current v, P into p->tau (nq × nels each). */
int femb200_store_stress(femb200_handle* h, const femb200_stokes_problem* p, double dt);

/* ---- Stokes solves --------------------------------------------------------- */

/* solve! / solve_stokes_dyrel! (src/stokes/solvers/DR.jl:302, :241, core :348-802).
 * With controls->assemble_scaling the pressure mass and scale are assembled first,
 * as solve! does. Returns FEMB200_ENOTCONV when the solve did not converge and
 * controls->throw_on_failure is set; FEMB200_ENAN / FEMB200_EKABOOM /
 * FEMB200_ELAMBDA on the reference's error paths. */
int femb200_solve_stokes(femb200_handle* h, const femb200_stokes_problem* p,
                         const femb200_stokes_controls* c, femb200_stokes_stats* stats);

/* ---- adjoint (3-D Hex27/P1-disc, FP64) ------------------------------------ */

/* Transposed Jacobian of the augmented residual (Rv with Pnum = γP·RP/M_P formed
 * inline when with_pnum, and RP) at the problem's forward state, applied to
 * λ = (lam_v, lam_P): out_dv = (dR/dv)ᵀλ, out_dP = (dR/dP)ᵀλ. Replaces the
 * reference's frozen element-block apply apply_adjoint_operator!
 * (src/stokes/assemblers/adjoint_operator.jl:640-660; the operator of :3-73) and
 * its Enzyme residual (src/stokes/solvers/DR_adjoint.jl:156-205), matrix-free.
 * Device pointers, nnodes and nnodesP entries. No Dirichlet rows are applied. */
int femb200_stokes_adjoint_residual(femb200_handle* h, const femb200_stokes_problem* p, double dt,
                                    int32_t finite_K, int32_t with_pnum, const void* const lam_v[3],
                                    const void* lam_P, void* const out_dv[3], void* out_dP);

/* λ·∂R/∂η at every integration point (nq × nels, the viscosity_ip layout): the
 * sensitivity of λᵀR to the viscosity field, from which a gradient with respect to
 * any viscosity parameterisation follows by the chain rule (the reference forms
 * per-element material gradients this way, examples/.../sinking_block_adj.jl:117-239,
 * and per phase in src/stokes/solvers/DR_adjoint.jl:495-531). */
int femb200_stokes_viscosity_sensitivity(femb200_handle* h, const femb200_stokes_problem* p, double dt,
                                         int32_t finite_K, int32_t with_pnum, const void* const lam_v[3],
                                         const void* lam_P, void* out_eta_ip);

/* solve_adjoint! (src/stokes/solvers/DR_adjoint.jl:396-433, core :3-325): solves
 * (dR/du)ᵀλ = −objective (objective = ∂J/∂v on the velocity DoFs, zero on the
 * constrained ones) by the Powell–Hestenes/DYREL iteration with the frozen operator
 * at the problem's forward state. The Gershgorin λmax of the Jacobian diagnostics
 * sets the pseudo-time step (the reference's measure_λmax = false). Uses
 * controls: dt, tolerance (adjoint_tol), check_interval (ncheck), rel_drop0
 * (rel_drop, default 0.1), iter_max (iterMax), max_iterations (total_iterMax),
 * max_ph_iterations, finite_K, cfl_v, c_fact, throw_on_failure. Writes the
 * problem's dRdv and PC. lam_v, lam_P: initial guess in, adjoint out. */
int femb200_solve_stokes_adjoint(femb200_handle* h, const femb200_stokes_problem* p,
                                 const femb200_stokes_controls* c, const void* const objective_v[3],
                                 void* const lam_v[3], void* lam_P, femb200_stokes_stats* stats);

/* ---- learned warm start (no reference counterpart: FEMTools.jl has no learned
 * component) --------------------------------------------------------------------
 * A convolutional network over the node grid of a structured 2-D Q9/P1-disc mesh
 * predicts the next time step's correction to linear extrapolation of (vx, vy, P);
 * its BF16 tensor-core kernels (tcgen05 MMAs with FP32 accumulation in tensor
 * memory) and the field transfers are below. Activations are NHWC BF16 with 16 or 32
 * channels; weights are [co][9·ci + 8] (k = (3·ky + kx)·ci + c, eight padding entries
 * per row). The activation, weight and mask arrays are read and written 16 bytes at a
 * time and must be 16-byte aligned (EINVAL otherwise). A tensor-core wait that gives
 * up is reported as ECUDA by a later convolution call or by the loss read-back of
 * femb200_mse_loss_grad. */

/* 3×3 same-padded convolution (zero outside the grid), ci, co ∈ {16, 32}.
 * mode 0: out = ReLU(conv + bias) as BF16; 1: out = conv + bias as FP32;
 * 2: out = conv where mask > 0, else 0, as BF16 (the data gradient through a ReLU:
 *    in = the output gradient, wt = the flipped weights, mask = the layer input). */
int femb200_conv3x3_forward(femb200_handle* h, const void* in, const void* wt, const float* bias,
                            const void* mask, void* out, int32_t batch, int32_t height, int32_t width,
                            int32_t ci, int32_t co, int32_t mode);
/* dw[co][k] += Σ_pixels patch(in)[k]·dy[co] (FP32), db[co] += Σ dy[co] (db may be NULL). */
int femb200_conv3x3_weight_grad(femb200_handle* h, const void* in, const void* dy, float* dw, float* db,
                                int32_t batch, int32_t height, int32_t width, int32_t ci, int32_t co);
/* The data-gradient weights: wT[c][(8 − tap)·co + o] = w[o][tap·ci + c], [ci][9·co + 8]. */
int femb200_conv3x3_flip_weights(femb200_handle* h, const void* w, void* wT, int32_t ci, int32_t co);
/* loss = scale·Σ (out[:, :nt] − target)² (out FP32 with co channels, target FP32 with nt);
 * dy = its gradient in out as BF16 (co channels). loss: host pointer or NULL. */
int femb200_mse_loss_grad(femb200_handle* h, const float* out, const float* target, int32_t nt, int32_t co,
                          double scale, void* dy, int64_t npix, double* loss);
/* One Adam step (Kingma & Ba, 2015) on FP32 parameters, writing a BF16 copy when
 * w_bf16 is not NULL; step counts from 1. */
int femb200_adam_step(femb200_handle* h, float* w, float* m, float* v, const float* g, void* w_bf16,
                      int64_t n, double lr, double beta1, double beta2, double eps, int64_t step);
int femb200_f32_to_bf16(femb200_handle* h, const float* x, void* y, int64_t n);
/* (vx, vy, P, ε̇II) of a 2-D Q9 FP64 state on its (2n+1)² node grid, FP32 (npix × 4):
 * P from the owning element's linear pressure at the node's (ξ, η), ε̇II of the
 * plane-strain deviatoric strain rate by central differences. */
int femb200_q9_grid_fields(femb200_handle* h, const femb200_stokes_problem* p, const int32_t* node_elem,
                           const int8_t* node_xi, const int8_t* node_eta, int32_t nx, int32_t ny, double dx,
                           double dy, float* out);
/* Network input of two consecutive grid states (BF16, 16 channels: F_cur and
 * F_cur − F_prev, divided by the 8 device-side scales; 8 unused) and the training target (F_next − (2 F_cur − F_prev))
 * of vx, vy, P divided by 3 device-side scales. */
int femb200_net_input(femb200_handle* h, const float* Fprev, const float* Fcur, const float* scale, void* X,
                      int64_t npix);
int femb200_net_target(femb200_handle* h, const float* Fprev, const float* Fcur, const float* Fnext,
                       const float* scale, float* target, int64_t npix);
/* Initial guess of the next step: v = 2 v_cur − v_prev (+ scale·out) on the nodes that
 * p's Dirichlet sets leave free, P = 2 P_cur − P_prev (+ scale·out at the node of each
 * P1-disc DoF). out: the network's FP32 output (co channels) or NULL; scale: 3 host
 * floats. Writes p->v and p->P. */
int femb200_apply_warm_start(femb200_handle* h, const femb200_stokes_problem* p, const void* const vprev[2],
                             const void* const vcur[2], const void* Pprev, const void* Pcur, const float* out,
                             int32_t co, const float scale[3]);

/* ---- element geometry (src/mesh/mesh.jl:592-682, src/mesh/mixed_mesh.jl:337-392) ---- */
/* precompute_geometry / update_geometry!: at every velocity integration point of
 * every element, J = Σ_a x_a ∂N_a/∂ξ from the node coordinates (precompute_geometry_kernel!,
 * mesh.jl:674-682), stored as J⁻¹ (column-major) and |det J|·ω in geo_v (nels × nq ×
 * (dim·dim + 1)) and |det J|·ω in geo_P (nels × nq; NULL skips it). coords is nnodes × dim,
 * interleaved (the memory of Julia's Vector{SVector{dim,Float64}}); el2n is nv × nels,
 * 1-based. J is inverted in FP64 and rounded once, on store, to geo_dtype (FEMB200_F64
 * or FEMB200_F32: the reference's geometry_precision, mesh.jl:583-591). dim 3: Hex27
 * (nv = nq = 27); dim 2: Q9 (nv = nq = 9). A connectivity entry outside 1..nnodes
 * returns FEMB200_EINVAL (its points are written as NaN). Synchronises the stream. */
int femb200_precompute_geometry(femb200_handle* h, int32_t dim, int64_t nels, int64_t nnodes,
                                const double* coords, const int32_t* el2n, void* geo_v, void* geo_P,
                                int32_t geo_dtype);

/* ---- lithostatic pressure (src/lithostatic_pressure/) ---- */
/* assemble_lithostatic_pressure_matrices_atomix! (assembly/residual_atomics.jl:1-19):
 * R = Σ_q (ρ ∇N·g − ∇N·∇P) dΩ, and with jac ≠ 0 the Jacobian's absolute row sums
 * (dRdP) and |diagonal| (PC). g has dim components. */
int femb200_lithostatic_residual(femb200_handle* h, const femb200_lithostatic_problem* p, double Tref,
                                 const double g[3], int32_t jac);
/* solve!(dr::LithostaticPressureDR, mesh, bc; …) (solvers/DR.jl:1-44) through
 * solve_dynamic_relaxation! (src/dynamic_relaxation/solver.jl:61-122). */
int femb200_solve_lithostatic(femb200_handle* h, const femb200_lithostatic_problem* p,
                              const femb200_lithostatic_controls* c, femb200_thermal_stats* st);

/* ---- cell-pressure Hex27 Stokes (src/stokes/solvers/DR.jl:980-1057) ---- */
/* stokes_preconditioner_3d! (momentum_residuals.jl:703-745): diagonal_c(a) =
 * Σ η_phase (|∇N_a|² + (∂_c N_a)²/3) dΩ and pressure_mass(m, e) = Σ mode_m² dΩ. */
int femb200_cell_pressure_preconditioner(femb200_handle* h, const femb200_cell_pressure_problem* p);
/* which bit 0: assemble_stokes_pressure_residual_3d! (pressure_residual.jl:330-364),
 * RP(m, e) = −Σ_q mode_m ∇·v dΩ; bit 1: assemble_stokes_momentum_residual_3d!
 * (momentum_residuals.jl:644-700), Rv = ∫ ∇N·(2η ε̇′ − P I) − N ρ g dΩ with η and ρ
 * interpolated over the cell (the reference's interp2ip_phase). The load is not
 * subtracted here. Connectivity outside 1..nnodes or phases outside 1..nphases return
 * FEMB200_EINVAL before any kernel reads by them. */
int femb200_cell_pressure_residuals(femb200_handle* h, const femb200_cell_pressure_problem* p, int32_t which);
/* The Arrow–Hurwicz dynamic relaxation of _relax_cell_pressure_stokes! (DR.jl:1004-1057):
 * P += pressure_step·RP/M, mean of mode 1 removed, v −= velocity_step·Rv/diagonal with
 * the Dirichlet values reapplied; every check_interval iterations (and at the last)
 * err = max(max_c ‖Rv_c‖, ‖RP‖) against the tolerance. The mean removal stays on the
 * device; only checks synchronise. */
int femb200_solve_cell_pressure(femb200_handle* h, const femb200_cell_pressure_problem* p,
                                const femb200_cell_pressure_controls* c, femb200_cell_pressure_stats* st);

/* ---- post-processing (src/postprocess/postprocess.jl:17-79, :168-215) ---- */
/* compute_strain_rate_stress_postprocess from integration-point stresses: per element,
 * the dΩ-weighted averages of the strain rate from p->v and of the deviatoric stress
 * tau_ip (nq × nels arrays: (xx, yy, zz, xy, xz, yz) in 3-D, (xx, yy, xy) in 2-D with
 * τzz = −(τxx + τyy)), and of their second invariants. out: nels arrays in p->dtype,
 * 3-D (14): εxx, εyy, εzz, εxy, εxz, εyz, εII, τxx, τyy, τzz, τxy, τxz, τyz, τII (the
 * invariants with the eps² floor of second_invariant, rheology.jl:395-400); 2-D (10):
 * εxx, εyy, εzz (= 0), εxy, εII, τxx, τyy, τzz, τxy, τII. Uses p's mesh, geometry and v. */
int femb200_strain_rate_stress(femb200_handle* h, const femb200_stokes_problem* p,
                               const void* const tau_ip[6], void* const out[14]);

/* ---- Drucker–Prager tensile cap (src/stokes/assemblers/rheology.jl:510-724) ---- */
/* cap_return_map / cap_local_update at every point of p: the composite yield
 * function (shear line τII = k·P + c closed by a circular cap through pT, tangent to
 * it) and the coupled return for x = (s, p, λ),
 *     s − s_trial + 2ηve·λ·Aτ = 0,  p − p_trial − Kb·Δt·λ·Ap = 0,  F − η_reg·λ = 0,
 * by Newton on residuals scaled by max(|s_trial|, |p_trial|, |F_trial|, eps) with
 * backtracking (at most 24 halvings, s ≥ 0, λ ≥ 0, Armijo decrease) to a scaled
 * infinity norm ≤ 100·eps, then one more full Newton step. An elastic trial state
 * (F ≤ 0) returns unchanged with λ = 0; a failure (ηve or Kb·Δt not positive and
 * finite, a non-finite step, a failed line search, an exhausted budget) returns the
 * trial state with converged = 0, and NaN γdot, θdot, τ and (ncomp > 0) P. */
int femb200_cap_update(femb200_handle* h, const femb200_cap_problem* p);

/* Initial guess of the next time step by linear extrapolation of a 2-D or 3-D FP64
 * state: v = 2 v_cur − v_prev on the DoFs p's Dirichlet sets leave free, P = 2 P_cur −
 * P_prev on every pressure DoF. Writes p->v and p->P. */
int femb200_extrapolate_state(femb200_handle* h, const femb200_stokes_problem* p, const void* const vprev[3],
                              const void* const vcur[3], const void* Pprev, const void* Pcur);

/* ---- thermal diffusion ---------------------------------------------------- */

/* assemble_diffusion_matrices_atomix! (src/heat_diffusion/assembly/residual_atomics.jl:10)
 * with element_residual / element_jacobian (src/heat_diffusion/assembly/residual.jl:7,30). */
int femb200_thermal_residual(femb200_handle* h, const femb200_thermal_problem* t,
                             double dt, double Tref, int32_t compute_jacobian);

/* ---- element colouring (host code) -------------------------------------- */

/* color_mesh_greedy / color_mesh (src/mesh/coloring.jl:26-64): elements are
 * visited in order and each takes the smallest positive colour not used by an
 * element sharing a node with it. Host arrays: el2n is nv × nels (1-based),
 * colors receives nels colours in 1..ncolors. Needs no GPU. */
int femb200_color_mesh(const int32_t* el2n, int32_t nv, int64_t nels, int64_t nnodes,
                       int32_t* colors, int32_t* ncolors);
/* generate_element_groups (src/mesh/coloring.jl:77-81): the 1-based element
 * indices of each colour, ascending, as CSR — group c is
 * elements[offsets[c-1] .. offsets[c]-1]; offsets has ncolors + 1 entries. Host
 * arrays; needs no GPU. */
int femb200_color_groups(const int32_t* colors, int64_t nels, int32_t ncolors,
                         int64_t* offsets, int32_t* elements);
/* assemble_diffusion_matrices_colored! (src/heat_diffusion/assembly/residual_colored.jl:10):
 * the thermal residual (and with jac the Jacobian row sums and |diagonal|) by one
 * launch per colour group, scattering with plain adds. groups: device array of
 * the CSR elements above; offsets: host array of ncolors + 1 entries. */
int femb200_thermal_residual_colored(femb200_handle* h, const femb200_thermal_problem* t,
                                     double dt, double Tref, int32_t jac,
                                     const int32_t* groups, const int64_t* offsets, int32_t ngroups);

/* solve!(::ThermalDiffusionDR, …) (src/heat_diffusion/solvers/DR.jl:50 →
 * src/dynamic_relaxation/solver.jl:61). */
int femb200_solve_thermal(femb200_handle* h, const femb200_thermal_problem* t,
                          const femb200_thermal_controls* c, femb200_thermal_stats* stats);

/* _transfer_temperature! (src/stokes/solvers/DR.jl:44): T_P[dofsP[i]] = T[el2nP[i]]. */
int femb200_transfer_temperature(femb200_handle* h, void* T_P, const void* T,
                                 const int32_t* dofsP, const int32_t* el2nP,
                                 int64_t n, int32_t dtype);

/* assemble_shear_heating! (src/stokes/assemblers/shear_heating.jl:18):
 * Φ = τ:(ε̇ − ε̇_el) at every velocity quadrature point into phi (nq × nels). */
int femb200_shear_heating(femb200_handle* h, const femb200_stokes_problem* p,
                          double dt, void* phi);

/* solve_coupled! (src/stokes/solvers/DR.jl:89): one thermal DR iteration per inner
 * Stokes iteration; `shear_heating` adds Φ to the heat source. */
int femb200_solve_coupled(femb200_handle* h, femb200_thermal_problem* t,
                          const femb200_stokes_problem* p,
                          const femb200_stokes_controls* c, double Tref,
                          int32_t shear_heating, void* phi_scratch,
                          femb200_stokes_stats* stats);

/* ---- measurement (no counterpart in the reference, which has no timers) ---- */

/* Kernel classes timed when profiling is on; slot FEMB200_PROF_ALL counts every
 * kernel the library launched (its milliseconds are not measured). In a
 * mixed-precision solve RESIDUAL holds the FP32 incremental sweeps and OUTER the
 * FP64 sweeps of the Powell–Hestenes steps. */
enum { FEMB200_PROF_RESIDUAL = 0, FEMB200_PROF_JACOBIAN = 1, FEMB200_PROF_NODE = 2, FEMB200_PROF_ALL = 3,
       FEMB200_PROF_OUTER = 4, FEMB200_PROF_COUNT = 5 };

/* Turn per-launch CUDA-event timing of the residual sweep, the Jacobian
 * diagnostics and the node update on (1) or off (0), and reset the totals. The
 * events are recorded on the handle's stream around each launch. */
int femb200_profile(femb200_handle* h, int32_t enable);
/* Totals since the last femb200_profile(h, 1): milliseconds and launch counts per
 * kernel class (arrays of FEMB200_PROF_COUNT). Synchronises the handle's stream. */
int femb200_profile_read(femb200_handle* h, double* ms, int64_t* launches);

/* Work counters of the profiled launches, since the last femb200_profile(h, 1):
 * FEMB200_COUNTER_STRESS_READS = (element, integration point) pairs whose base
 * trial stress the FP32 incremental sweep of the mixed-precision solve read; the
 * others were settled by its elastic bound, which needs only the base yield value.
 * FEMB200_COUNTER_SHARED_JACOBIANS = elements whose Jacobian diagnostics came from
 * their phase's shared elastic element Jacobian instead of their own 81 columns.
 * Writes min(n, FEMB200_COUNTER_COUNT) values. Synchronises the handle's stream. */
enum { FEMB200_COUNTER_STRESS_READS = 0, FEMB200_COUNTER_SHARED_JACOBIANS = 1, FEMB200_COUNTER_COUNT = 4 };
int femb200_profile_counters(femb200_handle* h, int64_t* out, int32_t n);

/* ---- allocation-free thermal solve ---------------------------------------- */

/* Largest thermal mesh (velocity-node count) femb200_solve_thermal_noalloc accepts. */
#define FEMB200_NOALLOC_MAX_NODES 8388608

/* No counterpart in the reference. The same thermal DR solve as
 * femb200_solve_thermal, for callers that must not have the library allocate GPU
 * or pinned host memory: a host that hands all device memory to its own pool
 * (Julia's CUDA.jl pool, PyTorch's caching allocator, an arena sized to the GPU)
 * and runs close to the limit, where a cudaMalloc from the library fails or forces
 * the pool to release memory; or a host that cannot afford the implicit device-wide
 * synchronisation of cudaFree and cudaMallocHost while other streams are busy.
 * femb200_solve_thermal grows its Dirichlet mask and reduction buffers with those
 * calls; this entry point uses instead one fixed scratch array in the library's
 * device image (FEMB200_NOALLOC_MAX_NODES bytes of mask plus about 100 KB of
 * reduction space, 8.5 MB in all), which every GPU that loads the library holds
 * until the process exits. It calls no cudaMalloc, cudaFree, cudaMallocHost or
 * other allocating routine.
 *
 * - Inputs, outputs and status are those of femb200_solve_thermal (FP64 only).
 * - t->nnodes above FEMB200_NOALLOC_MAX_NODES is rejected with FEMB200_EINVAL
 *   before any work is queued.
 * - The first call on a handle looks up the scratch array's device address
 *   (cudaGetSymbolAddress, with the handle's device current) and keeps it in the
 *   handle. Make that first call before any stream capture begins. After
 *   cudaDeviceReset, create new handles: the array may then sit elsewhere.
 * - The reductions use femb200_solve_thermal's split of 4 blocks per SM; a GPU
 *   with more than 256 SMs is rejected with FEMB200_EUNSUPPORTED, since that
 *   split no longer fits the fixed scratch.
 * - Every call, on every stream and handle of the process, shares the one array,
 *   and the array keeps the last call's contents; each call clears the part that
 *   must start at zero. Calls that overlap on the GPU (other streams, other host
 *   threads) race on it and give wrong results: serialise them. */
int femb200_solve_thermal_noalloc(femb200_handle* h, const femb200_thermal_problem* t,
                                  const femb200_thermal_controls* c, femb200_thermal_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* FEMTOOLS_B200_H */
