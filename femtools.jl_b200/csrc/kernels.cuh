// kernels.cuh — argument packs and launchers of the libfemtools_b200 kernels.
#pragma once
#include <limits>
#include <utility>
#include "common.cuh"

namespace femb {

// Kernels launched by this library since the last profile reset (every launcher
// adds one per launch); reported through femb200_profile_read.
extern unsigned long long g_kernel_launches;
// programmatic dependent launch of the inner iteration's kernels (launch_pdl); set from
// FEMB200_PDL at handle creation
extern int g_pdl_enabled;
inline void count_launch() { __atomic_fetch_add(&g_kernel_launches, 1ull, __ATOMIC_RELAXED); }

// Launches `kernel`, with programmatic stream serialization when `pdl` is set (the kernel
// calls pdl_enter() before touching global memory), so that it is scheduled while its
// predecessor drains.
template <class... KArgs, class... Args>
cudaError_t launch_pdl(bool pdl, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                       Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl && g_pdl_enabled ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

constexpr int H27_THREADS = 128;   // 4 warps × 3 elements per warp

template <class T, class TG>
struct H27Args {
    const int32_t* el2n;
    const int32_t* dofsP;
    const TG* geo_v;
    const TG* geo_P;
    const T* v[3];
    T* Rv[3];
    const T* P;
    const T* P0;          // nodal P_old (or P0)
    const T* P_old_ip;    // nq × nels P_old, or null
    const T* temp;        // T on pressure DoFs
    const T* temp0;
    const T* Q;
    const T* Pf;
    const T* gammaP;
    const T* MP;
    T* RP;
    T* Pnum_out;
    const T* Pnum_in;     // stored Pnum read instead of γP·RP/M_P, or null
    const int32_t* phv; int phv_layout;
    const int32_t* php; int php_layout;
    const T* told[6];
    const T* eta_ip;
    T* tau_store[6];
    T* phi;               // shear dissipation output (nq × nels) or null
    int64_t nels;
    T dt;
    int with_pnum;
    int do_momentum;
    int write_RP;
    // Mixed precision (FP32 increments about an FP64 base state, pipelined sweep only):
    // the base sweep writes the trial stress (6) and yield value (1) of every
    // integration point as FP32 into base_out (tiled, rheology.cuh base_index);
    // the incremental sweep reads them from base_in, takes v and P as the
    // increments δv, δP and adds its increments to Rv (pre-filled with the base
    // residual) and to RP_base.
    float* base_out;
    const float* base_in;
    const T* RP_base;
    // the element groups this launch processes, in order (group g is elements 3g … 3g + 2;
    // one colour of the ordered scatter, pipelined sweep only), or null for every group
    const int32_t* group_list;
    int64_t group_count;
};

template <class T, class TG>
cudaError_t launch_hex27_residual(const H27Args<T, TG>& args, int num_sms, cudaStream_t st);

// Pipelined sweep over affine Hex27 elements with one J⁻¹, |det J| per element.
template <class T>
cudaError_t launch_hex27_residual_pipe(const H27Args<T, T>& args, const T* geo_c, int num_sms, cudaStream_t st);
// FP32 incremental sweep of the mixed-precision solve (args.base_in, args.RP_base set).
cudaError_t launch_hex27_residual_incr(const H27Args<float, float>& args, const float* geo_c, int num_sms, cudaStream_t st);
template <class TG, class TC>
cudaError_t launch_compress_geometry(const TG* geo_v, const TG* geo_P, int64_t nels, TC* out, int* not_affine,
                                     cudaStream_t st);

// Thread-per-element FP32 incremental sweep (stokes3d_incr.cu) on meshes whose
// elements each carry one phase (any layout). Its per-element inputs are re-laid in tiles of 32 elements
// (element e at tile e/32, lane e%32) once per solve, so every per-element read of
// a warp is one coalesced line.
struct IncrPhase {
    float twoe;        // 2ηve at the solve's Δt
    float rho0beta;    // ρ0/K: EOS density increment per unit pressure increment
    float cC;          // C·cosϕ
    float sphi;        // sinϕ
    float inv_den;     // 1/(ηve + η_reg + Kb·Δt·sinΨ·sinϕ)
    float invbulkdt;   // 1/(bulk·Δt), 0 when every phase is incompressible
    float invG_dt;     // 1/(GΔt), for viscosities given per integration point
    float den_rest;    // η_reg + Kb·Δt·sinΨ·sinϕ, likewise
};
struct IncrArgs {
    const int32_t* el2n_t;   // [tiles][27][32] 0-based nodes in tensor order i + 3j + 9k
    const int32_t* dofs_t;   // [tiles][4][32]  0-based pressure DoFs
    const float* geo_t;      // [tiles][10][32] J⁻¹ (column-major) and |det J|
    const int32_t* phase_t;  // [2][tiles·32] 0-based phase of the element's velocity nodes, then of its pressure DoFs
    const float* base_t;     // tiled base data (rheology.cuh base_index)
    const float* eta_t;      // [tiles][27][32] viscosity per integration point, or null
    const float* pscale_t;   // [tiles][4][32] γP/M_P of the element's pressure DoFs
    const float* dv[3];
    const float* dP;
    float* R[3];             // pre-filled with the base residual; increments added
    float* RPinc;            // increment of the pressure residual at the DoFs
    int64_t nels;
    int dofs_linear;         // the pressure DoFs of element e are 4e … 4e+3 (dofs_t not read)
    int diag_geometry;       // every element's J⁻¹ is diagonal
    int plastic;
    float g[3];
    IncrPhase ph[MAXPH];
    // when set (profiling), the number of (element, point) pairs whose base trial stress
    // the sweep read is added here
    unsigned long long* stress_reads;
    // when set, the number of (element, point) pairs the elastic bound did not settle
    unsigned long long* bound_failures;
    // load every row's base trial stresses a row ahead (regions that yield) instead of
    // reading them on demand where the bound fails (elastic regions)
    int prefetch_stress;
    int* err_flag;   // set (to 1) when a bulk-copy wait of the sweep gave up; its warp then stops
    // the tiles this launch processes, in order (one colour of the ordered scatter), or
    // null for every tile
    const int32_t* tile_list;
    int64_t tile_count;
};
// Builds el2n_t, dofs_t, geo_t (from the compressed per-element geometry FP32
// copy), phase_t, pscale_t and, if eta is given (e·27 + q layout), eta_t of dst.
// Sets bit INCR_MIXED_PHASES of *flags when some element's nodes or DoFs carry
// more than one phase (the thread-per-element sweep then does not apply),
// INCR_DOFS_GENERAL when the pressure DoFs are not numbered 4e + p and
// INCR_GEOMETRY_FULL when some element's J⁻¹ has an off-diagonal entry.
enum { INCR_MIXED_PHASES = 1, INCR_DOFS_GENERAL = 2, INCR_GEOMETRY_FULL = 4 };
struct IncrTileSrc {
    const int32_t* el2n;
    const int32_t* dofsP;
    const float* geo_c;
    const float* eta;
    const float* gP;
    const float* MP;
    const int32_t* phv; int phv_layout;
    const int32_t* php; int php_layout;
    int nphases;
};
cudaError_t launch_incr_tiles(const IncrTileSrc& src, int64_t nels, const IncrArgs& dst, int32_t* flags,
                              cudaStream_t st);
// pdl: programmatic dependent launch (the mixed solve sets it when every warp of the sweep
// processes at most one tile, where the gap between the sweep and the node update is a
// sizeable part of an iteration)
cudaError_t launch_hex27_incr(const IncrArgs& a, int num_sms, cudaStream_t st, bool pdl = false);
// tiles the FP32 sweep processes at once: resident warps on num_sms SMs
int64_t incr_warp_slots(int num_sms);
// out = x + y (FP32)
cudaError_t launch_add_f32(float* out, const float* x, const float* y, int64_t n, cudaStream_t st);

// Adjoint (transposed-Jacobian) residual of the Hex27/P1-disc element at the forward
// state (adjoint3d.cu): out_dv += (dR/dv)ᵀλ (atomics), out_dP = (dR/dP)ᵀλ (element-
// private stores), optionally out_eta = λ·∂R/∂η per integration point.
template <class T>
struct AdjArgs {
    const int32_t* el2n;
    const int32_t* dofsP;
    const T* geo_v;
    const T* geo_P;
    const T* v[3];
    const T* P;
    const T* Pf;
    const T* gammaP;
    const T* MP;
    const int32_t* phv; int phv_layout;
    const int32_t* php; int php_layout;
    const T* told[6];
    const T* eta_ip;
    const T* lam_v[3];
    const T* lam_P;
    T* out_dv[3];
    T* out_dP;
    T* out_eta;
    int64_t nels;
    T dt;
    int with_pnum;
};
template <class T>
cudaError_t launch_hex27_adjoint(const AdjArgs<T>& args, int num_sms, cudaStream_t st);

// ---- learned warm start (conv_bf16.cu, warmstart_fields.cu) ----
// err: device word set to 1 when a tensor-core wait of the kernel gave up
cudaError_t launch_conv3x3(int ci, int co, int mode, const void* in, const void* wt, const float* bias,
                           const void* mask, void* out, int B, int H, int W, int num_sms, int* err, cudaStream_t st);
cudaError_t launch_conv3x3_wgrad(int ci, int co, const void* x, const void* dy, float* dw, float* db, int B, int H, int W,
                                 int num_sms, int* err, cudaStream_t st);
cudaError_t launch_flip_weights(const void* w, void* wT, int ci, int co, cudaStream_t st);
cudaError_t launch_mse(const float* out, const float* target, int nt, int co, float scale, void* dy, int64_t npix,
                       double* partials, int blocks, cudaStream_t st);
cudaError_t launch_adam(float* w, float* m, float* v, const float* g, void* wb, int64_t n, float lr, float b1, float b2,
                        float eps, int64_t step, cudaStream_t st);
cudaError_t launch_f32_to_bf16(const float* x, void* y, int64_t n, cudaStream_t st);
template <class T>
cudaError_t launch_grid_fields(const T* vx, const T* vy, const T* P, const int32_t* dofsP, const int32_t* node_elem,
                               const int8_t* node_xi, const int8_t* node_eta, int nx, int ny, float dx, float dy,
                               float* out, cudaStream_t st);
cudaError_t launch_net_input(const float* Fp, const float* Fc, const float* s, void* X, int64_t npix, cudaStream_t st);
cudaError_t launch_net_target(const float* Fp, const float* Fc, const float* Fn, const float* s, float* tgt, int64_t npix,
                              cudaStream_t st);
// Cell-pressure Hex27 Stokes (cellpressure.cu): FP64, P / RP / pressure_mass 4 × nels.
struct CpArgs {
    int64_t nels;
    const int32_t* el2n;
    const double* geo_v;
    const int32_t* phases;
    double eta[FEMB200_MAX_PHASES], rho[FEMB200_MAX_PHASES], g[3];
    const double* v[3];
    const double* P;
    double* Rv[3];
    double* RP;
    double* diagonal[3];
    double* pressure_mass;
    const double* geo_c;     // per-cell affine geometry (J⁻¹, |det J|) or null: per-point geo_v
};
cudaError_t launch_cp_compress_geometry(const double* geo_v, int64_t nels, double* out, int* not_affine, cudaStream_t st);
cudaError_t launch_cp_pressure_residual(const CpArgs& a, int num_sms, cudaStream_t st);
cudaError_t launch_cp_momentum_residual(const CpArgs& a, int num_sms, cudaStream_t st);
cudaError_t launch_cp_preconditioner(const CpArgs& a, int num_sms, cudaStream_t st);
int cp_mean_blocks(int num_sms);
cudaError_t launch_cp_validate(const int32_t* el2n, const int32_t* phases, int64_t nels, int64_t nnodes, int nphases,
                               int* bad, cudaStream_t st);
cudaError_t launch_cp_pressure_update(double* P, const double* RP, const double* M, int64_t nels, double step,
                                      double* partials, int nb, cudaStream_t st);
// The momentum step of one relaxation iteration for the three components at once: Rv_c
// less the load (where given), zero at the entries bit c of mask constrains, and
// v_c −= step·Rv_c/diagonal_c at the others (the constrained velocities keep their
// prescribed values). With zero set, Rv is left zeroed for the next momentum residual
// instead of holding this residual.
struct CpVelArgs {
    double* v[3];
    double* Rv[3];
    const double* diag[3];
    const double* load[3];
    const uint8_t* mask;
    int64_t n;
    double step;
    int zero;
};
cudaError_t launch_cp_velocity_step(const CpVelArgs& a, cudaStream_t st);

// Element-averaged strain-rate and stress diagnostics (postprocess.cu).
template <class T, class TG>
struct PostArgs {
    const int32_t* el2n;
    const TG* geo_v;
    const T* v[3];
    const T* tau[6];      // nq × nels each: 6 components in 3-D, (xx, yy, xy) in 2-D
    T* out[14];           // nels each: 14 fields in 3-D, 10 in 2-D
    int64_t nels;
};
template <class T, class TG>
cudaError_t launch_strain_rate_stress(int dim, const PostArgs<T, TG>& a, cudaStream_t st);

// Element geometry at the velocity integration points (geometry.cu).
template <class TG>
cudaError_t launch_geometry(int dim, const double* coords, const int32_t* el2n, int64_t nels, int64_t nnodes, TG* geo_v,
                            TG* geo_P, int* bad, cudaStream_t st);

template <class T>
cudaError_t launch_extrapolate_guess(int dim, const T* const* vprev, const T* const* vcur, const T* Pprev,
                                     const T* Pcur, const uint8_t* mask, T* const* v, T* P, int64_t nnodes,
                                     int64_t nP, cudaStream_t st);
template <class T>
cudaError_t launch_apply_guess(const T* vprev[2], const T* vcur[2], const T* Pprev, const T* Pcur, const float* out, int co,
                               const float* s, const uint8_t* mask, T* v[2], T* P, const int32_t* dofsP,
                               const int32_t* el2n, int64_t nnodes, int64_t nels, cudaStream_t st);

// Augmented Jacobian diagnostics of Hex27 (row sums → dRdv, |diag| → PC).
// Inputs and L1 row sums / |diagonal| of one phase's shared elastic element Jacobian
// (rows indexed [tensor node · 3 + component]).
template <class T>
struct JacTemplate {
    int32_t valid;
    T geo[27 * 11];
    T gam[4], MP[4], eta_pc;
    T rows[81], diag[81];
};

template <class T, class TG>
struct H27JacArgs {
    const int32_t* el2n;
    const int32_t* dofsP;
    const TG* geo_v;
    const TG* geo_P;
    const T* v[3];
    const T* P;
    const T* P0;
    const T* temp;
    const T* temp0;
    const T* Pf;
    const T* gammaP;
    const T* MP;
    const int32_t* phv; int phv_layout;
    const int32_t* php; int php_layout;
    const T* told[6];
    const T* eta_ip;
    T* dRdv[3];
    T* PC[3];
    int64_t nels;
    T dt;
    int diag_geometry;    // every J⁻¹ diagonal (the Hex27 kernel's DIAG specialisation)
    // Shared element Jacobians (Hex27 FP32 diagnostics, one phase per cell): JAC_TMPL_BUILD computes, for
    // the element pick[p] of each phase p, the diagnostics of its elastic linearisation
    // and its inputs into tmpl[p]; JAC_TMPL_USE lets a warp whose three elements are
    // all elastic at the current state and whose inputs equal their phase's template
    // take the template's rows instead of the 81 columns (the same code on inputs equal
    // within 4e-7 relative, jacobian3d.cu same_input).
    int tmpl_mode;
    struct JacTemplate<T>* tmpl;
    const int32_t* pick;
    int64_t pick_nels;    // element count of the mesh the picks index (bound of every pick)
    unsigned long long* shared_count;   // when set (profiling): elements that took a template
    // as H27Args::group_list (Hex27; not read when building templates)
    const int32_t* group_list;
    int64_t group_count;
};
enum { JAC_TMPL_OFF = 0, JAC_TMPL_USE = 1, JAC_TMPL_BUILD = 2 };
// fill of the pick array before launch_jac_pick (a byte-wise memset of 0x7f)
constexpr int32_t JAC_NO_PICK = 0x7f7f7f7f;
template <class TG>
cudaError_t launch_geo_offdiag(const TG* geo_v, int64_t nels, int* flag, cudaStream_t st);
// pick[p] ← the lowest element index whose cell phase is p + 1 (pick pre-filled with JAC_NO_PICK)
cudaError_t launch_jac_pick(const int32_t* phv, int64_t nels, int32_t* pick, cudaStream_t st);

template <class T, class TG>
cudaError_t launch_hex27_jacobian(const H27JacArgs<T, TG>& args, int num_sms, cudaStream_t st);

// Pressure mass and scale (pressure_scaling.jl:166-216).
template <class T, class TG>
cudaError_t launch_pressure_scaling(int dim, const int32_t* el2n, const int32_t* dofsP, const TG* geo_P,
                                    const int32_t* phv, int phv_layout, const T* eta_ip, int use_eta_ip,
                                    T* MP, T* gP, int64_t nels, int64_t nnodesP, T gfact, T dt, cudaStream_t st);

// Q9/P1-disc plane-strain residual sweep (thread per element).
template <class T, class TG>
cudaError_t launch_q9_residual(const H27Args<T, TG>& args, cudaStream_t st);
template <class T, class TG>
cudaError_t launch_q9_jacobian(const H27JacArgs<T, TG>& args, cudaStream_t st);

// ---- node-wise kernels -------------------------------------------------------

// Scalars of the DR iteration kept on the device (α, β per component and the
// Powell–Hestenes update factor), so launches need no host round trip.
struct IterScalars {
    double alpha[3];
    double beta[3];
};

// Block-partial reductions written by the fused node sweep on check iterations.
constexpr int RED_SLOTS = 12;   // per component: Σ R², Σ (a r)², Σ (a r)(R−R0)/PC ; + spare
constexpr int NODE_THREADS = 256;

template <class T>
struct NodeArgs {
    T* v[3];
    T* rate[3];
    T* Rv[3];
    T* Rv0[3];
    const T* PC[3];
    const uint8_t* mask;   // bit c: component c constrained at this node
    int64_t n;
    int dim;
    double alpha[3];       // negated Chebyshev step (v += alpha·rate)
    double beta[3];
    int save_R0;           // copy (masked) R into Rv0 after the update (the next iteration checks)
    int fill;              // then set Rv to the next sweep's starting value: Rfill, or 0
    const T* Rfill[3];
    int reduce;            // write block partials of the norms and λmin sums
    double lam_step[3];    // α used in the λmin sums (DR.jl:722-724)
    double* partials;      // gridDim.x × RED_SLOTS
};

template <class T>
cudaError_t launch_node_update(const NodeArgs<T>& a, int blocks, cudaStream_t st, bool pdl = false);

template <class T>
cudaError_t launch_dirichlet(T* x, const int32_t* dofs, const T* vals, int64_t n, cudaStream_t st);

cudaError_t launch_build_mask(uint8_t* mask, const int32_t* dofs, int64_t n, int comp, cudaStream_t st);

// Σ x² over an array (block partials), and Σ (RP/M_P)².
template <class T>
cudaError_t launch_sumsq(const T* x, const T* div, int64_t n, double* partials, int blocks, cudaStream_t st);

// P += γP·RP/M_P (DR.jl:777) and Pnum = γP·RP/M_P.
template <class T>
cudaError_t launch_pressure_update(T* P, const T* gP, const T* RP, const T* MP, int64_t n, cudaStream_t st);
template <class T>
cudaError_t launch_pnum(T* Pnum, const T* gP, const T* RP, const T* MP, int64_t n, cudaStream_t st);

// max(J/PC) with NaN propagation (block partials) for _checked_λmax.
template <class T>
cudaError_t launch_ratio_max(const T* J, const T* PC, int64_t n, double* partials, int blocks, cudaStream_t st);

template <class T>
cudaError_t launch_sub(T* x, const T* y, int64_t n, cudaStream_t st);
template <class T>
cudaError_t launch_copy(T* dst, const T* src, int64_t n, cudaStream_t st);
// Mixed precision: x += δ and δ = 0 (FP64 state, FP32 increment); y = (float)(x [+ δ]).
cudaError_t launch_fold(double* x, float* d, int64_t n, cudaStream_t st);
cudaError_t launch_round(float* y, const double* x, const float* d, int64_t n, cudaStream_t st);

template <class T>
cudaError_t launch_transfer_temperature(T* TP, const T* Tn, const int32_t* dofsP, const int32_t* el2nP, int64_t n,
                                        cudaStream_t st);

// Thermal diffusion element residual (+ Jacobian diagnostics).
template <class T, class TG>
struct ThermalArgs {
    int dim;
    const int32_t* el2n;
    const TG* geo;
    const T* Tn; const T* T0; const T* P; const T* src; const T* src_ip;
    const int32_t* ph; int ph_layout;
    T* R; T* dRdT; T* PC;
    int64_t nels;
    T dt, Tref;
    int jac;
    // colour group (1-based element indices, elements sharing no node) or null: with
    // a group the launch covers only its elements and scatters with plain adds
    const int32_t* group;
    int64_t ngroup;
};
template <class T, class TG>
cudaError_t launch_thermal(const ThermalArgs<T, TG>& a, int num_sms, cudaStream_t st);

// Lithostatic pressure (simple.cu): FP64, per-phase constants by value.
struct LithoArgs {
    int dim;
    const int32_t* el2n;
    const double* geo;
    const double* P;
    const double* Tn;
    const int32_t* ph;
    int ph_layout;
    double* R;
    double* dRdP;
    double* PC;
    int64_t nels;
    double Tref;
    double g[3];
    int jac;
    double rho0[MAXPH], alpha[MAXPH], beta[MAXPH];
};
cudaError_t launch_lithostatic(const LithoArgs& a, cudaStream_t st);

// Tensile-cap local updates, one thread per point (cap.cu).
cudaError_t launch_cap_update(const femb200_cap_problem& p, int num_sms, cudaStream_t st);

// Thermal DR node update: rate = R/PC + β rate; T += α rate, masked by Dirichlet.
template <class T>
cudaError_t launch_thermal_update(T* Tn, T* rate, T* R, const T* PC, const uint8_t* mask, int64_t n, double alpha,
                                  double beta, cudaStream_t st);

// Generic λmin sums of the thermal solver: Σ (s r)², Σ (s r)(R−R0)/PC.
template <class T>
cudaError_t launch_lmin_sums(const T* rate, const T* R, const T* R0, const T* PC, int64_t n, double step,
                             double* partials, int blocks, cudaStream_t st);

struct DevThermalMaterial {
    double k[MAXPH], Cp[MAXPH], rho0[MAXPH], alpha[MAXPH], beta[MAXPH];
};
extern __constant__ DevThermalMaterial c_tmat;

}  // namespace femb
