// api.cu — the C ABI of libfemtools_b200 (include/femtools_b200.h): handle,
// constant-memory set-up, kernel dispatch and the device-resident dynamic-
// relaxation drivers (the host side of _solve_stokes_dyrel!, DR.jl:348-802, and
// solve_dynamic_relaxation!, dynamic_relaxation/solver.jl:61-122).
//
// All state stays on the device; a convergence check reads back a handful of
// reduced scalars (one stream synchronisation per check, as the reference's
// host norms do) and the iteration scalars α, β are passed by value.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#include <mutex>
#include <type_traits>

#include "kernels.cuh"
#include "rheology.cuh"

namespace femb {
__constant__ DevStokesMaterial c_mat;
__constant__ DevTables c_tab;
unsigned long long g_kernel_launches = 0;
int g_pdl_enabled = 1;
}  // namespace femb

using namespace femb;

struct femb200_handle {
    cudaStream_t stream = nullptr;
    int device = 0;
    int num_sms = 148;
    double* d_partials = nullptr;
    size_t partials_cap = 0;    // doubles
    double* h_partials = nullptr;
    size_t h_partials_cap = 0;
    uint8_t* d_mask = nullptr;
    size_t mask_cap = 0;
    uint8_t* d_tmask = nullptr;
    size_t tmask_cap = 0;
    uint8_t* d_cpmask = nullptr;   // Dirichlet bits of the cell-pressure solve
    size_t cpmask_cap = 0;
    // device address of the allocation-free solve's scratch array, looked up by the
    // first femb200_solve_thermal_noalloc call on this handle
    unsigned char* noalloc_base = nullptr;
    std::string err;
    bool tables_ready = false;
    // profiling: event pairs per kernel class, folded into totals when the pool fills
    bool prof = false;
    std::vector<cudaEvent_t> ev_pool[FEMB200_PROF_COUNT];
    size_t ev_used[FEMB200_PROF_COUNT] = {};
    double prof_ms[FEMB200_PROF_COUNT] = {};
    int64_t prof_n[FEMB200_PROF_COUNT] = {};
    int prof_sweep = FEMB200_PROF_RESIDUAL;   // class of launch_residual's sweeps
    unsigned long long launches_at_reset = 0;
    // device counters of the profiled work (FEMB200_COUNTER_*), zeroed by femb200_profile
    unsigned long long* d_counters = nullptr;
    // shared elastic element Jacobians: one template per phase and the picked elements
    void* d_jac_tmpl = nullptr;
    int32_t* d_jac_pick = nullptr;
    int jac_shared = 1;   // FEMB200_JAC_SHARED=0 at creation turns the shared Jacobians off
    // points of the FP32 sweeps that failed the elastic bound since the last check (device
    // and pinned host word), and the sweep variant chosen from it: 1 = trial stresses
    // prefetched row by row (regions that yield), 0 = read on demand (elastic regions)
    unsigned long long* d_bound = nullptr;   // [0] bound failures, [1] bulk-copy wait failures of the FP32 sweep
    unsigned long long* h_bound = nullptr;
    // tensor-core convolutions: device word set when a wait on the MMA completion gave up,
    // and its pinned host mirror, refreshed after every convolution launch
    int* d_conv_err = nullptr;
    int* h_conv_err = nullptr;
    int incr_pre = 0;
    // ordered scatter of the FP32 sweep (femb200_set_ordered_scatter): the tiles sorted by
    // colour (no two tiles of a colour share a node) and the start of each colour
    int ordered_scatter = 0;
    int32_t* d_tile_list = nullptr;
    size_t tile_list_cap = 0;
    std::vector<int64_t> tile_colour_start;
    // the warp groups (three consecutive elements) of the pipelined sweep and the Jacobian
    // diagnostics, sorted by colour, and the start of each colour
    int32_t* d_group_list = nullptr;
    size_t group_list_cap = 0;
    std::vector<int64_t> group_colour_start;
    bool ordered_active = false;   // set inside a mixed solve with the ordered scatter
    // the diagonal-J⁻¹ test of the Jacobian diagnostics, valid for one public call (the
    // geometry cannot change inside a solve): the call's serial and the geometry it tested
    int64_t call_serial = 0;
    int64_t geo_diag_serial = -1;
    const void* geo_diag_ptr = nullptr;
    int geo_diag = 0;
    // compressed affine geometry (one J⁻¹, |det J| per element), rebuilt per call
    void* d_geo_c = nullptr;
    size_t geo_c_cap = 0;
    int* d_flag = nullptr;
    int* h_flag = nullptr;
    bool geo_c_valid = false;
    int use_pipe = 1;   // the pipelined sweep on affine meshes (0 forces the general sweep)
    void* adj_mem = nullptr;   // adjoint workspace: λrate, Resλv, Resλv0, ResλP
    size_t adj_cap = 0;
    int use_incr_thread = 1;   // the thread-per-element incremental sweep where it applies (0: warp-cooperative)
    // FP32 arrays of the mixed-precision solve, carved from one allocation
    struct Mixed {
        void* mem = nullptr;
        size_t cap = 0;
        float *dv[3], *rate[3], *R[3], *R0[3], *Rk[3], *dRdv[3], *PC[3], *v32[3];
        float *dP, *RP, *RPk, *gP, *MP, *P32, *P0, *T, *T0, *Pf;
        float *base, *told[6], *eta;
        float* geo;
        // tiled inputs of the thread-per-element incremental sweep
        int32_t *el2n_t, *dofs_t, *phase_t;
        float *geo_t, *eta_t, *pscale_t, *RPinc;
    } mixed;
};

namespace {

#define CK(...)                                                                                   \
    do {                                                                                          \
        cudaError_t e_ = (__VA_ARGS__);                                                           \
        if (e_ != cudaSuccess) {                                                                  \
            h->err = std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #__VA_ARGS__;  \
            return FEMB200_ECUDA;                                                                 \
        }                                                                                         \
    } while (0)

#define RC(...)                          \
    do {                                 \
        int r_ = (__VA_ARGS__);          \
        if (r_ != FEMB200_OK) return r_; \
    } while (0)

inline double line_N(double x, int node) {
    if (node == -1) return x * (x - 1) * 0.5;
    if (node == 0) return 1 - x * x;
    return x * (x + 1) * 0.5;
}
inline double line_dN(double x, int node) {
    if (node == -1) return x - 0.5;
    if (node == 0) return -2 * x;
    return x + 0.5;
}

// Hex27 / Q9 local node coordinates (src/elements/shape_functions.jl:414-442, :268-278).
const int H27[27][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1}, {-1, -1, 1}, {1, -1, 1}, {1, 1, 1},
                        {-1, 1, 1},   {0, -1, -1}, {1, 0, -1}, {0, 1, -1}, {-1, 0, -1}, {0, -1, 1}, {1, 0, 1},
                        {0, 1, 1},    {-1, 0, 1},  {-1, -1, 0}, {1, -1, 0}, {1, 1, 0},  {-1, 1, 0}, {0, 0, -1},
                        {0, -1, 0},   {1, 0, 0},   {0, 1, 0},   {-1, 0, 0}, {0, 0, 1},  {0, 0, 0}};
const int Q9[9][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}, {0, -1}, {1, 0}, {0, 1}, {-1, 0}, {0, 0}};

DevTables build_tables() {
    DevTables t;
    std::memset(&t, 0, sizeof(t));
    const double a = std::sqrt(3.0 / 5.0);
    const double pts[3] = {-a, 0.0, a};
    const double wts[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
    const int nodes1[3] = {-1, 0, 1};
    for (int q = 0; q < 3; ++q) {
        t.qx[q] = pts[q];
        t.w1[q] = wts[q];
        for (int i = 0; i < 3; ++i) { t.B[q][i] = line_N(pts[q], nodes1[i]); t.Dd[q][i] = line_dN(pts[q], nodes1[i]); }
    }
    for (int a3 = 0; a3 < 27; ++a3) t.tn3[(H27[a3][0] + 1) + 3 * (H27[a3][1] + 1) + 9 * (H27[a3][2] + 1)] = a3;
    for (int a2 = 0; a2 < 9; ++a2) t.tn2[(Q9[a2][0] + 1) + 3 * (Q9[a2][1] + 1)] = a2;
    for (int q = 0; q < 27; ++q) {
        const int qx = q % 3, qy = (q / 3) % 3, qz = q / 9;
        const double x[3] = {pts[qx], pts[qy], pts[qz]};
        t.w3[q] = wts[qx] * wts[qy] * wts[qz];
        double s = 0;
        for (int n = 0; n < 27; ++n) {
            double l[3], dl[3];
            for (int d = 0; d < 3; ++d) { l[d] = line_N(x[d], H27[n][d]); dl[d] = line_dN(x[d], H27[n][d]); }
            t.N3[q][n] = l[0] * l[1] * l[2];
            t.dN3[q][n][0] = dl[0] * l[1] * l[2];
            t.dN3[q][n][1] = l[0] * dl[1] * l[2];
            t.dN3[q][n][2] = l[0] * l[1] * dl[2];
            s += t.N3[q][n];
        }
        t.sumN3[q] = s;
        t.NP3[q][0] = 1 - x[0] - x[1] - x[2];
        t.NP3[q][1] = x[0]; t.NP3[q][2] = x[1]; t.NP3[q][3] = x[2];
    }
    const double w2[9] = {25.0 / 81, 40.0 / 81, 25.0 / 81, 40.0 / 81, 64.0 / 81, 40.0 / 81, 25.0 / 81, 40.0 / 81, 25.0 / 81};
    for (int q = 0; q < 9; ++q) {
        const double x[2] = {pts[q % 3], pts[q / 3]};
        t.w2[q] = w2[q];
        double s = 0;
        for (int n = 0; n < 9; ++n) {
            double l[2], dl[2];
            for (int d = 0; d < 2; ++d) { l[d] = line_N(x[d], Q9[n][d]); dl[d] = line_dN(x[d], Q9[n][d]); }
            t.N2[q][n] = l[0] * l[1];
            t.dN2[q][n][0] = dl[0] * l[1];
            t.dN2[q][n][1] = l[0] * dl[1];
            s += t.N2[q][n];
        }
        t.sumN2[q] = s;
        t.NP2[q][0] = 1 - x[0] - x[1];
        t.NP2[q][1] = x[0]; t.NP2[q][2] = x[1];
    }
    return t;
}

int ensure_tables(femb200_handle* h) {
    if (h->tables_ready) return FEMB200_OK;
    static DevTables host_tab = build_tables();
    CK(cudaMemcpyToSymbolAsync(c_tab, &host_tab, sizeof(DevTables), 0, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->tables_ready = true;
    return FEMB200_OK;
}

// Constant-memory material of one call. `finite_K` selects K as the storage
// modulus of the continuity residual and of the pressure scaling (DR.jl:419, :325).
int upload_material(femb200_handle* h, const femb200_stokes_material& m, int finite_K, double dt = 0.0) {
    if (m.nphases < 1 || m.nphases > FEMB200_MAX_PHASES) { h->err = "nphases must lie in 1:16"; return FEMB200_EINVAL; }
    static thread_local DevStokesMaterial d;   // host staging must outlive the async copy
    std::memset(&d, 0, sizeof(d));
    d.nphases = m.nphases;
    d.plastic = m.plastic;
    bool all_inf = true;
    for (int i = 0; i < FEMB200_MAX_PHASES; ++i) {
        d.eta[i] = m.eta[i];
        d.eta_scaling[i] = m.use_scaling_eta ? m.scaling_eta[i] : m.eta[i];
        d.invG[i] = 1.0 / m.G[i];
        d.alpha[i] = m.alpha[i];
        d.rho0[i] = m.rho0[i];
        d.beta[i] = 1.0 / m.K[i];
        d.bulk[i] = finite_K ? m.K[i] : m.eta_b[i];
        d.inv_Kscale[i] = 1.0 / d.bulk[i];
        if (i < m.nphases && !std::isinf(d.bulk[i])) all_inf = false;
        d.cos_phi[i] = m.cos_phi[i]; d.sin_phi[i] = m.sin_phi[i]; d.sin_psi[i] = m.sin_psi[i];
        d.C[i] = m.C[i]; d.eta_reg[i] = m.eta_reg[i]; d.Kb[i] = m.Kb[i];
    }
    d.all_bulk_inf = all_inf;
    d.dt_consts = dt;
    if (dt > 0) {
        for (int i = 0; i < FEMB200_MAX_PHASES; ++i) {
            const double etave = 1.0 / (1.0 / d.eta[i] + d.invG[i] / dt);
            d.u_twoe[i] = 2 * etave;
            d.u_twoe_el[i] = 2 * etave * (d.invG[i] / (2 * dt));
            d.u_cC[i] = d.cos_phi[i] * d.C[i];
            d.u_inv_den[i] = 1.0 / (etave + d.eta_reg[i] + d.Kb[i] * dt * (-d.sin_psi[i]) * (-d.sin_phi[i]));
            d.u_inv_bulkdt[i] = all_inf ? 0.0 : 1.0 / (d.bulk[i] * dt);
        }
    }
    for (int i = 0; i < 3; ++i) d.g[i] = m.g[i];
    d.Tref = m.Tref;
    CK(cudaMemcpyToSymbolAsync(c_mat, &d, sizeof(d), 0, cudaMemcpyHostToDevice, h->stream));
    // the staging buffer is reused by the next call: make this copy complete first
    CK(cudaStreamSynchronize(h->stream));
    return FEMB200_OK;
}

int check_problem(femb200_handle* h, const femb200_stokes_problem* p) {
    if (!h) return FEMB200_EINVAL;
    if (!p) { h->err = "null problem"; return FEMB200_EINVAL; }
    const bool h27 = p->dim == 3 && p->nv == 27 && p->np == 4 && p->nq == 27;
    const bool q9 = p->dim == 2 && p->nv == 9 && p->np == 3 && p->nq == 9;
    if (!h27 && !q9) { h->err = "libfemtools_b200 supports Hex27/P1-disc (3-D) and Q9/P1-disc (2-D) meshes"; return FEMB200_EUNSUPPORTED; }
    if ((p->dtype != FEMB200_F64 && p->dtype != FEMB200_F32) || (p->geo_dtype != FEMB200_F64 && p->geo_dtype != FEMB200_F32)) {
        h->err = "dtype must be FEMB200_F64 or FEMB200_F32"; return FEMB200_EINVAL;
    }
    if (p->nels <= 0 || p->nnodes <= 0 || p->nnodesP <= 0) { h->err = "empty mesh"; return FEMB200_EINVAL; }
    if (!p->el2n || !p->dofsP || !p->geo_v || !p->geo_P || !p->P) { h->err = "mesh arrays and P are required"; return FEMB200_EINVAL; }
    for (int c = 0; c < p->dim; ++c)
        if (!p->v[c]) { h->err = "velocity components are required"; return FEMB200_EINVAL; }
    return FEMB200_OK;
}

// ---- profiling ----------------------------------------------------------------
constexpr size_t PROF_PAIRS = 512;

int prof_flush(femb200_handle* h, int k) {
    if (h->ev_used[k] == 0) return FEMB200_OK;
    CK(cudaEventSynchronize(h->ev_pool[k][2 * h->ev_used[k] - 1]));
    for (size_t i = 0; i < h->ev_used[k]; ++i) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, h->ev_pool[k][2 * i], h->ev_pool[k][2 * i + 1]));
        h->prof_ms[k] += ms;
    }
    h->ev_used[k] = 0;
    return FEMB200_OK;
}

int prof_begin(femb200_handle* h, int k) {
    if (!h->prof) return FEMB200_OK;
    if (h->ev_pool[k].empty()) {
        h->ev_pool[k].resize(2 * PROF_PAIRS);
        for (auto& e : h->ev_pool[k]) CK(cudaEventCreate(&e));
    }
    if (h->ev_used[k] == PROF_PAIRS) RC(prof_flush(h, k));
    CK(cudaEventRecord(h->ev_pool[k][2 * h->ev_used[k]], h->stream));
    return FEMB200_OK;
}

int prof_end(femb200_handle* h, int k) {
    if (!h->prof) return FEMB200_OK;
    CK(cudaEventRecord(h->ev_pool[k][2 * h->ev_used[k] + 1], h->stream));
    ++h->ev_used[k];
    ++h->prof_n[k];
    return FEMB200_OK;
}

int red_blocks(femb200_handle* h, int64_t n) {
    int64_t b = (n + NODE_THREADS - 1) / NODE_THREADS;
    b = std::min<int64_t>(b, (int64_t)h->num_sms * 4);
    return (int)std::max<int64_t>(b, 1);
}

int ensure_partials(femb200_handle* h, size_t blocks) {
    const size_t need = blocks * RED_SLOTS;
    if (need > h->partials_cap) {
        if (h->d_partials) cudaFree(h->d_partials);
        if (h->h_partials) cudaFreeHost(h->h_partials);
        h->d_partials = nullptr; h->h_partials = nullptr;
        CK(cudaMalloc(&h->d_partials, need * sizeof(double)));
        CK(cudaMallocHost(&h->h_partials, need * sizeof(double)));
        h->partials_cap = need;
    }
    return FEMB200_OK;
}

// Copy block partials back and sum each slot in block order (deterministic).
int fetch_sums(femb200_handle* h, int blocks, int nslots, double* out) {
    CK(cudaMemcpyAsync(h->h_partials, h->d_partials, (size_t)blocks * RED_SLOTS * sizeof(double), cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int s = 0; s < nslots; ++s) {
        double t = 0;
        for (int b = 0; b < blocks; ++b) t += h->h_partials[(size_t)b * RED_SLOTS + s];
        out[s] = t;
    }
    return FEMB200_OK;
}

template <class T>
int sumsq(femb200_handle* h, const T* x, const T* div, int64_t n, double& out) {
    const int b = red_blocks(h, n);
    RC(ensure_partials(h, b));
    CK(launch_sumsq<T>(x, div, n, h->d_partials, b, h->stream));
    return fetch_sums(h, b, 1, &out);
}

// _checked_λmax (src/utils.jl:152-158)
template <class T>
int checked_lmax(femb200_handle* h, const T* J, const T* PC, int64_t n, const char* label, double& out) {
    const int b = red_blocks(h, n);
    RC(ensure_partials(h, b));
    CK(launch_ratio_max<T>(J, PC, n, h->d_partials, b, h->stream));
    CK(cudaMemcpyAsync(h->h_partials, h->d_partials, (size_t)b * RED_SLOTS * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    double m = -INFINITY; bool nan = false;
    for (int i = 0; i < b; ++i) { m = std::max(m, h->h_partials[(size_t)i * RED_SLOTS]); nan = nan || h->h_partials[(size_t)i * RED_SLOTS + 1] != 0; }
    if (nan) m = NAN;
    if (!(std::isfinite(m) && m > 0)) {
        char buf[256];
        std::snprintf(buf, sizeof buf, "%s preconditioner produced invalid λmax = %g; check for zero or non-finite preconditioner entries", label, m);
        h->err = buf;
        return FEMB200_ELAMBDA;
    }
    out = m;
    return FEMB200_OK;
}

template <class T, class TG>
H27Args<T, TG> residual_args(const femb200_stokes_problem* p, double dt) {
    H27Args<T, TG> a;
    std::memset(&a, 0, sizeof(a));
    a.el2n = p->el2n; a.dofsP = p->dofsP;
    a.geo_v = static_cast<const TG*>(p->geo_v); a.geo_P = static_cast<const TG*>(p->geo_P);
    for (int c = 0; c < 3; ++c) { a.v[c] = static_cast<const T*>(p->v[c]); a.Rv[c] = static_cast<T*>(p->Rv[c]); }
    a.P = static_cast<const T*>(p->P);
    const bool ip = p->P_old && p->P_old_layout == FEMB200_FIELD_IP;
    a.P0 = static_cast<const T*>(p->P_old && !ip ? p->P_old : p->P0);
    a.P_old_ip = ip ? static_cast<const T*>(p->P_old) : nullptr;
    // T enters only through α (EOS density and the α∂T/∂t continuity term): with
    // α = 0 in every phase the sweep need not read T and T0 at all.
    bool any_alpha = false;
    for (int i = 0; i < p->mat.nphases; ++i) any_alpha = any_alpha || p->mat.alpha[i] != 0.0;
    a.temp = any_alpha ? static_cast<const T*>(p->T) : nullptr;
    a.temp0 = any_alpha ? static_cast<const T*>(p->T0) : nullptr;
    a.Q = static_cast<const T*>(p->Q); a.Pf = static_cast<const T*>(p->Pf);
    a.gammaP = static_cast<const T*>(p->gammaP); a.MP = static_cast<const T*>(p->M_P);
    a.RP = static_cast<T*>(p->RP);
    a.phv = p->phases_v; a.phv_layout = p->phases_v_layout;
    a.php = p->phases_P; a.php_layout = p->phases_P_layout;
    const int nt = p->dim == 3 ? 6 : 3;
    for (int c = 0; c < 6; ++c)
        a.told[c] = (p->tau_old_layout == FEMB200_FIELD_IP && c < nt) ? static_cast<const T*>(p->tau_old[c]) : nullptr;
    a.eta_ip = static_cast<const T*>(p->viscosity_ip);
    a.nels = p->nels;
    a.dt = (T)dt;
    return a;
}

// Build the per-element affine geometry of a Hex27 problem (in the state type) and
// report whether every element is affine. Costs one read of geo_v.
template <class T, class TG>
int prepare_geometry(femb200_handle* h, const femb200_stokes_problem* p) {
    h->geo_c_valid = false;
    if (p->dim != 3 || !h->use_pipe) return FEMB200_OK;
    const size_t need = (size_t)p->nels * 10 * sizeof(T);
    if (need > h->geo_c_cap) {
        if (h->d_geo_c) cudaFree(h->d_geo_c);
        h->d_geo_c = nullptr;
        CK(cudaMalloc(&h->d_geo_c, need));
        h->geo_c_cap = need;
    }
    if (!h->d_flag) {
        CK(cudaMalloc(&h->d_flag, sizeof(int)));
        CK(cudaMallocHost(&h->h_flag, sizeof(int)));
    }
    CK(cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
    CK(launch_compress_geometry<TG, T>(static_cast<const TG*>(p->geo_v), static_cast<const TG*>(p->geo_P), p->nels,
                                       static_cast<T*>(h->d_geo_c), h->d_flag, h->stream));
    CK(cudaMemcpyAsync(h->h_flag, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->geo_c_valid = *h->h_flag == 0;
    return FEMB200_OK;
}

template <class T, class TG>
int launch_residual(femb200_handle* h, const femb200_stokes_problem* p, const H27Args<T, TG>& a,
                    bool rv_zeroed = false) {
    if (a.do_momentum && !rv_zeroed)
        for (int c = 0; c < p->dim; ++c) CK(cudaMemsetAsync(p->Rv[c], 0, sizeof(T) * p->nnodes, h->stream));
    RC(prof_begin(h, h->prof_sweep));
    if (p->dim == 3 && h->geo_c_valid) {
        H27Args<T, T> b;
        std::memcpy(&b, &a, sizeof(b));   // identical layout; the pipelined sweep reads geometry from d_geo_c
        b.geo_v = nullptr; b.geo_P = nullptr;
        if (h->ordered_active) {
            // one launch per colour of warp groups, in colour order
            for (size_t c = 0; c + 1 < h->group_colour_start.size(); ++c) {
                b.group_list = h->d_group_list + h->group_colour_start[c];
                b.group_count = h->group_colour_start[c + 1] - h->group_colour_start[c];
                CK(launch_hex27_residual_pipe<T>(b, static_cast<const T*>(h->d_geo_c), h->num_sms, h->stream));
            }
        } else {
            CK(launch_hex27_residual_pipe<T>(b, static_cast<const T*>(h->d_geo_c), h->num_sms, h->stream));
        }
    } else if (p->dim == 3) {
        CK(launch_hex27_residual<T, TG>(a, h->num_sms, h->stream));
    } else {
        CK(launch_q9_residual<T, TG>(a, h->stream));
    }
    RC(prof_end(h, h->prof_sweep));
    return FEMB200_OK;
}

// Residual sweep: RP (+ Pnum) and, optionally, Rv.
template <class T, class TG>
int residual_sweep(femb200_handle* h, const femb200_stokes_problem* p, double dt, int with_pnum, int do_momentum,
                   int write_RP, bool rv_zeroed = false) {
    H27Args<T, TG> a = residual_args<T, TG>(p, dt);
    a.with_pnum = with_pnum;
    a.do_momentum = do_momentum;
    a.write_RP = write_RP;
    a.Pnum_out = with_pnum ? static_cast<T*>(p->Pnum) : nullptr;
    if (!with_pnum && !write_RP && !do_momentum) return FEMB200_OK;
    if ((write_RP || with_pnum) && !p->RP) { h->err = "RP is required"; return FEMB200_EINVAL; }
    if (with_pnum && (!p->gammaP || !p->M_P)) { h->err = "γP and M_P are required for Pnum"; return FEMB200_EINVAL; }
    if (do_momentum)
        for (int c = 0; c < p->dim; ++c)
            if (!p->Rv[c]) { h->err = "Rv is required"; return FEMB200_EINVAL; }
    return launch_residual<T, TG>(h, p, a, rv_zeroed);
}

template <class T, class TG>
int jacobian_sweep(femb200_handle* h, const femb200_stokes_problem* p, double dt) {
    H27JacArgs<T, TG> a;
    std::memset(&a, 0, sizeof(a));
    a.el2n = p->el2n; a.dofsP = p->dofsP;
    a.geo_v = static_cast<const TG*>(p->geo_v); a.geo_P = static_cast<const TG*>(p->geo_P);
    for (int c = 0; c < 3; ++c) {
        a.v[c] = static_cast<const T*>(p->v[c]);
        a.dRdv[c] = static_cast<T*>(p->dRdv[c]); a.PC[c] = static_cast<T*>(p->PC[c]);
    }
    a.P = static_cast<const T*>(p->P); a.P0 = static_cast<const T*>(p->P0);
    a.temp = static_cast<const T*>(p->T); a.temp0 = static_cast<const T*>(p->T0);
    a.Pf = static_cast<const T*>(p->Pf);
    a.gammaP = static_cast<const T*>(p->gammaP); a.MP = static_cast<const T*>(p->M_P);
    a.phv = p->phases_v; a.phv_layout = p->phases_v_layout;
    a.php = p->phases_P; a.php_layout = p->phases_P_layout;
    const int nt = p->dim == 3 ? 6 : 3;
    for (int c = 0; c < 6; ++c)
        a.told[c] = (p->tau_old_layout == FEMB200_FIELD_IP && c < nt) ? static_cast<const T*>(p->tau_old[c]) : nullptr;
    a.eta_ip = static_cast<const T*>(p->viscosity_ip);
    a.nels = p->nels;
    a.dt = (T)dt;
    for (int c = 0; c < p->dim; ++c) {
        if (!p->dRdv[c] || !p->PC[c]) { h->err = "dRdv and PC are required"; return FEMB200_EINVAL; }
        CK(cudaMemsetAsync(p->dRdv[c], 0, sizeof(T) * p->nnodes, h->stream));
        CK(cudaMemsetAsync(p->PC[c], 0, sizeof(T) * p->nnodes, h->stream));
    }
    if (!p->gammaP || !p->M_P) { h->err = "γP and M_P are required by the augmented Jacobian"; return FEMB200_EINVAL; }
    if (p->dim == 3) {
        // axis-aligned cells (the structured boxes) take the diagonal-J⁻¹ kernel; one
        // read of the geometry and a synchronisation, at check iterations that synchronise anyway
        if (!h->d_flag) {
            CK(cudaMalloc(&h->d_flag, sizeof(int)));
            CK(cudaMallocHost(&h->h_flag, sizeof(int)));
        }
        if (h->geo_diag_serial != h->call_serial || h->geo_diag_ptr != a.geo_v) {
            CK(cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
            CK(launch_geo_offdiag<TG>(a.geo_v, p->nels, h->d_flag, h->stream));
            CK(cudaMemcpyAsync(h->h_flag, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            h->geo_diag = *h->h_flag == 0;
            h->geo_diag_serial = h->call_serial;
            h->geo_diag_ptr = a.geo_v;
        }
        a.diag_geometry = h->geo_diag;
    }
    // FP32 diagnostics (the mixed-precision solve) on one-phase cells: the elastic element
    // Jacobian of each phase is computed once (on the phase's first element) and shared by
    // every elastic element whose inputs match it
    const bool shared = std::is_same<T, float>::value && p->dim == 3 && h->jac_shared &&
                        (!p->phases_v || p->phases_v_layout == FEMB200_PHASE_CELL);
    RC(prof_begin(h, FEMB200_PROF_JACOBIAN));
    if (shared) {
        if (!h->d_jac_tmpl) {
            CK(cudaMalloc(&h->d_jac_tmpl, sizeof(JacTemplate<double>) * MAXPH));
            CK(cudaMalloc(&h->d_jac_pick, sizeof(int32_t) * MAXPH));
        }
        CK(cudaMemsetAsync(h->d_jac_pick, 0x7f, sizeof(int32_t) * MAXPH, h->stream));   // JAC_NO_PICK
        CK(launch_jac_pick(p->phases_v, p->nels, h->d_jac_pick, h->stream));
        H27JacArgs<T, TG> b = a;
        b.tmpl_mode = JAC_TMPL_BUILD;
        b.tmpl = static_cast<JacTemplate<T>*>(h->d_jac_tmpl);
        b.pick = h->d_jac_pick;
        b.pick_nels = p->nels;
        b.nels = MAXPH;
        CK(launch_hex27_jacobian<T, TG>(b, h->num_sms, h->stream));
        a.tmpl_mode = JAC_TMPL_USE;
        a.tmpl = b.tmpl;
        a.pick = b.pick;
        a.shared_count = h->prof ? h->d_counters + FEMB200_COUNTER_SHARED_JACOBIANS : nullptr;
    }
    if (p->dim == 3 && h->ordered_active) {
        for (size_t c = 0; c + 1 < h->group_colour_start.size(); ++c) {
            a.group_list = h->d_group_list + h->group_colour_start[c];
            a.group_count = h->group_colour_start[c + 1] - h->group_colour_start[c];
            CK(launch_hex27_jacobian<T, TG>(a, h->num_sms, h->stream));
        }
    } else if (p->dim == 3) {
        CK(launch_hex27_jacobian<T, TG>(a, h->num_sms, h->stream));
    } else {
        CK(launch_q9_jacobian<T, TG>(a, h->stream));
    }
    RC(prof_end(h, FEMB200_PROF_JACOBIAN));
    return FEMB200_OK;
}

template <class T, class TG>
int pressure_scaling_impl(femb200_handle* h, const femb200_stokes_problem* p, double gfact, double dt) {
    if (!p->M_P || !p->gammaP) { h->err = "M_P and γP are required"; return FEMB200_EINVAL; }
    CK(cudaMemsetAsync(p->M_P, 0, sizeof(T) * p->nnodesP, h->stream));
    CK(cudaMemsetAsync(p->gammaP, 0, sizeof(T) * p->nnodesP, h->stream));
    const bool use_ip = p->viscosity_ip && !p->mat.use_scaling_eta;
    CK(launch_pressure_scaling<T, TG>(p->dim, p->el2n, p->dofsP, static_cast<const TG*>(p->geo_P), p->phases_v,
                                      p->phases_v_layout, static_cast<const T*>(p->viscosity_ip), use_ip ? 1 : 0,
                                      static_cast<T*>(p->M_P), static_cast<T*>(p->gammaP), p->nels, p->nnodesP, (T)gfact,
                                      (T)dt, h->stream));
    return FEMB200_OK;
}

int build_mask(femb200_handle* h, const femb200_stokes_problem* p) {
    const size_t n = (size_t)p->nnodes;
    if (n > h->mask_cap) {
        if (h->d_mask) cudaFree(h->d_mask);
        h->d_mask = nullptr;
        CK(cudaMalloc(&h->d_mask, n));
        h->mask_cap = n;
    }
    CK(cudaMemsetAsync(h->d_mask, 0, n, h->stream));
    for (int c = 0; c < p->dim; ++c)
        if (p->bc_n[c] > 0) CK(launch_build_mask(h->d_mask, p->bc_dofs[c], p->bc_n[c], c, h->stream));
    return FEMB200_OK;
}

inline double julia_eps(double x) { x = std::fabs(x); return std::nextafter(x, INFINITY) - x; }
// max / min with Julia's semantics: NaN when either argument is NaN. std::max and
// std::min return their first argument when a comparison with NaN fails, which would
// hide a NaN residual from the reference's isnan / isfinite exits.
inline double jl_max(double a, double b) { return (std::isnan(a) || std::isnan(b)) ? NAN : std::max(a, b); }
inline double jl_min(double a, double b) { return (std::isnan(a) || std::isnan(b)) ? NAN : std::min(a, b); }

void cheb(double dtau, double lmin, double c_fact, double& a, double& b) {
    const double c = 2 * std::sqrt(lmin) * c_fact;
    a = 2 * dtau * dtau / (2 + c * dtau);
    b = (2 - c * dtau) / (2 + c * dtau);
}

// Coupled thermal state (DR.jl:604-663).
struct Coupled {
    femb200_thermal_problem* t;
    double Tref;
    void* phi;
};

template <class T, class TG>
int thermal_assemble(femb200_handle* h, const femb200_thermal_problem* t, double dt, double Tref, bool jac,
                     const void* src_ip) {
    ThermalArgs<T, TG> a;
    std::memset(&a, 0, sizeof(a));
    a.dim = t->dim; a.el2n = t->el2n; a.geo = static_cast<const TG*>(t->geo);
    a.Tn = static_cast<const T*>(t->T); a.T0 = static_cast<const T*>(t->T0); a.P = static_cast<const T*>(t->P);
    a.src = static_cast<const T*>(t->source); a.src_ip = static_cast<const T*>(src_ip);
    a.ph = t->phases; a.ph_layout = t->phases_layout;
    a.R = static_cast<T*>(t->R); a.dRdT = static_cast<T*>(t->dRdT); a.PC = static_cast<T*>(t->PC);
    a.nels = t->nels; a.dt = (T)dt; a.Tref = (T)Tref; a.jac = jac ? 1 : 0;
    CK(cudaMemsetAsync(t->R, 0, sizeof(T) * t->nnodes, h->stream));
    if (jac) {
        CK(cudaMemsetAsync(t->dRdT, 0, sizeof(T) * t->nnodes, h->stream));
        CK(cudaMemsetAsync(t->PC, 0, sizeof(T) * t->nnodes, h->stream));
    }
    CK(launch_thermal<T, TG>(a, h->num_sms, h->stream));
    return FEMB200_OK;
}

// assemble_dr_matrices_colored! (src/dynamic_relaxation/assembly.jl:71-92): the
// colour groups one launch after another, each scattering with plain adds.
template <class T, class TG>
int thermal_assemble_colored(femb200_handle* h, const femb200_thermal_problem* t, double dt, double Tref, bool jac,
                             const int32_t* groups, const int64_t* offsets, int32_t ngroups) {
    ThermalArgs<T, TG> a;
    std::memset(&a, 0, sizeof(a));
    a.dim = t->dim; a.el2n = t->el2n; a.geo = static_cast<const TG*>(t->geo);
    a.Tn = static_cast<const T*>(t->T); a.T0 = static_cast<const T*>(t->T0); a.P = static_cast<const T*>(t->P);
    a.src = static_cast<const T*>(t->source); a.src_ip = static_cast<const T*>(t->source_ip);
    a.ph = t->phases; a.ph_layout = t->phases_layout;
    a.R = static_cast<T*>(t->R); a.dRdT = static_cast<T*>(t->dRdT); a.PC = static_cast<T*>(t->PC);
    a.nels = t->nels; a.dt = (T)dt; a.Tref = (T)Tref; a.jac = jac ? 1 : 0;
    CK(cudaMemsetAsync(t->R, 0, sizeof(T) * t->nnodes, h->stream));
    if (jac) {
        CK(cudaMemsetAsync(t->dRdT, 0, sizeof(T) * t->nnodes, h->stream));
        CK(cudaMemsetAsync(t->PC, 0, sizeof(T) * t->nnodes, h->stream));
    }
    for (int32_t g = 0; g < ngroups; ++g) {
        a.group = groups + offsets[g];
        a.ngroup = offsets[g + 1] - offsets[g];
        CK(launch_thermal<T, TG>(a, h->num_sms, h->stream));
    }
    return FEMB200_OK;
}

int upload_thermal_material(femb200_handle* h, const femb200_thermal_problem* t) {
    static thread_local DevThermalMaterial d;
    for (int i = 0; i < FEMB200_MAX_PHASES; ++i) {
        d.k[i] = t->k[i]; d.Cp[i] = t->Cp[i]; d.rho0[i] = t->rho0[i]; d.alpha[i] = t->alpha[i]; d.beta[i] = 1.0 / t->K[i];
    }
    CK(cudaMemcpyToSymbolAsync(c_tmat, &d, sizeof(d), 0, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return FEMB200_OK;
}

int build_tmask(femb200_handle* h, const femb200_thermal_problem* t) {
    const size_t n = (size_t)t->nnodes;
    if (n > h->tmask_cap) {
        if (h->d_tmask) cudaFree(h->d_tmask);
        h->d_tmask = nullptr;
        CK(cudaMalloc(&h->d_tmask, n));
        h->tmask_cap = n;
    }
    CK(cudaMemsetAsync(h->d_tmask, 0, n, h->stream));
    if (t->bc_n > 0) CK(launch_build_mask(h->d_tmask, t->bc_dofs, t->bc_n, 0, h->stream));
    return FEMB200_OK;
}

// One thermal DR iteration of the coupled loop, and its check (DR.jl:604-663).
struct ThermalIter {
    int64_t iter = 0;
    double err = INFINITY, a = 0, b = 0, lmax = 0, nr0 = 0;
    bool converged = false;
};

template <class T, class TG>
int shear_heating_impl(femb200_handle* h, const femb200_stokes_problem* p, double dt, void* phi);

template <class T, class TG>
int thermal_coupled_step(femb200_handle* h, Coupled& cp, ThermalIter& ti, const femb200_stokes_problem* p, int64_t nout,
                         double dt) {
    femb200_thermal_problem* t = cp.t;
    const int64_t n = t->nnodes;
    ++ti.iter;
    const bool check = ti.iter == 1 || ti.iter % nout == 0;
    if (check) CK(launch_copy<T>(static_cast<T*>(t->R0), static_cast<const T*>(t->R), n, h->stream));
    RC((thermal_assemble<T, TG>(h, t, dt, cp.Tref, check, cp.phi)));
    if (check) {
        // the Dirichlet rows of R are zeroed by the update kernel below; λmax reads J and PC only
        RC(checked_lmax<T>(h, static_cast<const T*>(t->dRdT), static_cast<const T*>(t->PC), n, "thermal diffusion", ti.lmax));
    }
    CK(launch_thermal_update<T>(static_cast<T*>(t->T), static_cast<T*>(t->rate), static_cast<T*>(t->R),
                                static_cast<const T*>(t->PC), h->d_tmask, n, ti.a, ti.b, h->stream));
    if (t->bc_n > 0) CK(launch_dirichlet<T>(static_cast<T*>(t->T), t->bc_dofs, static_cast<const T*>(t->bc_vals), t->bc_n, h->stream));
    CK(launch_transfer_temperature<T>(static_cast<T*>(p->T), static_cast<const T*>(t->T), p->dofsP, p->el2nP,
                                      (int64_t)p->np * p->nels, h->stream));
    if (check) {
        const double dtau = 2 / std::sqrt(ti.lmax) * t->cfl;
        const int b = red_blocks(h, n);
        RC(ensure_partials(h, b));
        CK(launch_lmin_sums<T>(static_cast<const T*>(t->rate), static_cast<const T*>(t->R), static_cast<const T*>(t->R0),
                               static_cast<const T*>(t->PC), n, dtau, h->d_partials, b, h->stream));
        double s[3];
        RC(fetch_sums(h, b, 3, s));
        const double nr = std::sqrt(s[2]);
        if (ti.iter == 1) ti.nr0 = std::max(nr, julia_eps(nr));
        ti.err = nr / ti.nr0;
        if (!std::isfinite(ti.err)) {
            char buf[128];
            std::snprintf(buf, sizeof buf, "non-finite thermal residual at coupled iteration %lld", (long long)ti.iter);
            h->err = buf;
            return FEMB200_ENONFINITE;
        }
        const double lmin = (ti.iter == 1 || s[0] == 0) ? 0.0 : std::fabs(s[1]) / s[0];
        cheb(dtau, lmin, t->c_fact, ti.a, ti.b);
        ti.converged = ti.err < t->eps;
        if (cp.phi) RC((shear_heating_impl<T, TG>(h, p, dt, cp.phi)));
    }
    return FEMB200_OK;
}

template <class T, class TG>
int shear_heating_impl(femb200_handle* h, const femb200_stokes_problem* p, double dt, void* phi) {
    H27Args<T, TG> a = residual_args<T, TG>(p, dt);
    a.phi = static_cast<T*>(phi);
    a.do_momentum = 0; a.write_RP = 0; a.with_pnum = 0;
    if (p->dim == 3) CK(launch_hex27_residual<T, TG>(a, h->num_sms, h->stream));
    else CK(launch_q9_residual<T, TG>(a, h->stream));
    return FEMB200_OK;
}

// _solve_stokes_dyrel! (src/stokes/solvers/DR.jl:348-802), device-resident.
template <class T, class TG>
int solve_dyrel(femb200_handle* h, const femb200_stokes_problem* p, const femb200_stokes_controls* c,
                femb200_stokes_stats* st, Coupled* cp) {
    const int D = p->dim;
    const int64_t nn = p->nnodes, nP = p->nnodesP;
    const double dt = c->dt;
    const int finite_K = c->finite_K;
    const bool freeze = c->freeze_jacobian < 0 ? (p->mat.plastic == 0) : (c->freeze_jacobian != 0);
    const int64_t nout = c->check_interval > 0 ? c->check_interval : 50;
    const double cfl = c->cfl_v > 0 ? c->cfl_v : 0.98, cf = c->c_fact > 0 ? c->c_fact : 0.9;
    static const char* labels[3] = {"stokes vx", "stokes vy", "stokes vz"};
    std::memset(st, 0, sizeof(*st));
    for (int k = 0; k < D; ++k)
        if (!p->rate[k] || !p->Rv0[k] || !p->Rv[k] || !p->PC[k] || !p->dRdv[k]) { h->err = "DR work arrays are required"; return FEMB200_EINVAL; }
    if (!p->RP || !p->M_P || !p->gammaP || !p->Pnum) { h->err = "RP, M_P, γP and Pnum are required"; return FEMB200_EINVAL; }

    RC(upload_material(h, p->mat, finite_K, dt));
    RC((prepare_geometry<T, TG>(h, p)));
    RC(build_mask(h, p));
    for (int k = 0; k < D; ++k) {
        CK(cudaMemsetAsync(p->rate[k], 0, sizeof(T) * nn, h->stream));
        CK(cudaMemsetAsync(p->Rv0[k], 0, sizeof(T) * nn, h->stream));
    }
    RC((jacobian_sweep<T, TG>(h, p, dt)));
    double lmax[3] = {0, 0, 0};
    for (int k = 0; k < D; ++k)
        RC(checked_lmax<T>(h, static_cast<const T*>(p->dRdv[k]), static_cast<const T*>(p->PC[k]), nn, labels[k], lmax[k]));
    double lmax_g = *std::max_element(lmax, lmax + D);
    int64_t jac_assemblies = 1;
    double alpha[3] = {0, 0, 0}, beta[3] = {0, 0, 0}, dtau[3];
    for (int k = 0; k < D; ++k) { dtau[k] = 2 / std::sqrt(lmax[k]) * cfl; cheb(dtau[k], 0.0, cf, alpha[k], beta[k]); }

    double err_min = INFINITY, eps = c->tolerance;
    double err = 2 * eps, err_abs = INFINITY, err_rel = INFINITY;
    double err_v0 = 1.0, err_P0 = 1.0, err_v00 = 1.0, err_v = INFINITY, err_P = INFINITY;
    int64_t iter = 0, itPH_done = 0, hist = 0;
    bool converged = false;
    double rel_drop = c->rel_drop0;
    const double sq_nn = std::sqrt((double)nn), sq_nP = std::sqrt((double)nP);
    auto push_hist = [&](double it, double ev, double eP, const double* comps) {
        if (c->history && hist < c->history_capacity) {
            double* hh = c->history + hist * (4 + D);
            hh[0] = it; hh[1] = ev; hh[2] = eP; hh[3] = 0;
            for (int k = 0; k < D; ++k) hh[4 + k] = comps[k];
        }
        ++hist;
    };

    ThermalIter ti;
    bool thermal_converged = cp == nullptr;
    if (cp) {
        RC(upload_thermal_material(h, cp->t));
        RC(build_tmask(h, cp->t));
        CK(cudaMemsetAsync(cp->t->rate, 0, sizeof(T) * cp->t->nnodes, h->stream));
        CK(cudaMemsetAsync(cp->t->R0, 0, sizeof(T) * cp->t->nnodes, h->stream));
        if (cp->phi) RC((shear_heating_impl<T, TG>(h, p, dt, cp->phi)));
    }

    const int nb = red_blocks(h, nn);
    RC(ensure_partials(h, std::max(nb, red_blocks(h, nP))));

    auto apply_bc_R = [&]() -> int {
        for (int k = 0; k < D; ++k) {
            if (p->body_force[k]) CK(launch_sub<T>(static_cast<T*>(p->Rv[k]), static_cast<const T*>(p->body_force[k]), nn, h->stream));
            if (p->bc_n[k] > 0) CK(launch_dirichlet<T>(static_cast<T*>(p->Rv[k]), p->bc_dofs[k], nullptr, p->bc_n[k], h->stream));
        }
        return FEMB200_OK;
    };

    for (int64_t itPH = 1; itPH <= c->max_ph_iterations; ++itPH) {
        itPH_done = itPH;
        RC((residual_sweep<T, TG>(h, p, dt, 0, 1, 1)));
        RC(apply_bc_R());
        double sP;
        RC(sumsq<T>(h, static_cast<const T*>(p->RP), static_cast<const T*>(p->M_P), nP, sP));
        err_P = std::sqrt(sP) / sq_nP;
        double comps[3] = {0, 0, 0};
        err_v = 0;
        for (int k = 0; k < D; ++k) {
            double s;
            RC(sumsq<T>(h, static_cast<const T*>(p->Rv[k]), (const T*)nullptr, nn, s));
            comps[k] = std::sqrt(s) / (2 * sq_nn);
            err_v = jl_max(err_v, std::sqrt(s));
        }
        err_v /= 2 * sq_nn;
        push_hist((double)iter, err_v, err_P, comps);
        if (itPH == 1) { err_P0 = err_P + julia_eps(err_P); err_v0 = err_v + julia_eps(err_v); }
        else if (itPH == 2) err_P0 = err_P + julia_eps(err_P);
        const double err_v_rel = err_v / err_v0, err_P_rel = err_P / err_P0;
        err_abs = jl_max(err_v, err_P);
        err_rel = jl_max(err_v_rel, err_P_rel);
        err = jl_min(err_abs, err_rel);
        if (std::isnan(err)) { char b[96]; std::snprintf(b, sizeof b, "NaN detected in outer loop at PH=%lld", (long long)itPH); h->err = b; return FEMB200_ENAN; }
        if (err > 1e10) { char b[96]; std::snprintf(b, sizeof b, "Kaboom! Error > 1e10 in outer loop at PH=%lld", (long long)itPH); h->err = b; return FEMB200_EKABOOM; }
        if (err < eps && thermal_converged) { converged = true; break; }
        if (err > err_min * 1.05) rel_drop = std::max(rel_drop * 0.1, 1.0e-3);
        err_min = std::min(err_min, err);
        const double eps_vel = err * rel_drop;
        int64_t itPT = 0;
        while ((err > eps_vel || !thermal_converged) && itPT <= c->iter_max) {
            ++itPT; ++iter;
            const bool do_check = iter % nout == 0;
            // After the first iteration of a Powell–Hestenes step the previous node
            // update has zeroed Rv for this sweep and, before a check, saved R0.
            const bool fused = itPT > 1 && nout > 1;
            if (do_check && !fused)
                for (int k = 0; k < D; ++k) CK(launch_copy<T>(static_cast<T*>(p->Rv0[k]), static_cast<const T*>(p->Rv[k]), nn, h->stream));
            if (cp) {
                RC((thermal_coupled_step<T, TG>(h, *cp, ti, p, nout, dt)));
                thermal_converged = ti.converged;
            }
            RC((residual_sweep<T, TG>(h, p, dt, 1, 1, 1, fused)));
            RC(apply_bc_R());
            NodeArgs<T> na;
            std::memset(&na, 0, sizeof(na));
            for (int k = 0; k < 3; ++k) {
                na.v[k] = static_cast<T*>(p->v[k]); na.rate[k] = static_cast<T*>(p->rate[k]);
                na.Rv[k] = static_cast<T*>(p->Rv[k]); na.Rv0[k] = static_cast<T*>(p->Rv0[k]);
                na.PC[k] = static_cast<const T*>(p->PC[k]);
                na.alpha[k] = -alpha[k]; na.beta[k] = beta[k]; na.lam_step[k] = alpha[k];
            }
            na.mask = h->d_mask; na.n = nn; na.dim = D;
            na.reduce = do_check ? 1 : 0;
            na.partials = h->d_partials;
            na.save_R0 = nout > 1 && (iter + 1) % nout == 0;
            na.fill = nout > 1;
            RC(prof_begin(h, FEMB200_PROF_NODE));
            CK(launch_node_update<T>(na, nb, h->stream));
            RC(prof_end(h, FEMB200_PROF_NODE));
            for (int k = 0; k < D; ++k)
                if (p->bc_n[k] > 0) CK(launch_dirichlet<T>(static_cast<T*>(p->v[k]), p->bc_dofs[k], static_cast<const T*>(p->bc_vals[k]), p->bc_n[k], h->stream));
            if (do_check) {
                double s[RED_SLOTS];
                RC(fetch_sums(h, nb, RED_SLOTS, s));
                double ev = 0, cmp[3] = {0, 0, 0};
                for (int k = 0; k < D; ++k) { ev = jl_max(ev, std::sqrt(s[3 * k])); cmp[k] = std::sqrt(s[3 * k]) / (2 * sq_nn); }
                ev /= 2 * sq_nn;
                if (iter == nout) err_v00 = ev + julia_eps(ev);
                err = ev <= eps ? ev : jl_max(ev / err_v00, ev);
                if (std::isnan(err)) { char b[96]; std::snprintf(b, sizeof b, "NaN detected in inner loop PH=%lld PT=%lld", (long long)itPH, (long long)itPT); h->err = b; return FEMB200_ENAN; }
                if (err > 1e10) { char b[96]; std::snprintf(b, sizeof b, "Kaboom! Error > 1e10 in inner loop PH=%lld PT=%lld", (long long)itPH, (long long)itPT); h->err = b; return FEMB200_EKABOOM; }
                if (c->history) {
                    double sPc;
                    RC(sumsq<T>(h, static_cast<const T*>(p->RP), static_cast<const T*>(p->M_P), nP, sPc));
                    push_hist((double)iter, ev, std::sqrt(sPc) / sq_nP, cmp);
                } else {
                    ++hist;
                }
                double lmin[3];
                for (int k = 0; k < D; ++k) lmin[k] = s[3 * k + 1] == 0 ? 0.0 : std::fabs(s[3 * k + 2]) / s[3 * k + 1];
                if (!freeze) {
                    ++jac_assemblies;
                    RC((jacobian_sweep<T, TG>(h, p, dt)));
                    for (int k = 0; k < D; ++k)
                        RC(checked_lmax<T>(h, static_cast<const T*>(p->dRdv[k]), static_cast<const T*>(p->PC[k]), nn, labels[k], lmax[k]));
                    lmax_g = *std::max_element(lmax, lmax + D);
                }
                for (int k = 0; k < D; ++k) { dtau[k] = 2 / std::sqrt(lmax[k]) * cfl; cheb(dtau[k], lmin[k], cf, alpha[k], beta[k]); }
            }
            if (iter > c->max_iterations) break;
        }
        CK(launch_pressure_update<T>(static_cast<T*>(p->P), static_cast<const T*>(p->gammaP), static_cast<const T*>(p->RP),
                                     static_cast<const T*>(p->M_P), nP, h->stream));
        if (iter > c->max_iterations) break;
    }
    CK(cudaStreamSynchronize(h->stream));
    st->itPH = itPH_done; st->iter = iter; st->err = err; st->err_abs = err_abs; st->err_rel = err_rel;
    st->err_v = err_v; st->err_P = err_P; st->converged = converged; st->reached_total_iter = iter > c->max_iterations;
    st->lambda_max = *std::max_element(lmax, lmax + D); st->lambda_max_gershgorin = lmax_g;
    st->jacobian_assemblies = jac_assemblies;
    st->history_len = c->history ? std::min<int64_t>(hist, c->history_capacity) : 0;
    st->err_T = cp ? ti.err : 0.0; st->thermal_iterations = ti.iter;
    return FEMB200_OK;
}

// ---- mixed precision: FP32 Chebyshev iterations on increments, FP64 outer steps ----
//
// The solve runs the DR iteration of solve_dyrel with one change in how the
// residual is evaluated. At every Powell–Hestenes step the FP32 increments
// (δv, δP) are folded into the caller's FP64 state and an FP64 sweep gives the
// outer convergence test exactly as the plain solve computes it; a second FP64
// sweep (with Pnum) gives the base residual R_k and stores the trial stress and
// yield value of every integration point in FP32. The Chebyshev iterations then
// update δ in FP32 against R_k + [R(x_k + δ) − R(x_k)], whose bracket the
// incremental sweep forms from δ alone, so that FP32 rounding scales with the
// increment (and, late in the solve, with the small residual) rather than with
// the state. The Jacobian diagnostics (λmax and the preconditioner) run in FP32 on
// the FP32 image of x_k + δ. FP64 is used for every norm and convergence test,
// the outer residual, and the return map of points near the yield-surface apex.

int ensure_mixed(femb200_handle* h, const femb200_stokes_problem* p) {
    auto& m = h->mixed;
    const size_t nn = p->nnodes, nP = p->nnodesP, nip = (size_t)p->nq * p->nels;
    const bool ip = p->tau_old_layout == FEMB200_FIELD_IP;
    std::vector<std::pair<float**, size_t>> parts;
    for (int c = 0; c < 3; ++c)
        for (float** a : {&m.dv[c], &m.rate[c], &m.R[c], &m.R0[c], &m.Rk[c], &m.dRdv[c], &m.PC[c], &m.v32[c]})
            parts.push_back({a, c < p->dim ? nn : 0});
    for (float** a : {&m.dP, &m.RP, &m.RPk, &m.gP, &m.MP, &m.P32}) parts.push_back({a, nP});
    parts.push_back({&m.P0, p->P0 ? nP : 0});
    parts.push_back({&m.T, p->T ? nP : 0});
    parts.push_back({&m.T0, p->T0 ? nP : 0});
    parts.push_back({&m.Pf, p->Pf ? nP : 0});
    const size_t nslots = ((size_t)p->nels + 31) / 32 * 32;
    parts.push_back({&m.base, nslots * 27 * BASE_FIELDS});
    parts.push_back({reinterpret_cast<float**>(&m.el2n_t), nslots * 27});
    parts.push_back({reinterpret_cast<float**>(&m.dofs_t), nslots * 4});
    parts.push_back({reinterpret_cast<float**>(&m.phase_t), nslots * 2});
    parts.push_back({&m.geo_t, nslots * 10});
    parts.push_back({&m.eta_t, p->viscosity_ip ? nslots * 27 : 0});
    parts.push_back({&m.pscale_t, nslots * 4});
    parts.push_back({&m.RPinc, nP});
    for (int c = 0; c < 6; ++c) parts.push_back({&m.told[c], ip && p->tau_old[c] ? nip : 0});
    parts.push_back({&m.eta, p->viscosity_ip ? nip : 0});
    parts.push_back({&m.geo, (size_t)p->nels * 10});
    auto al = [](size_t n) { return (n * sizeof(float) + 255) / 256 * 256; };
    size_t total = 0;
    for (auto& pr : parts) total += al(pr.second);
    if (total > m.cap) {
        if (m.mem) cudaFree(m.mem);
        m.mem = nullptr; m.cap = 0;
        CK(cudaMalloc(&m.mem, total));
        m.cap = total;
    }
    char* b = static_cast<char*>(m.mem);
    size_t off = 0;
    for (auto& pr : parts) {
        *pr.first = pr.second ? reinterpret_cast<float*>(b + off) : nullptr;
        off += al(pr.second);
    }
    return FEMB200_OK;
}

// Colours of the ordered scatter, for units of U consecutive elements (U = 32: the FP32
// sweep's tiles; U = 3: the warp groups of the pipelined sweep and of the Jacobian
// diagnostics), from the connectivity in tensor order (tn[27e + t], t = i + 3j + 9k,
// 0-based). Greedy in unit order: a unit takes the lowest colour that no earlier unit
// sharing one of its nodes holds. Inside a unit the kernels fold the ξ = −1 node of
// line L (t = 3L) of element e + 1 into the ξ = +1 node (t = 3L + 2) of element e when
// the two are one node; every other node of the unit must be distinct, so that within
// one colour every node receives at most one addition. Returns the units sorted by
// colour and the start of each colour (colours + 1 entries).
int colour_units(femb200_handle* h, const std::vector<int32_t>& tn, int64_t nels, int64_t nnodes, int U,
                 std::vector<int32_t>& order, std::vector<int64_t>& start) {
    const int64_t nunits = (nels + U - 1) / U;
    std::vector<uint64_t> used((size_t)nnodes, 0);
    std::vector<int64_t> seen((size_t)nnodes, -1);
    std::vector<int32_t> colour((size_t)nunits);
    std::vector<int32_t> nodes;
    nodes.reserve((size_t)27 * U);
    int ncol = 0;
    for (int64_t u = 0; u < nunits; ++u) {
        nodes.clear();
        uint64_t mask = 0;
        for (int64_t e = u * U; e < std::min<int64_t>((u + 1) * U, nels); ++e)
            for (int t = 0; t < 27; ++t) {
                const int32_t n = tn[(size_t)(27 * e + t)];
                if (n < 0 || n >= nnodes) {
                    h->err = "ordered scatter: node index out of range in the connectivity";
                    return FEMB200_EINVAL;
                }
                if (t % 3 == 0 && e > u * U && tn[(size_t)(27 * (e - 1) + t + 2)] == n) continue;
                if (seen[(size_t)n] == u) {
                    h->err = "ordered scatter needs consecutive elements whose only shared nodes are the ξ faces of "
                             "neighbouring elements within each unit of " + std::to_string(U) +
                             " elements (element " + std::to_string(e + 1) + " repeats a node of its unit)";
                    return FEMB200_EUNSUPPORTED;
                }
                seen[(size_t)n] = u;
                mask |= used[(size_t)n];
                nodes.push_back(n);
            }
        if (~mask == 0) {
            h->err = "ordered scatter: more than 64 colours";
            return FEMB200_EUNSUPPORTED;
        }
        const int c = __builtin_ctzll(~mask);
        colour[(size_t)u] = c;
        ncol = std::max(ncol, c + 1);
        for (int32_t n : nodes) used[(size_t)n] |= 1ull << c;
    }
    start.assign((size_t)ncol + 1, 0);
    for (int64_t u = 0; u < nunits; ++u) ++start[(size_t)colour[(size_t)u] + 1];
    for (int c = 0; c < ncol; ++c) start[(size_t)c + 1] += start[(size_t)c];
    order.assign((size_t)nunits, 0);
    std::vector<int64_t> fill(start.begin(), start.end() - 1);
    for (int64_t u = 0; u < nunits; ++u) order[(size_t)fill[(size_t)colour[(size_t)u]]++] = (int32_t)u;
    return FEMB200_OK;
}

// Uploads a unit order into a handle-owned device array, growing it when needed.
int upload_order(femb200_handle* h, const std::vector<int32_t>& order, int32_t*& d, size_t& cap) {
    if (cap < order.size()) {
        if (d) CK(cudaFree(d));
        d = nullptr;
        cap = 0;
        CK(cudaMalloc(&d, order.size() * sizeof(int32_t)));
        cap = order.size();
    }
    CK(cudaMemcpyAsync(d, order.data(), order.size() * sizeof(int32_t), cudaMemcpyHostToDevice, h->stream));
    return FEMB200_OK;
}

// The handle's ordered-scatter state is valid for the duration of one solve.
struct OrderedScope {
    femb200_handle* h;
    ~OrderedScope() { h->ordered_active = false; }
};

template <class TG>
int solve_dyrel_mixed(femb200_handle* h, const femb200_stokes_problem* p, const femb200_stokes_controls* c,
                      femb200_stokes_stats* st) {
    using T = double;
    const int D = p->dim;
    const int64_t nn = p->nnodes, nP = p->nnodesP;
    const double dt = c->dt;
    const int finite_K = c->finite_K;
    const bool freeze = c->freeze_jacobian < 0 ? (p->mat.plastic == 0) : (c->freeze_jacobian != 0);
    const int64_t nout = c->check_interval > 0 ? c->check_interval : 50;
    const double cfl = c->cfl_v > 0 ? c->cfl_v : 0.98, cf = c->c_fact > 0 ? c->c_fact : 0.9;
    static const char* labels[3] = {"stokes vx", "stokes vy", "stokes vz"};
    std::memset(st, 0, sizeof(*st));
    if (D != 3) { h->err = "the mixed-precision solve needs a 3-D Hex27 mesh"; return FEMB200_EUNSUPPORTED; }
    if (!p->RP || !p->M_P || !p->gammaP || !p->Pnum) { h->err = "RP, M_P, γP and Pnum are required"; return FEMB200_EINVAL; }
    if (p->P_old && p->P_old_layout == FEMB200_FIELD_IP) { h->err = "the mixed-precision solve takes P_old on pressure DoFs"; return FEMB200_EUNSUPPORTED; }

    RC(upload_material(h, p->mat, finite_K, dt));
    RC((prepare_geometry<T, TG>(h, p)));
    if (!h->geo_c_valid) { h->err = "the mixed-precision solve needs affine (parallelepiped) Hex27 elements"; return FEMB200_EUNSUPPORTED; }
    // the FP64 outer sweeps are timed apart from the FP32 incremental sweeps
    struct SweepClass {
        femb200_handle* h;
        ~SweepClass() { h->prof_sweep = FEMB200_PROF_RESIDUAL; }
    } restore{h};
    h->prof_sweep = FEMB200_PROF_OUTER;
    RC(build_mask(h, p));
    RC(ensure_mixed(h, p));
    auto& m = h->mixed;
    cudaStream_t s = h->stream;
    const size_t nip = (size_t)p->nq * p->nels;
    CK(launch_compress_geometry<TG, float>(static_cast<const TG*>(p->geo_v), static_cast<const TG*>(p->geo_P), p->nels,
                                           m.geo, h->d_flag, s));
    CK(launch_round(m.gP, static_cast<const T*>(p->gammaP), nullptr, nP, s));
    CK(launch_round(m.MP, static_cast<const T*>(p->M_P), nullptr, nP, s));
    if (m.P0) CK(launch_round(m.P0, static_cast<const T*>(p->P0), nullptr, nP, s));
    if (m.T) CK(launch_round(m.T, static_cast<const T*>(p->T), nullptr, nP, s));
    if (m.T0) CK(launch_round(m.T0, static_cast<const T*>(p->T0), nullptr, nP, s));
    if (m.Pf) CK(launch_round(m.Pf, static_cast<const T*>(p->Pf), nullptr, nP, s));
    for (int k = 0; k < 6; ++k)
        if (m.told[k]) CK(launch_round(m.told[k], static_cast<const T*>(p->tau_old[k]), nullptr, (int64_t)nip, s));
    if (m.eta) CK(launch_round(m.eta, static_cast<const T*>(p->viscosity_ip), nullptr, (int64_t)nip, s));
    for (int k = 0; k < D; ++k) {
        CK(cudaMemsetAsync(m.dv[k], 0, sizeof(float) * nn, s));
        CK(cudaMemsetAsync(m.rate[k], 0, sizeof(float) * nn, s));
        CK(cudaMemsetAsync(m.R0[k], 0, sizeof(float) * nn, s));
    }
    CK(cudaMemsetAsync(m.dP, 0, sizeof(float) * nP, s));

    // FP32 image of x_k + δ for the Jacobian diagnostics
    femb200_stokes_problem pj = *p;
    pj.dtype = FEMB200_F32;
    for (int k = 0; k < 3; ++k) { pj.v[k] = m.v32[k]; pj.dRdv[k] = m.dRdv[k]; pj.PC[k] = m.PC[k]; }
    pj.P = m.P32; pj.P0 = m.P0; pj.T = m.T; pj.T0 = m.T0; pj.Pf = m.Pf; pj.gammaP = m.gP; pj.M_P = m.MP;
    for (int k = 0; k < 6; ++k) pj.tau_old[k] = m.told[k];
    pj.viscosity_ip = m.eta;
    double lmax[3] = {0, 0, 0};
    int64_t jac_assemblies = 0;
    auto jacobian32 = [&]() -> int {
        for (int k = 0; k < D; ++k) CK(launch_round(m.v32[k], static_cast<const T*>(p->v[k]), m.dv[k], nn, s));
        CK(launch_round(m.P32, static_cast<const T*>(p->P), m.dP, nP, s));
        RC((jacobian_sweep<float, TG>(h, &pj, dt)));
        ++jac_assemblies;
        for (int k = 0; k < D; ++k) RC(checked_lmax<float>(h, m.dRdv[k], m.PC[k], nn, labels[k], lmax[k]));
        return FEMB200_OK;
    };

    // incremental FP32 sweep: v, P are δv, δP; Rv starts from R_k
    femb200_stokes_problem pi = *p;
    pi.dtype = FEMB200_F32; pi.geo_dtype = FEMB200_F32; pi.geo_v = nullptr; pi.geo_P = nullptr;
    for (int k = 0; k < 3; ++k) { pi.v[k] = m.dv[k]; pi.Rv[k] = m.R[k]; pi.tau_old[k] = nullptr; pi.tau_old[k + 3] = nullptr; }
    pi.P = m.dP; pi.P0 = nullptr; pi.P_old = nullptr; pi.T = nullptr; pi.T0 = nullptr; pi.Q = nullptr; pi.Pf = nullptr;
    pi.gammaP = m.gP; pi.M_P = m.MP; pi.RP = m.RP; pi.viscosity_ip = m.eta;
    H27Args<float, float> ai = residual_args<float, float>(&pi, dt);
    ai.with_pnum = 1; ai.do_momentum = 1; ai.write_RP = 1; ai.Pnum_out = nullptr;
    ai.base_in = m.base;
    ai.RP_base = m.RPk;
    // the thread-per-element sweep, on meshes whose elements each carry one phase
    IncrArgs at;
    std::memset(&at, 0, sizeof(at));
    at.el2n_t = m.el2n_t; at.dofs_t = m.dofs_t; at.geo_t = m.geo_t; at.phase_t = m.phase_t; at.base_t = m.base;
    at.eta_t = m.eta ? m.eta_t : nullptr;
    at.pscale_t = m.pscale_t;
    for (int k = 0; k < 3; ++k) { at.dv[k] = m.dv[k]; at.R[k] = m.R[k]; at.g[k] = (float)p->mat.g[k]; }
    at.dP = m.dP; at.RPinc = m.RPinc;
    at.stress_reads = h->prof ? h->d_counters + FEMB200_COUNTER_STRESS_READS : nullptr;
    if (!h->d_bound) {
        CK(cudaMalloc(&h->d_bound, 2 * sizeof(unsigned long long)));
        CK(cudaMallocHost(&h->h_bound, 2 * sizeof(unsigned long long)));
    }
    CK(cudaMemsetAsync(h->d_bound, 0, 2 * sizeof(unsigned long long), s));
    at.bound_failures = h->d_bound;
    at.err_flag = reinterpret_cast<int*>(h->d_bound + 1);
    at.prefetch_stress = h->incr_pre;
    int64_t sweeps_since_check = 0;
    at.nels = p->nels;
    at.plastic = p->mat.plastic;
    {
        bool all_inf = true;
        for (int i = 0; i < p->mat.nphases; ++i) all_inf = all_inf && std::isinf(finite_K ? p->mat.K[i] : p->mat.eta_b[i]);
        for (int i = 0; i < FEMB200_MAX_PHASES; ++i) {
            const femb200_stokes_material& mt = p->mat;
            const double invG = 1.0 / mt.G[i];
            const double etave = 1.0 / (1.0 / mt.eta[i] + invG / dt);
            const double rest = mt.eta_reg[i] + mt.Kb[i] * dt * (-mt.sin_psi[i]) * (-mt.sin_phi[i]);
            IncrPhase& q = at.ph[i];
            q.twoe = (float)(2 * etave);
            q.rho0beta = (float)(mt.rho0[i] / mt.K[i]);
            q.cC = (float)(mt.cos_phi[i] * mt.C[i]);
            q.sphi = (float)mt.sin_phi[i];
            q.inv_den = (float)(1.0 / (etave + rest));
            q.invbulkdt = all_inf ? 0.0f : (float)(1.0 / ((finite_K ? mt.K[i] : mt.eta_b[i]) * dt));
            q.invG_dt = (float)(invG / dt);
            q.den_rest = (float)rest;
        }
    }
    {
        IncrTileSrc ts;
        ts.el2n = p->el2n; ts.dofsP = p->dofsP; ts.geo_c = m.geo; ts.eta = m.eta; ts.gP = m.gP; ts.MP = m.MP;
        ts.phv = p->phases_v; ts.phv_layout = p->phases_v_layout;
        ts.php = p->phases_P; ts.php_layout = p->phases_P_layout;
        ts.nphases = p->mat.nphases;
        CK(cudaMemsetAsync(m.base, 0, sizeof(float) * ((size_t)p->nels + 31) / 32 * 32 * 27 * BASE_FIELDS, s));
        CK(cudaMemsetAsync(h->d_flag, 0, sizeof(int), s));
        CK(launch_incr_tiles(ts, p->nels, at, h->d_flag, s));
        CK(cudaMemcpyAsync(h->h_flag, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
    }
    const bool thread_sweep = (*h->h_flag & INCR_MIXED_PHASES) == 0 && h->use_incr_thread;
    at.dofs_linear = (*h->h_flag & INCR_DOFS_GENERAL) == 0;
    at.diag_geometry = (*h->h_flag & INCR_GEOMETRY_FULL) == 0;
    // ordered scatter: every sweep and Jacobian assembly of this solve adds to each node
    // at most once per launch (colours of tiles and of warp groups)
    OrderedScope ordered_scope{h};
    // programmatic dependent launch of the sweep and the node update where every warp of
    // the sweep takes at most one tile (measured: 10 % faster at 32³, 2 % slower at 64³)
    const bool pdl = thread_sweep && (p->nels + 31) / 32 <= incr_warp_slots(h->num_sms);
    const bool ordered = h->ordered_scatter != 0;
    if (ordered) {
        if (!thread_sweep || !h->geo_c_valid) {
            h->err = "ordered scatter needs the thread-per-element FP32 sweep and the pipelined FP64 sweep "
                     "(one phase per cell, affine elements)";
            return FEMB200_EUNSUPPORTED;
        }
        std::vector<int32_t> el2n_h((size_t)p->nels * 27);
        CK(cudaMemcpyAsync(el2n_h.data(), p->el2n, el2n_h.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        int tn3[27];
        for (int a3 = 0; a3 < 27; ++a3) tn3[(H27[a3][0] + 1) + 3 * (H27[a3][1] + 1) + 9 * (H27[a3][2] + 1)] = a3;
        std::vector<int32_t> tn(el2n_h.size());
        for (int64_t e = 0; e < p->nels; ++e)
            for (int t = 0; t < 27; ++t) tn[(size_t)(27 * e + t)] = el2n_h[(size_t)(27 * e + tn3[t])] - 1;
        std::vector<int32_t> order;
        RC(colour_units(h, tn, p->nels, p->nnodes, 32, order, h->tile_colour_start));
        RC(upload_order(h, order, h->d_tile_list, h->tile_list_cap));
        RC(colour_units(h, tn, p->nels, p->nnodes, 3, order, h->group_colour_start));
        RC(upload_order(h, order, h->d_group_list, h->group_list_cap));
        CK(cudaStreamSynchronize(s));
        h->ordered_active = true;
    }
    // the thread-per-element sweep writes the increment of RP; RP itself is formed
    // where it is read (checks and the Powell–Hestenes pressure update)
    auto form_RP = [&]() -> int {
        if (thread_sweep) CK(launch_add_f32(m.RP, m.RPk, m.RPinc, nP, s));
        return FEMB200_OK;
    };
    auto incr_sweep = [&](bool prefilled) -> int {
        if (!prefilled)
            for (int k = 0; k < D; ++k) CK(launch_copy<float>(m.R[k], m.Rk[k], nn, s));
        RC(prof_begin(h, FEMB200_PROF_RESIDUAL));
        ++sweeps_since_check;
        if (thread_sweep && ordered) {
            // one launch per tile colour, in colour order: each node receives at most one
            // addition per launch, so the increments do not depend on the atomics' order
            for (size_t c = 0; c + 1 < h->tile_colour_start.size(); ++c) {
                at.tile_list = h->d_tile_list + h->tile_colour_start[c];
                at.tile_count = h->tile_colour_start[c + 1] - h->tile_colour_start[c];
                CK(launch_hex27_incr(at, h->num_sms, s, pdl));
            }
            at.tile_list = nullptr;
            at.tile_count = 0;
        } else if (thread_sweep) CK(launch_hex27_incr(at, h->num_sms, s, pdl));
        else CK(launch_hex27_residual_incr(ai, m.geo, h->num_sms, s));
        RC(prof_end(h, FEMB200_PROF_RESIDUAL));
        return FEMB200_OK;
    };
    auto apply_bc_R = [&]() -> int {
        for (int k = 0; k < D; ++k) {
            if (p->body_force[k]) CK(launch_sub<T>(static_cast<T*>(p->Rv[k]), static_cast<const T*>(p->body_force[k]), nn, s));
            if (p->bc_n[k] > 0) CK(launch_dirichlet<T>(static_cast<T*>(p->Rv[k]), p->bc_dofs[k], nullptr, p->bc_n[k], s));
        }
        return FEMB200_OK;
    };
    // FP64 base sweep at x_k (with Pnum): R_k, RP_k and the per-point base data
    int64_t base_sweeps = 0;
    auto base_sweep = [&]() -> int {
        H27Args<T, TG> a = residual_args<T, TG>(p, dt);
        a.with_pnum = 1; a.do_momentum = 1; a.write_RP = 1;
        a.Pnum_out = static_cast<T*>(p->Pnum);
        a.base_out = m.base;
        RC((launch_residual<T, TG>(h, p, a)));
        RC(apply_bc_R());
        for (int k = 0; k < D; ++k) CK(launch_round(m.Rk[k], static_cast<const T*>(p->Rv[k]), nullptr, nn, s));
        CK(launch_round(m.RPk, static_cast<const T*>(p->RP), nullptr, nP, s));
        ++base_sweeps;
        return FEMB200_OK;
    };
    // x_k += δ, then the Dirichlet values on v (DR.jl:697): δ is pinned to zero on the
    // constrained DoFs, so the base state carries the boundary values from here on
    auto fold = [&]() -> int {
        for (int k = 0; k < D; ++k) {
            CK(launch_fold(static_cast<T*>(p->v[k]), m.dv[k], nn, s));
            if (p->bc_n[k] > 0)
                CK(launch_dirichlet<T>(static_cast<T*>(p->v[k]), p->bc_dofs[k], static_cast<const T*>(p->bc_vals[k]),
                                       p->bc_n[k], s));
        }
        CK(launch_fold(static_cast<T*>(p->P), m.dP, nP, s));
        return FEMB200_OK;
    };

    RC(jacobian32());
    double lmax_g = *std::max_element(lmax, lmax + D);
    double alpha[3] = {0, 0, 0}, beta[3] = {0, 0, 0}, dtau[3];
    for (int k = 0; k < D; ++k) { dtau[k] = 2 / std::sqrt(lmax[k]) * cfl; cheb(dtau[k], 0.0, cf, alpha[k], beta[k]); }

    double err_min = INFINITY, eps = c->tolerance;
    double err = 2 * eps, err_abs = INFINITY, err_rel = INFINITY;
    double err_v0 = 1.0, err_P0 = 1.0, err_v00 = 1.0, err_v = INFINITY, err_P = INFINITY;
    int64_t iter = 0, itPH_done = 0, hist = 0;
    bool converged = false;
    double rel_drop = c->rel_drop0;
    const double sq_nn = std::sqrt((double)nn), sq_nP = std::sqrt((double)nP);
    auto push_hist = [&](double it, double ev, double eP, const double* comps) {
        if (c->history && hist < c->history_capacity) {
            double* hh = c->history + hist * (4 + D);
            hh[0] = it; hh[1] = ev; hh[2] = eP; hh[3] = 0;
            for (int k = 0; k < D; ++k) hh[4 + k] = comps[k];
        }
        ++hist;
    };
    const int nb = red_blocks(h, nn);
    RC(ensure_partials(h, std::max(nb, red_blocks(h, nP))));

    for (int64_t itPH = 1; itPH <= c->max_ph_iterations; ++itPH) {
        itPH_done = itPH;
        RC(fold());
        RC((residual_sweep<T, TG>(h, p, dt, 0, 1, 1)));
        RC(apply_bc_R());
        double sP;
        RC(sumsq<T>(h, static_cast<const T*>(p->RP), static_cast<const T*>(p->M_P), nP, sP));
        err_P = std::sqrt(sP) / sq_nP;
        double comps[3] = {0, 0, 0};
        err_v = 0;
        for (int k = 0; k < D; ++k) {
            double sv;
            RC(sumsq<T>(h, static_cast<const T*>(p->Rv[k]), (const T*)nullptr, nn, sv));
            comps[k] = std::sqrt(sv) / (2 * sq_nn);
            err_v = jl_max(err_v, std::sqrt(sv));
        }
        err_v /= 2 * sq_nn;
        push_hist((double)iter, err_v, err_P, comps);
        if (itPH == 1) { err_P0 = err_P + julia_eps(err_P); err_v0 = err_v + julia_eps(err_v); }
        else if (itPH == 2) err_P0 = err_P + julia_eps(err_P);
        err_abs = jl_max(err_v, err_P);
        err_rel = jl_max(err_v / err_v0, err_P / err_P0);
        err = jl_min(err_abs, err_rel);
        if (std::isnan(err)) { char b[96]; std::snprintf(b, sizeof b, "NaN detected in outer loop at PH=%lld", (long long)itPH); h->err = b; return FEMB200_ENAN; }
        if (err > 1e10) { char b[96]; std::snprintf(b, sizeof b, "Kaboom! Error > 1e10 in outer loop at PH=%lld", (long long)itPH); h->err = b; return FEMB200_EKABOOM; }
        if (err < eps) { converged = true; break; }
        if (err > err_min * 1.05) rel_drop = std::max(rel_drop * 0.1, 1.0e-3);
        err_min = std::min(err_min, err);
        const double eps_vel = err * rel_drop;
        RC(base_sweep());
        int64_t itPT = 0;
        while (err > eps_vel && itPT <= c->iter_max) {
            ++itPT; ++iter;
            const bool do_check = iter % nout == 0;
            // after the first iteration of the step the previous node update has set
            // R = R_k for this sweep and, before a check, saved R0
            const bool fused = itPT > 1 && nout > 1;
            if (do_check && !fused)
                for (int k = 0; k < D; ++k) CK(launch_copy<float>(m.R0[k], m.R[k], nn, s));
            RC(incr_sweep(fused));
            NodeArgs<float> na;
            std::memset(&na, 0, sizeof(na));
            for (int k = 0; k < 3; ++k) {
                na.v[k] = m.dv[k]; na.rate[k] = m.rate[k]; na.Rv[k] = m.R[k]; na.Rv0[k] = m.R0[k]; na.PC[k] = m.PC[k];
                na.alpha[k] = -alpha[k]; na.beta[k] = beta[k]; na.lam_step[k] = alpha[k];
            }
            na.mask = h->d_mask; na.n = nn; na.dim = D;
            na.reduce = do_check ? 1 : 0;
            na.partials = h->d_partials;
            na.save_R0 = nout > 1 && (iter + 1) % nout == 0;
            na.fill = nout > 1;
            for (int k = 0; k < 3; ++k) na.Rfill[k] = m.Rk[k];
            RC(prof_begin(h, FEMB200_PROF_NODE));
            CK(launch_node_update<float>(na, nb, s, pdl));
            RC(prof_end(h, FEMB200_PROF_NODE));
            if (do_check) {
                double sr[RED_SLOTS];
                // the elastic-bound failures of the sweeps since the last check travel with
                // the check's own synchronisation
                CK(cudaMemcpyAsync(h->h_bound, h->d_bound, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
                RC(fetch_sums(h, nb, RED_SLOTS, sr));
                if (h->h_bound[1] != 0) {
                    h->err = "the FP32 sweep gave up waiting for a bulk copy of its tile data";
                    return FEMB200_ECUDA;
                }
                if (thread_sweep && sweeps_since_check > 0) {
                    // prefetch the trial stresses while more than 1e-3 of the points need them
                    const double pts = (double)sweeps_since_check * 27.0 * (double)p->nels;
                    h->incr_pre = (double)*h->h_bound > 1e-3 * pts ? 1 : 0;
                    at.prefetch_stress = h->incr_pre;
                    CK(cudaMemsetAsync(h->d_bound, 0, sizeof(unsigned long long), s));
                    sweeps_since_check = 0;
                }
                double ev = 0, cmp[3] = {0, 0, 0};
                for (int k = 0; k < D; ++k) { ev = jl_max(ev, std::sqrt(sr[3 * k])); cmp[k] = std::sqrt(sr[3 * k]) / (2 * sq_nn); }
                ev /= 2 * sq_nn;
                if (iter == nout) err_v00 = ev + julia_eps(ev);
                err = ev <= eps ? ev : jl_max(ev / err_v00, ev);
                if (std::isnan(err)) { char b[96]; std::snprintf(b, sizeof b, "NaN detected in inner loop PH=%lld PT=%lld", (long long)itPH, (long long)itPT); h->err = b; return FEMB200_ENAN; }
                if (err > 1e10) { char b[96]; std::snprintf(b, sizeof b, "Kaboom! Error > 1e10 in inner loop PH=%lld PT=%lld", (long long)itPH, (long long)itPT); h->err = b; return FEMB200_EKABOOM; }
                if (c->history) {
                    double sPc;
                    RC(form_RP());
                    RC(sumsq<float>(h, m.RP, m.MP, nP, sPc));
                    push_hist((double)iter, ev, std::sqrt(sPc) / sq_nP, cmp);
                } else {
                    ++hist;
                }
                double lmin[3];
                for (int k = 0; k < D; ++k) lmin[k] = sr[3 * k + 1] == 0 ? 0.0 : std::fabs(sr[3 * k + 2]) / sr[3 * k + 1];
                if (!freeze) {
                    RC(jacobian32());
                    lmax_g = *std::max_element(lmax, lmax + D);
                }
                for (int k = 0; k < D; ++k) { dtau[k] = 2 / std::sqrt(lmax[k]) * cfl; cheb(dtau[k], lmin[k], cf, alpha[k], beta[k]); }
            }
            if (iter > c->max_iterations) break;
        }
        RC(form_RP());
        CK(launch_pressure_update<float>(m.dP, m.gP, m.RP, m.MP, nP, s));
        if (iter > c->max_iterations) break;
    }
    RC(fold());
    CK(cudaStreamSynchronize(s));
    st->itPH = itPH_done; st->iter = iter; st->err = err; st->err_abs = err_abs; st->err_rel = err_rel;
    st->err_v = err_v; st->err_P = err_P; st->converged = converged; st->reached_total_iter = iter > c->max_iterations;
    st->lambda_max = *std::max_element(lmax, lmax + D); st->lambda_max_gershgorin = lmax_g;
    st->jacobian_assemblies = jac_assemblies;
    st->defect_corrections = base_sweeps;
    st->history_len = c->history ? std::min<int64_t>(hist, c->history_capacity) : 0;
    return FEMB200_OK;
}

int finish_solve(femb200_handle* h, const femb200_stokes_controls* c, femb200_stokes_stats* st) {
    if (!st->converged && c->throw_on_failure) {
        char b[256];
        std::snprintf(b, sizeof b, "Stokes solve did not converge after %lld iterations (residual = %g, tolerance = %g)",
                      (long long)st->iter, st->err_abs, c->tolerance);
        h->err = b;
        return FEMB200_ENOTCONV;
    }
    return FEMB200_OK;
}

// dtype dispatch
template <template <class, class> class F, class... Args>
int dispatch(const femb200_stokes_problem* p, Args&&... args) {
    if (p->dtype == FEMB200_F64 && p->geo_dtype == FEMB200_F64) return F<double, double>::run(args...);
    if (p->dtype == FEMB200_F32 && p->geo_dtype == FEMB200_F32) return F<float, float>::run(args...);
    if (p->dtype == FEMB200_F64 && p->geo_dtype == FEMB200_F32) return F<double, float>::run(args...);
    return F<float, double>::run(args...);
}

template <class T, class TG> struct DoResidual {
    static int run(femb200_handle* h, const femb200_stokes_problem* p, double dt, int with_pnum, int do_momentum, int write_RP) {
        RC((prepare_geometry<T, TG>(h, p)));
        return residual_sweep<T, TG>(h, p, dt, with_pnum, do_momentum, write_RP);
    }
};
template <class T, class TG> struct DoMomentum {
    // assemble_momentum_residual_kernel! with the caller's Pnum array (or none).
    static int run(femb200_handle* h, const femb200_stokes_problem* p, double dt, int with_pnum) {
        H27Args<T, TG> a = residual_args<T, TG>(p, dt);
        a.do_momentum = 1; a.write_RP = 0; a.with_pnum = with_pnum;
        a.Pnum_in = with_pnum ? static_cast<const T*>(p->Pnum) : nullptr;
        h->geo_c_valid = false;   // the pipelined sweep has no stored-Pnum input
        return launch_residual<T, TG>(h, p, a);
    }
};
template <class T, class TG> struct DoJacobian {
    static int run(femb200_handle* h, const femb200_stokes_problem* p, double dt) { return jacobian_sweep<T, TG>(h, p, dt); }
};
template <class T, class TG> struct DoScaling {
    static int run(femb200_handle* h, const femb200_stokes_problem* p, double g, double dt) { return pressure_scaling_impl<T, TG>(h, p, g, dt); }
};
template <class T, class TG> struct DoStore {
    static int run(femb200_handle* h, const femb200_stokes_problem* p, double dt) {
        H27Args<T, TG> a = residual_args<T, TG>(p, dt);
        const int nt = p->dim == 3 ? 6 : 3;
        for (int c = 0; c < nt; ++c) {
            if (!p->tau[c]) { h->err = "tau output components are required"; return FEMB200_EINVAL; }
            a.tau_store[c] = static_cast<T*>(p->tau[c]);
        }
        a.do_momentum = 1; a.write_RP = 0; a.with_pnum = 0;
        a.eta_ip = nullptr;   // update_stokes_current_stress! uses dr.η (DR.jl:890)
        RC((prepare_geometry<T, TG>(h, p)));
        return launch_residual<T, TG>(h, p, a);
    }
};
template <class T, class TG> struct DoShear {
    static int run(femb200_handle* h, const femb200_stokes_problem* p, double dt, void* phi) {
        h->geo_c_valid = false;
        return shear_heating_impl<T, TG>(h, p, dt, phi);
    }
};
template <class T, class TG> struct DoSolve {
    static int run(femb200_handle* h, const femb200_stokes_problem* p, const femb200_stokes_controls* c, femb200_stokes_stats* st, Coupled* cp) {
        if (c->assemble_scaling) {
            RC(upload_material(h, p->mat, c->finite_K, c->dt));
            RC((pressure_scaling_impl<T, TG>(h, p, c->pressure_factor, c->dt)));
        }
        if (c->precision == FEMB200_PRECISION_MIXED) {
            if (!std::is_same<T, double>::value) { h->err = "the mixed-precision solve takes an FP64 state"; return FEMB200_EUNSUPPORTED; }
            if (cp) { h->err = "the coupled solve runs in FP64 only"; return FEMB200_EUNSUPPORTED; }
            return solve_dyrel_mixed<TG>(h, p, c, st);
        }
        RC((solve_dyrel<T, TG>(h, p, c, st, cp)));
        return FEMB200_OK;
    }
};

// ---- adjoint ------------------------------------------------------------------

int check_adjoint_problem(femb200_handle* h, const femb200_stokes_problem* p) {
    RC(check_problem(h, p));
    if (p->dim != 3) { h->err = "the adjoint is implemented for 3-D Hex27/P1-disc meshes"; return FEMB200_EUNSUPPORTED; }
    if (p->dtype != FEMB200_F64 || p->geo_dtype != FEMB200_F64) { h->err = "the adjoint runs in FP64"; return FEMB200_EUNSUPPORTED; }
    if (p->tau_old_layout == FEMB200_FIELD_NODAL) { h->err = "the adjoint takes τ_old at integration points"; return FEMB200_EUNSUPPORTED; }
    if (p->P_old && p->P_old_layout == FEMB200_FIELD_IP) {
        // P_old enters only the storage term's constant part; its layout does not matter
    }
    return FEMB200_OK;
}

AdjArgs<double> adjoint_args(const femb200_stokes_problem* p, double dt, int with_pnum, const void* const lam_v[3],
                             const void* lam_P) {
    AdjArgs<double> a;
    std::memset(&a, 0, sizeof(a));
    a.el2n = p->el2n; a.dofsP = p->dofsP;
    a.geo_v = static_cast<const double*>(p->geo_v); a.geo_P = static_cast<const double*>(p->geo_P);
    for (int c = 0; c < 3; ++c) { a.v[c] = static_cast<const double*>(p->v[c]); a.lam_v[c] = static_cast<const double*>(lam_v[c]); }
    a.P = static_cast<const double*>(p->P);
    a.Pf = static_cast<const double*>(p->Pf);
    a.gammaP = static_cast<const double*>(p->gammaP);
    a.MP = static_cast<const double*>(p->M_P);
    a.phv = p->phases_v; a.phv_layout = p->phases_v_layout;
    a.php = p->phases_P; a.php_layout = p->phases_P_layout;
    for (int c = 0; c < 6; ++c)
        a.told[c] = p->tau_old_layout == FEMB200_FIELD_IP ? static_cast<const double*>(p->tau_old[c]) : nullptr;
    a.eta_ip = static_cast<const double*>(p->viscosity_ip);
    a.lam_P = static_cast<const double*>(lam_P);
    a.nels = p->nels;
    a.dt = dt;
    a.with_pnum = with_pnum && p->gammaP && p->M_P;
    return a;
}

// Adjoint PH/DYREL solve with the frozen operator (_solve_stokes_adjoint_dyrel!,
// src/stokes/solvers/DR_adjoint.jl:3-325): the velocity adjoint advances by the
// Chebyshev-accelerated damped iteration, the pressure adjoint by the
// Arrow–Hurwicz update λP += γP·ResλP/M_P, with the Gershgorin λmax of the
// augmented Jacobian diagnostics (the :matrix_free/:enzyme paths' λmax, :94-116).
struct AdjWork {
    void* mem = nullptr;
    size_t cap = 0;
};

int solve_adjoint_impl(femb200_handle* h, const femb200_stokes_problem* p, const femb200_stokes_controls* c,
                       const void* const objective_v[3], void* const lam_v[3], void* lam_P, femb200_stokes_stats* st) {
    using T = double;
    const int64_t nn = p->nnodes, nP = p->nnodesP;
    const double dt = c->dt;
    const int64_t ncheck = c->check_interval > 0 ? c->check_interval : 50;
    const double cfl = c->cfl_v > 0 ? c->cfl_v : 0.98, cf = c->c_fact > 0 ? c->c_fact : 0.9;
    const double tol = c->tolerance > 0 ? c->tolerance : 1e-6;
    const double rel_drop = c->rel_drop0 > 0 ? c->rel_drop0 : 0.1;
    const int64_t iter_max = c->iter_max > 0 ? c->iter_max : 50000;
    const int64_t total_max = c->max_iterations > 0 ? c->max_iterations : 50000;
    const int64_t max_ph = c->max_ph_iterations > 0 ? c->max_ph_iterations : 100;
    static const char* labels[3] = {"adjoint vx", "adjoint vy", "adjoint vz"};
    std::memset(st, 0, sizeof(*st));
    if (!p->dRdv[0] || !p->PC[0] || !p->gammaP || !p->M_P) { h->err = "dRdv, PC, γP and M_P are required"; return FEMB200_EINVAL; }
    cudaStream_t s = h->stream;
    RC(upload_material(h, p->mat, c->finite_K, dt));
    RC(build_mask(h, p));
    // workspace: λrate, Resλv, Resλv0 (3 each) and ResλP
    const size_t need = (9 * (size_t)nn + (size_t)nP) * sizeof(T);
    if (need > h->adj_cap) {
        if (h->adj_mem) cudaFree(h->adj_mem);
        h->adj_mem = nullptr; h->adj_cap = 0;
        CK(cudaMalloc(&h->adj_mem, need));
        h->adj_cap = need;
    }
    T* w = static_cast<T*>(h->adj_mem);
    T *rate[3], *Res[3], *Res0[3];
    for (int k = 0; k < 3; ++k) { rate[k] = w + k * nn; Res[k] = w + (3 + k) * nn; Res0[k] = w + (6 + k) * nn; }
    T* ResP = w + 9 * nn;
    for (int k = 0; k < 3; ++k) CK(cudaMemsetAsync(rate[k], 0, sizeof(T) * nn, s));
    // λ on the constrained velocity DoFs is zero
    for (int k = 0; k < 3; ++k)
        if (p->bc_n[k] > 0) CK(launch_dirichlet<T>(static_cast<T*>(lam_v[k]), p->bc_dofs[k], nullptr, p->bc_n[k], s));

    // Jacobi diagonal and Gershgorin row sums of the augmented Jacobian at the forward state
    RC((jacobian_sweep<T, T>(h, p, dt)));
    double lmax[3];
    for (int k = 0; k < 3; ++k) RC(checked_lmax<T>(h, static_cast<const T*>(p->dRdv[k]), static_cast<const T*>(p->PC[k]), nn, labels[k], lmax[k]));
    double dtau[3], alpha[3], beta[3];
    for (int k = 0; k < 3; ++k) { dtau[k] = 2 / std::sqrt(lmax[k]) * cfl; cheb(dtau[k], 0.0, cf, alpha[k], beta[k]); }

    const void* lv[3] = {lam_v[0], lam_v[1], lam_v[2]};
    AdjArgs<T> a = adjoint_args(p, dt, 1, lv, lam_P);
    for (int k = 0; k < 3; ++k) a.out_dv[k] = Res[k];
    a.out_dP = ResP;
    auto assemble = [&]() -> int {
        for (int k = 0; k < 3; ++k) CK(launch_copy<T>(Res[k], static_cast<const T*>(objective_v[k]), nn, s));
        RC(prof_begin(h, FEMB200_PROF_RESIDUAL));
        CK(launch_hex27_adjoint<T>(a, h->num_sms, s));
        RC(prof_end(h, FEMB200_PROF_RESIDUAL));
        for (int k = 0; k < 3; ++k)
            if (p->bc_n[k] > 0) CK(launch_dirichlet<T>(Res[k], p->bc_dofs[k], nullptr, p->bc_n[k], s));
        return FEMB200_OK;
    };
    const double sq_nn = std::sqrt((double)nn), sq_nP = std::sqrt((double)nP);
    auto velocity_error = [&](double& ev) -> int {
        ev = 0;
        for (int k = 0; k < 3; ++k) {
            double sv;
            RC(sumsq<T>(h, Res[k], (const T*)nullptr, nn, sv));
            ev = jl_max(ev, std::sqrt(sv));
        }
        ev /= sq_nn;
        return FEMB200_OK;
    };
    auto pressure_error = [&](double& ep) -> int {
        double sp;
        RC(sumsq<T>(h, ResP, (const T*)nullptr, nP, sp));
        ep = std::sqrt(sp) / sq_nP;
        return FEMB200_OK;
    };
    const int nb = red_blocks(h, nn);
    RC(ensure_partials(h, nb));

    int64_t iter = 0, itPH_done = 0;
    double err = INFINITY, err_v0 = 1.0, err_P0 = 1.0, err_v = INFINITY, err_P = INFINITY;
    bool converged = false;
    for (int64_t itPH = 1; itPH <= max_ph; ++itPH) {
        itPH_done = itPH;
        RC(assemble());
        RC(velocity_error(err_v));
        RC(pressure_error(err_P));
        if (itPH == 1) { err_v0 = err_v + julia_eps(err_v); err_P0 = err_P + julia_eps(err_P); }
        err = jl_max(jl_min(err_v, err_v / err_v0), jl_min(err_P, err_P / err_P0));
        if (std::isnan(err)) { h->err = "NaN detected in the adjoint solve"; return FEMB200_ENAN; }
        if (err < tol) { converged = true; break; }
        const double target_v = jl_max(err_v * rel_drop, tol);
        int64_t inner = 0;
        while (err_v > target_v && inner < iter_max && iter < total_max) {
            ++inner; ++iter;
            NodeArgs<T> na;
            std::memset(&na, 0, sizeof(na));
            for (int k = 0; k < 3; ++k) {
                na.v[k] = static_cast<T*>(lam_v[k]); na.rate[k] = rate[k]; na.Rv[k] = Res[k]; na.Rv0[k] = Res0[k];
                na.PC[k] = static_cast<const T*>(p->PC[k]);
                na.alpha[k] = -alpha[k]; na.beta[k] = beta[k];
            }
            na.mask = h->d_mask; na.n = nn; na.dim = 3;
            na.save_R0 = 1;
            RC(prof_begin(h, FEMB200_PROF_NODE));
            CK(launch_node_update<T>(na, nb, s));
            RC(prof_end(h, FEMB200_PROF_NODE));
            RC(assemble());
            if (iter % ncheck == 0) {
                RC(velocity_error(err_v));
                if (std::isnan(err_v)) { h->err = "NaN detected in the adjoint solve"; return FEMB200_ENAN; }
                // λmin from the change of the residual over the last step (_stokes_λmin, DR.jl:32-37)
                for (int k = 0; k < 3; ++k) {
                    CK(launch_lmin_sums<T>(rate[k], Res[k], Res0[k], static_cast<const T*>(p->PC[k]), nn, alpha[k],
                                           h->d_partials, nb, s));
                    double r[3];
                    RC(fetch_sums(h, nb, 3, r));
                    const double lmin = r[0] == 0 ? 0.0 : std::fabs(r[1]) / r[0];
                    cheb(dtau[k], lmin, cf, alpha[k], beta[k]);
                }
            }
        }
        // Arrow–Hurwicz update of the pressure adjoint (DR_adjoint.jl:296)
        CK(launch_pressure_update<T>(static_cast<T*>(lam_P), static_cast<const T*>(p->gammaP), ResP,
                                     static_cast<const T*>(p->M_P), nP, s));
        if (iter >= total_max) break;
    }
    if (!converged) {
        RC(assemble());
        RC(velocity_error(err_v));
        RC(pressure_error(err_P));
        err = jl_max(jl_min(err_v, err_v / err_v0), jl_min(err_P, err_P / err_P0));
    }
    CK(cudaStreamSynchronize(s));
    st->itPH = itPH_done; st->iter = iter; st->err = err; st->err_v = err_v; st->err_P = err_P;
    st->converged = converged || err < tol;
    st->reached_total_iter = iter >= total_max;
    st->lambda_max = *std::max_element(lmax, lmax + 3);
    st->lambda_max_gershgorin = st->lambda_max;
    st->jacobian_assemblies = 1;
    return FEMB200_OK;
}

int check_controls(femb200_handle* h, const femb200_stokes_controls* c) {
    if (!c) { h->err = "null controls"; return FEMB200_EINVAL; }
    if (!(c->dt > 0)) { h->err = "dt must be positive"; return FEMB200_EINVAL; }
    if (c->check_interval <= 0) { h->err = "check_interval must be positive"; return FEMB200_EINVAL; }
    if (c->precision != FEMB200_PRECISION_FP64 && c->precision != FEMB200_PRECISION_MIXED) { h->err = "unknown precision"; return FEMB200_EINVAL; }
    return FEMB200_OK;
}

}  // namespace

namespace {
int check_cp_problem(femb200_handle* h, const femb200_cell_pressure_problem* p) {
    if (!h) return FEMB200_EINVAL;
    if (!p) { h->err = "null problem"; return FEMB200_EINVAL; }
    if (p->nels <= 0 || p->nnodes <= 0) { h->err = "empty mesh"; return FEMB200_EINVAL; }
    if (p->nphases < 1 || p->nphases > FEMB200_MAX_PHASES) { h->err = "nphases must lie in 1:16"; return FEMB200_EINVAL; }
    if (!p->el2n || !p->geo_v || !p->phases || !p->P || !p->RP || !p->pressure_mass) {
        h->err = "mesh, phase, pressure and scratch arrays are required";
        return FEMB200_EINVAL;
    }
    for (int c = 0; c < 3; ++c)
        if (!p->v[c] || !p->Rv[c] || !p->diagonal[c] || (p->bc_n[c] > 0 && !p->bc_dofs[c]) || p->bc_n[c] < 0) {
            h->err = "velocity, residual and preconditioner components are required";
            return FEMB200_EINVAL;
        }
    return FEMB200_OK;
}

CpArgs cp_args(const femb200_cell_pressure_problem* p) {
    CpArgs a;
    std::memset(&a, 0, sizeof(a));
    a.nels = p->nels;
    a.el2n = p->el2n;
    a.geo_v = p->geo_v;
    a.phases = p->phases;
    for (int k = 0; k < FEMB200_MAX_PHASES; ++k) { a.eta[k] = p->eta[k]; a.rho[k] = p->rho[k]; }
    for (int c = 0; c < 3; ++c) {
        a.g[c] = p->g[c];
        a.v[c] = p->v[c];
        a.Rv[c] = p->Rv[c];
        a.diagonal[c] = p->diagonal[c];
    }
    a.P = p->P;
    a.RP = p->RP;
    a.pressure_mass = p->pressure_mass;
    return a;
}

// The device checks of the connectivity and the phases (one synchronisation).
int cp_validate(femb200_handle* h, const femb200_cell_pressure_problem* p) {
    if (!h->d_flag) {
        CK(cudaMalloc(&h->d_flag, sizeof(int)));
        CK(cudaMallocHost(&h->h_flag, sizeof(int)));
    }
    CK(cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
    CK(launch_cp_validate(p->el2n, p->phases, p->nels, p->nnodes, p->nphases, h->d_flag, h->stream));
    CK(cudaMemcpyAsync(h->h_flag, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (*h->h_flag & 1) { h->err = "connectivity entry outside 1:nnodes"; return FEMB200_EINVAL; }
    if (*h->h_flag & 2) { h->err = "phases must lie in 1:nphases"; return FEMB200_EINVAL; }
    return FEMB200_OK;
}

int cp_preconditioner(femb200_handle* h, const femb200_cell_pressure_problem* p) {
    for (int c = 0; c < 3; ++c) CK(cudaMemsetAsync(p->diagonal[c], 0, sizeof(double) * p->nnodes, h->stream));
    CK(launch_cp_preconditioner(cp_args(p), h->num_sms, h->stream));
    return FEMB200_OK;
}

int cp_residuals(femb200_handle* h, const femb200_cell_pressure_problem* p, int which, const double* geo_c = nullptr,
                 bool rv_zeroed = false) {
    CpArgs a = cp_args(p);
    a.geo_c = geo_c;
    if (which & 1) CK(launch_cp_pressure_residual(a, h->num_sms, h->stream));
    if (which & 2) {
        if (!rv_zeroed)
            for (int c = 0; c < 3; ++c) CK(cudaMemsetAsync(p->Rv[c], 0, sizeof(double) * p->nnodes, h->stream));
        CK(launch_cp_momentum_residual(a, h->num_sms, h->stream));
    }
    return FEMB200_OK;
}

// solve_dynamic_relaxation! (src/dynamic_relaxation/solver.jl:61-122) for one nodal
// unknown u with a diagonal preconditioner: the thermal and lithostatic DR solves.
// `assemble(jac)` fills R (and on check iterations the Jacobian row sums and |diag|);
// the Dirichlet pins of R and the rate are folded into the update through `mask`.
struct DrNodal {
    double *u, *rate, *R, *R0;
    const double *dRdu, *PC;
    int64_t n;
    const int32_t* bc_dofs;
    const double* bc_vals;
    int64_t bc_n;
    double cfl, c_fact;
};

template <class Asm>
int dr_nodal_solve(femb200_handle* h, const DrNodal& f, const uint8_t* mask, double tolerance, int64_t max_it,
                   int64_t check, int32_t throw_on_failure, const char* label, const char* title, Asm assemble,
                   femb200_thermal_stats* st) {
    using T = double;
    double a = 0, b = 0, nr0 = 0, last = NAN, lmax = 0;
    const int nbk = red_blocks(h, f.n);
    RC(ensure_partials(h, nbk));
    for (int64_t it = 1; it <= max_it; ++it) {
        const bool dj = (it % check == 0) || it == 1;
        if (dj) CK(launch_copy<T>(f.R0, f.R, f.n, h->stream));
        RC(assemble(dj));
        if (dj) RC(checked_lmax<T>(h, f.dRdu, f.PC, f.n, label, lmax));
        CK(launch_thermal_update<T>(f.u, f.rate, f.R, f.PC, mask, f.n, a, b, h->stream));
        if (f.bc_n > 0) CK(launch_dirichlet<T>(f.u, f.bc_dofs, f.bc_vals, f.bc_n, h->stream));
        if (dj) {
            const double dtau = 2 / std::sqrt(lmax) * f.cfl;
            CK(launch_lmin_sums<T>(f.rate, f.R, f.R0, f.PC, f.n, dtau, h->d_partials, nbk, h->stream));
            double s[3];
            RC(fetch_sums(h, nbk, 3, s));
            const double nr = std::sqrt(s[2]);
            if (it == 1) nr0 = std::max(nr, julia_eps(nr));
            if (std::isnan(nr / nr0)) { char bb[64]; std::snprintf(bb, sizeof bb, "NaNs at PT iter %lld", (long long)it); h->err = bb; return FEMB200_ENAN; }
            const double lmin = (it == 1 || s[0] == 0) ? 0.0 : std::fabs(s[1]) / s[0];
            cheb(dtau, lmin, f.c_fact, a, b);
            last = nr / nr0;
            if (last < tolerance) { st->converged = 1; st->iterations = it; st->residual = last; return FEMB200_OK; }
        }
    }
    st->converged = 0; st->iterations = max_it; st->residual = last;
    if (throw_on_failure) {
        char bb[256];
        std::snprintf(bb, sizeof bb, "%s DR solver did not converge after %lld pseudo-transient iterations (relative residual = %g)",
                      title, (long long)max_it, last);
        h->err = bb;
        return FEMB200_ENOTCONV;
    }
    return FEMB200_OK;
}

int build_node_mask(femb200_handle* h, const int32_t* dofs, int64_t bc_n, int64_t nnodes) {
    const size_t n = (size_t)nnodes;
    if (n > h->tmask_cap) {
        if (h->d_tmask) cudaFree(h->d_tmask);
        h->d_tmask = nullptr;
        CK(cudaMalloc(&h->d_tmask, n));
        h->tmask_cap = n;
    }
    CK(cudaMemsetAsync(h->d_tmask, 0, n, h->stream));
    if (bc_n > 0) CK(launch_build_mask(h->d_tmask, dofs, bc_n, 0, h->stream));
    return FEMB200_OK;
}

int check_litho_problem(femb200_handle* h, const femb200_lithostatic_problem* p) {
    if (!h) return FEMB200_EINVAL;
    if (!p) { h->err = "null problem"; return FEMB200_EINVAL; }
    const bool h27 = p->dim == 3 && p->nv == 27 && p->nq == 27, q9 = p->dim == 2 && p->nv == 9 && p->nq == 9;
    if (!h27 && !q9) { h->err = "lithostatic pressure: Hex27 (3-D) or Q9 (2-D) meshes"; return FEMB200_EUNSUPPORTED; }
    if (p->nels <= 0 || p->nnodes <= 0) { h->err = "empty mesh"; return FEMB200_EINVAL; }
    if (p->nphases < 1 || p->nphases > FEMB200_MAX_PHASES) { h->err = "nphases must lie in 1:16"; return FEMB200_EINVAL; }
    if (!p->el2n || !p->geo || !p->P || !p->rate || !p->R || !p->R0 || !p->dRdP || !p->PC || !p->phases ||
        (p->bc_n > 0 && !p->bc_dofs) || p->bc_n < 0) {
        h->err = "lithostatic pressure: mesh, state and phase arrays are required";
        return FEMB200_EINVAL;
    }
    return FEMB200_OK;
}

int litho_assemble(femb200_handle* h, const femb200_lithostatic_problem* p, double Tref, const double* g, bool jac) {
    LithoArgs a;
    std::memset(&a, 0, sizeof(a));
    a.dim = p->dim; a.el2n = p->el2n; a.geo = p->geo; a.P = p->P; a.Tn = p->T;
    a.ph = p->phases; a.ph_layout = p->phases_layout;
    a.R = p->R; a.dRdP = p->dRdP; a.PC = p->PC; a.nels = p->nels; a.Tref = Tref; a.jac = jac ? 1 : 0;
    for (int k = 0; k < p->dim; ++k) a.g[k] = g[k];
    for (int i = 0; i < FEMB200_MAX_PHASES; ++i) {
        a.rho0[i] = p->rho0[i]; a.alpha[i] = p->alpha[i]; a.beta[i] = 1.0 / p->K[i];   // β = 1/K: 0 for K = ∞
    }
    CK(cudaMemsetAsync(p->R, 0, sizeof(double) * p->nnodes, h->stream));
    if (jac) {
        CK(cudaMemsetAsync(p->dRdP, 0, sizeof(double) * p->nnodes, h->stream));
        CK(cudaMemsetAsync(p->PC, 0, sizeof(double) * p->nnodes, h->stream));
    }
    CK(launch_lithostatic(a, h->stream));
    return FEMB200_OK;
}

template <class T, class TG>
int strain_rate_stress_impl(femb200_handle* h, const femb200_stokes_problem* p, const void* const tau_ip[6],
                            void* const out[14]) {
    PostArgs<T, TG> a;
    std::memset(&a, 0, sizeof(a));
    a.el2n = p->el2n;
    a.geo_v = static_cast<const TG*>(p->geo_v);
    a.nels = p->nels;
    const int nt = p->dim == 3 ? 6 : 3, nf = p->dim == 3 ? 14 : 10;
    for (int c = 0; c < p->dim; ++c) a.v[c] = static_cast<const T*>(p->v[c]);
    for (int c = 0; c < nt; ++c) a.tau[c] = static_cast<const T*>(tau_ip[c]);
    for (int k = 0; k < nf; ++k) a.out[k] = static_cast<T*>(out[k]);
    CK(launch_strain_rate_stress<T, TG>(p->dim, a, h->stream));
    return FEMB200_OK;
}
}  // namespace

extern "C" {

int femb200_create(femb200_handle** out) {
    if (!out) return FEMB200_EINVAL;
    femb200_handle* h = new femb200_handle();
    cudaError_t e = cudaGetDevice(&h->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device);
    if (e != cudaSuccess) {
        delete h;
        *out = nullptr;
        return FEMB200_ECUDA;
    }
    int rc = ensure_tables(h);
    if (rc) { delete h; *out = nullptr; return rc; }
    // FEMB200_INCR_SWEEP=warp selects the warp-cooperative incremental sweep of the
    // mixed-precision solve (for comparisons); the default is thread-per-element
    if (const char* v = std::getenv("FEMB200_INCR_SWEEP")) h->use_incr_thread = std::strcmp(v, "warp") != 0;
    // FEMB200_JAC_SHARED=0 assembles every element's Jacobian columns (for comparisons)
    if (const char* v = std::getenv("FEMB200_JAC_SHARED")) h->jac_shared = std::strcmp(v, "0") != 0;
    // FEMB200_PDL=0 launches the inner iteration's kernels without programmatic dependent
    // launch (for comparisons; process-wide)
    if (const char* v = std::getenv("FEMB200_PDL")) g_pdl_enabled = std::strcmp(v, "0") != 0;
    *out = h;
    return FEMB200_OK;
}

int femb200_profile(femb200_handle* h, int32_t enable) {
    if (!h) return FEMB200_EINVAL;
    if (!h->d_counters) CK(cudaMalloc(&h->d_counters, sizeof(unsigned long long) * FEMB200_COUNTER_COUNT));
    CK(cudaMemsetAsync(h->d_counters, 0, sizeof(unsigned long long) * FEMB200_COUNTER_COUNT, h->stream));
    for (int k = 0; k < FEMB200_PROF_COUNT; ++k) {
        RC(prof_flush(h, k));
        h->prof_ms[k] = 0;
        h->prof_n[k] = 0;
    }
    h->prof = enable != 0;
    h->launches_at_reset = __atomic_load_n(&g_kernel_launches, __ATOMIC_RELAXED);
    return FEMB200_OK;
}

int femb200_profile_counters(femb200_handle* h, int64_t* out, int32_t n) {
    if (!h || !out || n < 0) return FEMB200_EINVAL;
    unsigned long long c[FEMB200_COUNTER_COUNT] = {};
    if (h->d_counters) {
        CK(cudaMemcpyAsync(c, h->d_counters, sizeof(c), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    for (int k = 0; k < n && k < FEMB200_COUNTER_COUNT; ++k) out[k] = (int64_t)c[k];
    return FEMB200_OK;
}

int femb200_profile_read(femb200_handle* h, double* ms, int64_t* launches) {
    if (!h || !ms || !launches) return FEMB200_EINVAL;
    for (int k = 0; k < FEMB200_PROF_COUNT; ++k) {
        RC(prof_flush(h, k));
        ms[k] = h->prof_ms[k];
        launches[k] = h->prof_n[k];
    }
    launches[FEMB200_PROF_ALL] = (int64_t)(__atomic_load_n(&g_kernel_launches, __ATOMIC_RELAXED) - h->launches_at_reset);
    return FEMB200_OK;
}

int femb200_destroy(femb200_handle* h) {
    if (!h) return FEMB200_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (int k = 0; k < FEMB200_PROF_COUNT; ++k)
        for (auto& e : h->ev_pool[k]) cudaEventDestroy(e);
    if (h->d_partials) cudaFree(h->d_partials);
    if (h->h_partials) cudaFreeHost(h->h_partials);
    if (h->d_mask) cudaFree(h->d_mask);
    if (h->d_tmask) cudaFree(h->d_tmask);
    if (h->d_cpmask) cudaFree(h->d_cpmask);
    if (h->d_geo_c) cudaFree(h->d_geo_c);
    if (h->d_flag) cudaFree(h->d_flag);
    if (h->h_flag) cudaFreeHost(h->h_flag);
    if (h->d_counters) cudaFree(h->d_counters);
    if (h->d_bound) cudaFree(h->d_bound);
    if (h->h_bound) cudaFreeHost(h->h_bound);
    if (h->d_conv_err) cudaFree(h->d_conv_err);
    if (h->h_conv_err) cudaFreeHost(h->h_conv_err);
    if (h->d_jac_tmpl) cudaFree(h->d_jac_tmpl);
    if (h->d_jac_pick) cudaFree(h->d_jac_pick);
    if (h->d_tile_list) cudaFree(h->d_tile_list);
    if (h->d_group_list) cudaFree(h->d_group_list);
    if (h->mixed.mem) cudaFree(h->mixed.mem);
    if (h->adj_mem) cudaFree(h->adj_mem);
    delete h;
    return FEMB200_OK;
}

int femb200_set_stream(femb200_handle* h, void* stream) {
    if (!h) return FEMB200_EINVAL;
    h->stream = static_cast<cudaStream_t>(stream);
    return FEMB200_OK;
}

int femb200_set_ordered_scatter(femb200_handle* h, int32_t on) {
    if (!h) return FEMB200_EINVAL;
    h->ordered_scatter = on != 0;
    return FEMB200_OK;
}

const char* femb200_last_error(const femb200_handle* h) { return h ? h->err.c_str() : "null handle"; }

const char* femb200_version(void) { return "libfemtools_b200 0.1 (sm_100a)"; }

int femb200_pressure_residual(femb200_handle* h, const femb200_stokes_problem* p, double dt, int32_t finite_K) {
    RC(check_problem(h, p));
    RC(upload_material(h, p->mat, finite_K, dt));
    return dispatch<DoResidual>(p, h, p, dt, 0, 0, 1);
}

int femb200_momentum_residual(femb200_handle* h, const femb200_stokes_problem* p, double dt, int32_t with_pnum) {
    RC(check_problem(h, p));
    RC(upload_material(h, p->mat, 0, dt));
    if (with_pnum && !p->Pnum) { h->err = "Pnum is required"; return FEMB200_EINVAL; }
    return dispatch<DoMomentum>(p, h, p, dt, (int)with_pnum);
}

int femb200_stokes_residuals(femb200_handle* h, const femb200_stokes_problem* p, double dt, int32_t finite_K) {
    RC(check_problem(h, p));
    RC(upload_material(h, p->mat, finite_K, dt));
    return dispatch<DoResidual>(p, h, p, dt, 1, 1, 1);
}

int femb200_velocity_update(femb200_handle* h, const femb200_stokes_problem* p, const double* beta, const double* alpha) {
    RC(check_problem(h, p));
    if (!beta || !alpha) { h->err = "alpha and beta are required"; return FEMB200_EINVAL; }
    auto go = [&](auto tag) -> int {
        using T = decltype(tag);
        NodeArgs<T> na;
        std::memset(&na, 0, sizeof(na));
        for (int k = 0; k < 3; ++k) {
            na.v[k] = static_cast<T*>(p->v[k]); na.rate[k] = static_cast<T*>(p->rate[k]);
            na.Rv[k] = static_cast<T*>(p->Rv[k]); na.PC[k] = static_cast<const T*>(p->PC[k]);
            na.alpha[k] = k < p->dim ? alpha[k] : 0; na.beta[k] = k < p->dim ? beta[k] : 0;
        }
        na.mask = nullptr; na.n = p->nnodes; na.dim = p->dim; na.reduce = 0;
        CK(launch_node_update<T>(na, red_blocks(h, p->nnodes), h->stream));
        return FEMB200_OK;
    };
    return p->dtype == FEMB200_F64 ? go(double()) : go(float());
}

int femb200_apply_dirichlet(femb200_handle* h, void* x, const int32_t* dofs, const void* vals, int64_t n, int32_t dtype) {
    if (!h) return FEMB200_EINVAL;
    if (n == 0) return FEMB200_OK;
    if (!x || !dofs) { h->err = "x and dofs are required"; return FEMB200_EINVAL; }
    if (dtype == FEMB200_F64) CK(launch_dirichlet<double>(static_cast<double*>(x), dofs, static_cast<const double*>(vals), n, h->stream));
    else CK(launch_dirichlet<float>(static_cast<float*>(x), dofs, static_cast<const float*>(vals), n, h->stream));
    return FEMB200_OK;
}

int femb200_jacobian_diagnostics(femb200_handle* h, const femb200_stokes_problem* p, double dt, int32_t finite_K) {
    RC(check_problem(h, p));
    ++h->call_serial;
    RC(upload_material(h, p->mat, finite_K, dt));
    return dispatch<DoJacobian>(p, h, p, dt);
}

int femb200_pressure_scaling(femb200_handle* h, const femb200_stokes_problem* p, double gamma_fact, double dt, int32_t finite_K) {
    RC(check_problem(h, p));
    RC(upload_material(h, p->mat, finite_K, dt));
    return dispatch<DoScaling>(p, h, p, gamma_fact, dt);
}

int femb200_store_stress(femb200_handle* h, const femb200_stokes_problem* p, double dt) {
    RC(check_problem(h, p));
    RC(upload_material(h, p->mat, 0, dt));
    return dispatch<DoStore>(p, h, p, dt);
}

int femb200_shear_heating(femb200_handle* h, const femb200_stokes_problem* p, double dt, void* phi) {
    RC(check_problem(h, p));
    if (!phi) { h->err = "phi is required"; return FEMB200_EINVAL; }
    RC(upload_material(h, p->mat, 0, dt));
    return dispatch<DoShear>(p, h, p, dt, phi);
}

int femb200_solve_stokes(femb200_handle* h, const femb200_stokes_problem* p, const femb200_stokes_controls* c,
                         femb200_stokes_stats* st) {
    RC(check_problem(h, p));
    RC(check_controls(h, c));
    if (!st) { h->err = "null stats"; return FEMB200_EINVAL; }
    ++h->call_serial;
    RC(dispatch<DoSolve>(p, h, p, c, st, (Coupled*)nullptr));
    return finish_solve(h, c, st);
}

// The convolutions' error word: allocated and cleared on first use; a failure recorded by
// an earlier launch is reported once its mirror has reached the host (at the latest at the
// loss read-back, which synchronises the stream).
static int conv_err_word(femb200_handle* h, int** dev) {
    if (!h->d_conv_err) {
        CK(cudaMalloc(&h->d_conv_err, sizeof(int)));
        CK(cudaMallocHost(&h->h_conv_err, sizeof(int)));
        *h->h_conv_err = 0;
        CK(cudaMemsetAsync(h->d_conv_err, 0, sizeof(int), h->stream));
    }
    if (*h->h_conv_err != 0) {
        h->err = "tensor-core convolution: a wait on the MMA completion gave up";
        return FEMB200_ECUDA;
    }
    *dev = h->d_conv_err;
    return FEMB200_OK;
}

static int conv_err_mirror(femb200_handle* h) {
    CK(cudaMemcpyAsync(h->h_conv_err, h->d_conv_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    return FEMB200_OK;
}

int femb200_conv3x3_forward(femb200_handle* h, const void* in, const void* wt, const float* bias, const void* mask,
                            void* out, int32_t batch, int32_t height, int32_t width, int32_t ci, int32_t co,
                            int32_t mode) {
    if (!h) return FEMB200_EINVAL;
    if ((ci != 16 && ci != 32) || (co != 16 && co != 32) || mode < 0 || mode > 2) {
        h->err = "conv3x3: ci and co must be 16 or 32, mode 0, 1 or 2"; return FEMB200_EUNSUPPORTED;
    }
    if (!in || !wt || !out || (mode != 2 && !bias) || (mode == 2 && !mask) || batch < 1 || height < 1 || width < 1) {
        h->err = "conv3x3: missing array or empty grid"; return FEMB200_EINVAL;
    }
    if (height > 65535) { h->err = "conv3x3: height above 65535"; return FEMB200_EINVAL; }
    if (((uintptr_t)in | (uintptr_t)wt | (uintptr_t)mask | (uintptr_t)out) & 15u) {
        h->err = "conv3x3: in, wt, mask and out must be 16-byte aligned"; return FEMB200_EINVAL;
    }
    int* err = nullptr;
    RC(conv_err_word(h, &err));
    CK(launch_conv3x3(ci, co, mode, in, wt, bias, mask, out, batch, height, width, h->num_sms, err, h->stream));
    return conv_err_mirror(h);
}

int femb200_conv3x3_weight_grad(femb200_handle* h, const void* in, const void* dy, float* dw, float* db, int32_t batch,
                                int32_t height, int32_t width, int32_t ci, int32_t co) {
    if (!h) return FEMB200_EINVAL;
    if ((ci != 16 && ci != 32) || (co != 16 && co != 32)) { h->err = "conv3x3: ci and co must be 16 or 32"; return FEMB200_EUNSUPPORTED; }
    if (!in || !dy || !dw || batch < 1 || height < 1 || width < 1) { h->err = "conv3x3: missing array or empty grid"; return FEMB200_EINVAL; }
    if (((uintptr_t)in | (uintptr_t)dy) & 15u) { h->err = "conv3x3: in and dy must be 16-byte aligned"; return FEMB200_EINVAL; }
    int* err = nullptr;
    RC(conv_err_word(h, &err));
    CK(launch_conv3x3_wgrad(ci, co, in, dy, dw, db, batch, height, width, h->num_sms, err, h->stream));
    return conv_err_mirror(h);
}

int femb200_conv3x3_flip_weights(femb200_handle* h, const void* w, void* wT, int32_t ci, int32_t co) {
    if (!h) return FEMB200_EINVAL;
    if ((ci != 16 && ci != 32) || (co != 16 && co != 32) || !w || !wT) { h->err = "conv3x3: bad flip arguments"; return FEMB200_EINVAL; }
    CK(launch_flip_weights(w, wT, ci, co, h->stream));
    return FEMB200_OK;
}

int femb200_mse_loss_grad(femb200_handle* h, const float* out, const float* target, int32_t nt, int32_t co, double scale,
                          void* dy, int64_t npix, double* loss) {
    if (!h) return FEMB200_EINVAL;
    if (!out || !target || !dy || nt < 1 || nt > co || npix < 1) { h->err = "mse: bad arguments"; return FEMB200_EINVAL; }
    const int blocks = red_blocks(h, npix * co);
    RC(ensure_partials(h, blocks));
    CK(launch_mse(out, target, nt, co, (float)scale, dy, npix, h->d_partials, blocks, h->stream));
    if (loss) {
        double s;
        RC(fetch_sums(h, blocks, 1, &s));
        *loss = scale * s;
        if (h->h_conv_err && *h->h_conv_err != 0) {
            h->err = "tensor-core convolution: a wait on the MMA completion gave up";
            return FEMB200_ECUDA;
        }
    }
    return FEMB200_OK;
}

int femb200_adam_step(femb200_handle* h, float* w, float* m, float* v, const float* g, void* w_bf16, int64_t n, double lr,
                      double beta1, double beta2, double eps, int64_t step) {
    if (!h) return FEMB200_EINVAL;
    if (!w || !m || !v || !g || n < 1 || step < 1) { h->err = "adam: bad arguments"; return FEMB200_EINVAL; }
    CK(launch_adam(w, m, v, g, w_bf16, n, (float)lr, (float)beta1, (float)beta2, (float)eps, step, h->stream));
    return FEMB200_OK;
}

int femb200_f32_to_bf16(femb200_handle* h, const float* x, void* y, int64_t n) {
    if (!h) return FEMB200_EINVAL;
    if (!x || !y || n < 0) { h->err = "f32_to_bf16: bad arguments"; return FEMB200_EINVAL; }
    if (n) CK(launch_f32_to_bf16(x, y, n, h->stream));
    return FEMB200_OK;
}

int femb200_q9_grid_fields(femb200_handle* h, const femb200_stokes_problem* p, const int32_t* node_elem,
                           const int8_t* node_xi, const int8_t* node_eta, int32_t nx, int32_t ny, double dx, double dy,
                           float* out) {
    RC(check_problem(h, p));
    if (p->dim != 2 || p->dtype != FEMB200_F64) { h->err = "grid fields: 2-D Q9 FP64 states only"; return FEMB200_EUNSUPPORTED; }
    if ((int64_t)nx * ny != p->nnodes || !node_elem || !node_xi || !node_eta || !out) { h->err = "grid fields: the grid must cover the nodes"; return FEMB200_EINVAL; }
    CK(launch_grid_fields<double>(static_cast<const double*>(p->v[0]), static_cast<const double*>(p->v[1]),
                                  static_cast<const double*>(p->P), p->dofsP, node_elem, node_xi, node_eta, nx, ny,
                                  (float)dx, (float)dy, out, h->stream));
    return FEMB200_OK;
}

int femb200_net_input(femb200_handle* h, const float* Fprev, const float* Fcur, const float* scale, void* X, int64_t npix) {
    if (!h) return FEMB200_EINVAL;
    if (!Fprev || !Fcur || !scale || !X || npix < 1) { h->err = "net input: bad arguments"; return FEMB200_EINVAL; }
    CK(launch_net_input(Fprev, Fcur, scale, X, npix, h->stream));
    return FEMB200_OK;
}

int femb200_net_target(femb200_handle* h, const float* Fprev, const float* Fcur, const float* Fnext, const float* scale,
                       float* target, int64_t npix) {
    if (!h) return FEMB200_EINVAL;
    if (!Fprev || !Fcur || !Fnext || !scale || !target || npix < 1) { h->err = "net target: bad arguments"; return FEMB200_EINVAL; }
    CK(launch_net_target(Fprev, Fcur, Fnext, scale, target, npix, h->stream));
    return FEMB200_OK;
}

int femb200_precompute_geometry(femb200_handle* h, int32_t dim, int64_t nels, int64_t nnodes, const double* coords,
                                const int32_t* el2n, void* geo_v, void* geo_P, int32_t geo_dtype) {
    if (!h) return FEMB200_EINVAL;
    if ((dim != 2 && dim != 3) || nels < 0 || (geo_dtype != FEMB200_F64 && geo_dtype != FEMB200_F32)) {
        h->err = "precompute_geometry: bad arguments";
        return FEMB200_EINVAL;
    }
    if (nels == 0) return FEMB200_OK;
    if (nnodes < 1 || !coords || !el2n || !geo_v) { h->err = "precompute_geometry: bad arguments"; return FEMB200_EINVAL; }
    RC(ensure_tables(h));
    if (!h->d_flag) {
        CK(cudaMalloc(&h->d_flag, sizeof(int)));
        CK(cudaMallocHost(&h->h_flag, sizeof(int)));
    }
    CK(cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
    if (geo_dtype == FEMB200_F64)
        CK(launch_geometry<double>(dim, coords, el2n, nels, nnodes, static_cast<double*>(geo_v), static_cast<double*>(geo_P),
                                   h->d_flag, h->stream));
    else
        CK(launch_geometry<float>(dim, coords, el2n, nels, nnodes, static_cast<float*>(geo_v), static_cast<float*>(geo_P),
                                  h->d_flag, h->stream));
    CK(cudaMemcpyAsync(h->h_flag, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (*h->h_flag) { h->err = "precompute_geometry: a connectivity entry lies outside 1:nnodes"; return FEMB200_EINVAL; }
    return FEMB200_OK;
}


int femb200_cell_pressure_preconditioner(femb200_handle* h, const femb200_cell_pressure_problem* p) {
    RC(check_cp_problem(h, p));
    RC(ensure_tables(h));
    RC(cp_validate(h, p));
    return cp_preconditioner(h, p);
}

int femb200_cell_pressure_residuals(femb200_handle* h, const femb200_cell_pressure_problem* p, int32_t which) {
    RC(check_cp_problem(h, p));
    if (which < 1 || which > 3) { h->err = "which: bit 0 pressure residual, bit 1 momentum residual"; return FEMB200_EINVAL; }
    RC(ensure_tables(h));
    RC(cp_validate(h, p));
    return cp_residuals(h, p, which);
}

int femb200_solve_cell_pressure(femb200_handle* h, const femb200_cell_pressure_problem* p,
                                const femb200_cell_pressure_controls* c, femb200_cell_pressure_stats* st) {
    RC(check_cp_problem(h, p));
    if (!c || !st) { h->err = "controls and stats are required"; return FEMB200_EINVAL; }
    if (!(c->tolerance > 0) || c->max_iterations < 1 || c->check_interval < 1 || !std::isfinite(c->velocity_step) ||
        !std::isfinite(c->pressure_step)) {
        h->err = "tolerance, max_iterations, check_interval and the step sizes must be positive and finite";
        return FEMB200_EINVAL;
    }
    RC(ensure_tables(h));
    RC(cp_validate(h, p));
    std::memset(st, 0, sizeof(*st));
    const int64_t nn = p->nnodes, nels = p->nels;
    const cudaStream_t s = h->stream;
    RC(cp_preconditioner(h, p));
    // affine cells (a box or sheared mesh): the residuals read one J⁻¹ and |det J| per
    // cell, built here once per solve in the handle's geometry scratch
    const double* geo_c = nullptr;
    {
        const size_t need = (size_t)nels * 10 * sizeof(double);
        if (need > h->geo_c_cap) {
            if (h->d_geo_c) cudaFree(h->d_geo_c);
            h->d_geo_c = nullptr;
            CK(cudaMalloc(&h->d_geo_c, need));
            h->geo_c_cap = need;
        }
        h->geo_c_valid = false;   // the StokesDR sweeps rebuild theirs at their next solve
        CK(cudaMemsetAsync(h->d_flag, 0, sizeof(int), s));
        CK(launch_cp_compress_geometry(p->geo_v, nels, static_cast<double*>(h->d_geo_c), h->d_flag, s));
        CK(cudaMemcpyAsync(h->h_flag, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (*h->h_flag == 0) geo_c = static_cast<const double*>(h->d_geo_c);
    }
    // the first residual sees the prescribed boundary velocities too; the velocity step
    // leaves the constrained entries (bit k of the mask) at these values
    for (int k = 0; k < 3; ++k) CK(launch_dirichlet<double>(p->v[k], p->bc_dofs[k], p->bc_vals[k], p->bc_n[k], s));
    if ((size_t)nn > h->cpmask_cap) {
        if (h->d_cpmask) cudaFree(h->d_cpmask);
        h->d_cpmask = nullptr;
        CK(cudaMalloc(&h->d_cpmask, (size_t)nn));
        h->cpmask_cap = (size_t)nn;
    }
    CK(cudaMemsetAsync(h->d_cpmask, 0, (size_t)nn, s));
    for (int k = 0; k < 3; ++k)
        if (p->bc_n[k] > 0) CK(launch_build_mask(h->d_cpmask, p->bc_dofs[k], p->bc_n[k], k, s));
    CpVelArgs va;
    for (int k = 0; k < 3; ++k) {
        va.v[k] = p->v[k];
        va.Rv[k] = p->Rv[k];
        va.diag[k] = p->diagonal[k];
        va.load[k] = p->load[k];
    }
    va.mask = h->d_cpmask;
    va.n = nn;
    va.step = c->velocity_step;
    bool rv_zeroed = false;   // the previous velocity step left Rv zeroed
    const int nb = cp_mean_blocks(h->num_sms);
    RC(ensure_partials(h, nb));
    double err_v = INFINITY, err_P = INFINITY, err = INFINITY;
    int64_t iter = 0, hist = 0;
    for (int64_t it = 1; it <= c->max_iterations; ++it) {
        iter = it;
        const bool check = it % c->check_interval == 0 || it == c->max_iterations;
        RC(cp_residuals(h, p, 1, geo_c));
        CK(launch_cp_pressure_update(p->P, p->RP, p->pressure_mass, nels, c->pressure_step, h->d_partials, nb, s));
        RC(cp_residuals(h, p, 2, geo_c, rv_zeroed));
        // between checks nothing reads Rv after the step: it is zeroed there for the next
        // momentum residual; a check iteration keeps it for the norms (and the caller)
        va.zero = check ? 0 : 1;
        CK(launch_cp_velocity_step(va, s));
        rv_zeroed = !check;
        if (!check) continue;
        err_v = 0;
        for (int k = 0; k < 3; ++k) {
            double ss = 0;
            RC(sumsq<double>(h, p->Rv[k], nullptr, nn, ss));
            err_v = jl_max(err_v, std::sqrt(ss));
        }
        double sp = 0;
        RC(sumsq<double>(h, p->RP, nullptr, 4 * nels, sp));
        err_P = std::sqrt(sp);
        err = jl_max(err_v, err_P);
        if (!std::isfinite(err)) { h->err = "non-finite residual in 3-D Stokes solve"; return FEMB200_ENONFINITE; }
        if (c->history && hist < c->history_capacity) {
            c->history[3 * hist] = (double)it;
            c->history[3 * hist + 1] = err_v;
            c->history[3 * hist + 2] = err_P;
            ++hist;
        }
        if (err < c->tolerance) break;
    }
    st->converged = err < c->tolerance;
    st->iterations = iter;
    st->residual = err;
    st->err_v = err_v;
    st->err_P = err_P;
    st->reached_total_iter = iter >= c->max_iterations && !st->converged;
    st->history_len = hist;
    if (!st->converged && c->throw_on_failure) {
        char b[160];
        std::snprintf(b, sizeof b, "3-D Stokes solve did not converge after %lld iterations (residual = %g, tolerance = %g)",
                      (long long)iter, err, c->tolerance);
        h->err = b;
        return FEMB200_ENOTCONV;
    }
    return FEMB200_OK;
}

int femb200_strain_rate_stress(femb200_handle* h, const femb200_stokes_problem* p, const void* const tau_ip[6],
                               void* const out[14]) {
    RC(check_problem(h, p));
    const int nt = p->dim == 3 ? 6 : 3, nf = p->dim == 3 ? 14 : 10;
    if (!tau_ip || !out) { h->err = "strain_rate_stress: stresses and outputs are required"; return FEMB200_EINVAL; }
    for (int c = 0; c < nt; ++c)
        if (!tau_ip[c]) { h->err = "strain_rate_stress: stresses and outputs are required"; return FEMB200_EINVAL; }
    for (int k = 0; k < nf; ++k)
        if (!out[k]) { h->err = "strain_rate_stress: stresses and outputs are required"; return FEMB200_EINVAL; }
    RC(ensure_tables(h));
    const bool d = p->dtype == FEMB200_F64, gd = p->geo_dtype == FEMB200_F64;
    if (d && gd) return strain_rate_stress_impl<double, double>(h, p, tau_ip, out);
    if (d) return strain_rate_stress_impl<double, float>(h, p, tau_ip, out);
    if (gd) return strain_rate_stress_impl<float, double>(h, p, tau_ip, out);
    return strain_rate_stress_impl<float, float>(h, p, tau_ip, out);
}

int femb200_cap_update(femb200_handle* h, const femb200_cap_problem* p) {
    if (!h) return FEMB200_EINVAL;
    if (!p) { h->err = "cap_update: problem is required"; return FEMB200_EINVAL; }
    if (p->n < 0) { h->err = "cap_update: negative point count"; return FEMB200_EINVAL; }
    if (p->ncomp != 0 && p->ncomp != 3 && p->ncomp != 6) {
        h->err = "cap_update: ncomp must be 0 (scalar return map), 3 (plane strain) or 6 (3-D)";
        return FEMB200_EINVAL;
    }
    if (p->maxiter < 0) { h->err = "cap_update: maxiter must be >= 0"; return FEMB200_EINVAL; }
    if (p->n == 0) return FEMB200_OK;
    const bool trial = p->ncomp > 0 ? p->tau_trial != nullptr : p->s_trial != nullptr;
    if (!trial || !p->P_trial || !p->eta_ve || !p->K_dt || !p->k || !p->kq || !p->c || !p->pT || !p->eta_reg) {
        h->err = "cap_update: the trial state and every material array are required";
        return FEMB200_EINVAL;
    }
    CK(launch_cap_update(*p, h->num_sms, h->stream));
    return FEMB200_OK;
}

int femb200_extrapolate_state(femb200_handle* h, const femb200_stokes_problem* p, const void* const vprev[3],
                              const void* const vcur[3], const void* Pprev, const void* Pcur) {
    RC(check_problem(h, p));
    if (p->dtype != FEMB200_F64) { h->err = "extrapolation: FP64 states only"; return FEMB200_EUNSUPPORTED; }
    if (!vprev || !vcur || !Pprev || !Pcur) { h->err = "extrapolation: bad arguments"; return FEMB200_EINVAL; }
    RC(build_mask(h, p));
    const double* vp[3];
    const double* vc[3];
    double* v[3];
    for (int k = 0; k < p->dim; ++k) {
        vp[k] = static_cast<const double*>(vprev[k]); vc[k] = static_cast<const double*>(vcur[k]);
        v[k] = static_cast<double*>(p->v[k]);
    }
    CK(launch_extrapolate_guess<double>(p->dim, vp, vc, static_cast<const double*>(Pprev), static_cast<const double*>(Pcur),
                                        h->d_mask, v, static_cast<double*>(p->P), p->nnodes, p->nnodesP, h->stream));
    return FEMB200_OK;
}

int femb200_apply_warm_start(femb200_handle* h, const femb200_stokes_problem* p, const void* const vprev[2],
                             const void* const vcur[2], const void* Pprev, const void* Pcur, const float* out,
                             int32_t co, const float scale[3]) {
    RC(check_problem(h, p));
    if (p->dim != 2 || p->dtype != FEMB200_F64 || p->np != 3) { h->err = "warm start: 2-D Q9/P1-disc FP64 states only"; return FEMB200_EUNSUPPORTED; }
    if (!vprev || !vcur || !Pprev || !Pcur || (out && (!scale || co < 3))) { h->err = "warm start: bad arguments"; return FEMB200_EINVAL; }
    RC(build_mask(h, p));
    const double* vp[2] = {static_cast<const double*>(vprev[0]), static_cast<const double*>(vprev[1])};
    const double* vc[2] = {static_cast<const double*>(vcur[0]), static_cast<const double*>(vcur[1])};
    double* v[2] = {static_cast<double*>(p->v[0]), static_cast<double*>(p->v[1])};
    CK(launch_apply_guess<double>(vp, vc, static_cast<const double*>(Pprev), static_cast<const double*>(Pcur), out, co,
                                  scale, h->d_mask, v, static_cast<double*>(p->P), p->dofsP, p->el2n, p->nnodes, p->nels,
                                  h->stream));
    return FEMB200_OK;
}

int femb200_stokes_adjoint_residual(femb200_handle* h, const femb200_stokes_problem* p, double dt, int32_t finite_K,
                                    int32_t with_pnum, const void* const lam_v[3], const void* lam_P,
                                    void* const out_dv[3], void* out_dP) {
    RC(check_adjoint_problem(h, p));
    if (!lam_v || !lam_P || !out_dv || !out_dP) { h->err = "λ and the outputs are required"; return FEMB200_EINVAL; }
    RC(upload_material(h, p->mat, finite_K, dt));
    AdjArgs<double> a = adjoint_args(p, dt, with_pnum, lam_v, lam_P);
    for (int k = 0; k < 3; ++k) {
        a.out_dv[k] = static_cast<double*>(out_dv[k]);
        CK(cudaMemsetAsync(out_dv[k], 0, sizeof(double) * p->nnodes, h->stream));
    }
    a.out_dP = static_cast<double*>(out_dP);
    CK(launch_hex27_adjoint<double>(a, h->num_sms, h->stream));
    return FEMB200_OK;
}

int femb200_stokes_viscosity_sensitivity(femb200_handle* h, const femb200_stokes_problem* p, double dt,
                                         int32_t finite_K, int32_t with_pnum, const void* const lam_v[3],
                                         const void* lam_P, void* out_eta_ip) {
    RC(check_adjoint_problem(h, p));
    if (!lam_v || !lam_P || !out_eta_ip) { h->err = "λ and the output are required"; return FEMB200_EINVAL; }
    RC(upload_material(h, p->mat, finite_K, dt));
    AdjArgs<double> a = adjoint_args(p, dt, with_pnum, lam_v, lam_P);
    a.out_eta = static_cast<double*>(out_eta_ip);
    CK(launch_hex27_adjoint<double>(a, h->num_sms, h->stream));
    return FEMB200_OK;
}

int femb200_solve_stokes_adjoint(femb200_handle* h, const femb200_stokes_problem* p, const femb200_stokes_controls* c,
                                 const void* const objective_v[3], void* const lam_v[3], void* lam_P,
                                 femb200_stokes_stats* st) {
    RC(check_adjoint_problem(h, p));
    RC(check_controls(h, c));
    if (!st || !objective_v || !lam_v || !lam_P) { h->err = "objective, λ and stats are required"; return FEMB200_EINVAL; }
    ++h->call_serial;
    RC(solve_adjoint_impl(h, p, c, objective_v, lam_v, lam_P, st));
    if (c->throw_on_failure && !st->converged) {
        char b[160];
        std::snprintf(b, sizeof b, "Adjoint solve did not converge: err=%.3e after %lld iterations", st->err, (long long)st->iter);
        h->err = b;
        return FEMB200_ENOTCONV;
    }
    return FEMB200_OK;
}

int femb200_transfer_temperature(femb200_handle* h, void* TP, const void* Tn, const int32_t* dofsP, const int32_t* el2nP,
                                 int64_t n, int32_t dtype) {
    if (!h) return FEMB200_EINVAL;
    if (dtype == FEMB200_F64) CK(launch_transfer_temperature<double>(static_cast<double*>(TP), static_cast<const double*>(Tn), dofsP, el2nP, n, h->stream));
    else CK(launch_transfer_temperature<float>(static_cast<float*>(TP), static_cast<const float*>(Tn), dofsP, el2nP, n, h->stream));
    return FEMB200_OK;
}

int femb200_thermal_residual(femb200_handle* h, const femb200_thermal_problem* t, double dt, double Tref, int32_t jac) {
    if (!h || !t) return FEMB200_EINVAL;
    RC(ensure_tables(h));
    RC(upload_thermal_material(h, t));
    if (t->dtype == FEMB200_F64) return thermal_assemble<double, double>(h, t, dt, Tref, jac != 0, t->source_ip);
    return thermal_assemble<float, float>(h, t, dt, Tref, jac != 0, t->source_ip);
}

int femb200_thermal_residual_colored(femb200_handle* h, const femb200_thermal_problem* t, double dt, double Tref,
                                     int32_t jac, const int32_t* groups, const int64_t* offsets, int32_t ngroups) {
    if (!h || !t) return FEMB200_EINVAL;
    if (!groups || !offsets || ngroups < 1) { h->err = "colour groups are required"; return FEMB200_EINVAL; }
    if (offsets[0] != 0 || offsets[ngroups] != t->nels) { h->err = "colour groups must cover every element once"; return FEMB200_EINVAL; }
    for (int32_t g = 0; g < ngroups; ++g)
        if (offsets[g + 1] < offsets[g]) { h->err = "colour group offsets must not decrease"; return FEMB200_EINVAL; }
    RC(ensure_tables(h));
    RC(upload_thermal_material(h, t));
    if (t->dtype == FEMB200_F64) return thermal_assemble_colored<double, double>(h, t, dt, Tref, jac != 0, groups, offsets, ngroups);
    return thermal_assemble_colored<float, float>(h, t, dt, Tref, jac != 0, groups, offsets, ngroups);
}

int femb200_solve_thermal(femb200_handle* h, const femb200_thermal_problem* t, const femb200_thermal_controls* c,
                          femb200_thermal_stats* st) {
    if (!h || !t || !c || !st) return FEMB200_EINVAL;
    if (t->dtype != FEMB200_F64 || t->geo_dtype != FEMB200_F64) { h->err = "the thermal solver runs in FP64"; return FEMB200_EUNSUPPORTED; }
    using T = double;
    RC(upload_thermal_material(h, t));
    RC(build_tmask(h, t));
    DrNodal f{static_cast<T*>(t->T), static_cast<T*>(t->rate), static_cast<T*>(t->R), static_cast<T*>(t->R0),
              static_cast<const T*>(t->dRdT), static_cast<const T*>(t->PC), t->nnodes, t->bc_dofs,
              static_cast<const T*>(t->bc_vals), t->bc_n, t->cfl, t->c_fact};
    auto assemble = [&](bool dj) { return thermal_assemble<T, T>(h, t, c->dt, c->Tref, dj, t->source_ip); };
    return dr_nodal_solve(h, f, h->d_tmask, c->tolerance, c->max_iterations, c->check_interval, c->throw_on_failure,
                          "thermal diffusion", "Thermal diffusion", assemble, st);
}

int femb200_lithostatic_residual(femb200_handle* h, const femb200_lithostatic_problem* p, double Tref,
                                 const double g[3], int32_t jac) {
    RC(check_litho_problem(h, p));
    if (!g) { h->err = "lithostatic pressure: g is required"; return FEMB200_EINVAL; }
    RC(ensure_tables(h));
    return litho_assemble(h, p, Tref, g, jac != 0);
}

int femb200_solve_lithostatic(femb200_handle* h, const femb200_lithostatic_problem* p,
                              const femb200_lithostatic_controls* c, femb200_thermal_stats* st) {
    RC(check_litho_problem(h, p));
    if (!c || !st) { h->err = "controls and stats are required"; return FEMB200_EINVAL; }
    if (c->max_iterations < 1 || c->check_interval < 1) { h->err = "max_iterations and check_interval must be positive"; return FEMB200_EINVAL; }
    RC(ensure_tables(h));
    RC(build_node_mask(h, p->bc_dofs, p->bc_n, p->nnodes));
    std::memset(st, 0, sizeof(*st));
    DrNodal f{p->P, p->rate, p->R, p->R0, p->dRdP, p->PC, p->nnodes, p->bc_dofs, p->bc_vals, p->bc_n, p->cfl, p->c_fact};
    auto assemble = [&](bool dj) { return litho_assemble(h, p, c->Tref, c->g, dj); };
    return dr_nodal_solve(h, f, h->d_tmask, c->tolerance, c->max_iterations, c->check_interval, c->throw_on_failure,
                          "lithostatic pressure", "Lithostatic pressure", assemble, st);
}

int femb200_solve_coupled(femb200_handle* h, femb200_thermal_problem* t, const femb200_stokes_problem* p,
                          const femb200_stokes_controls* c, double Tref, int32_t shear_heating, void* phi_scratch,
                          femb200_stokes_stats* st) {
    RC(check_problem(h, p));
    RC(check_controls(h, c));
    if (!t || !st) { h->err = "thermal problem and stats are required"; return FEMB200_EINVAL; }
    if (t->nnodes != p->nnodes) { h->err = "thermal mesh nodes must match the Stokes velocity-node layout"; return FEMB200_EINVAL; }
    ++h->call_serial;
    if (t->dtype != p->dtype) { h->err = "thermal and Stokes states must share a precision"; return FEMB200_EINVAL; }
    if (shear_heating && !phi_scratch) { h->err = "shear heating needs an nq × nels scratch array"; return FEMB200_EINVAL; }
    const int64_t ntr = (int64_t)p->np * p->nels;
    if (p->dtype == FEMB200_F64) {
        CK(launch_transfer_temperature<double>(static_cast<double*>(p->T), static_cast<const double*>(t->T), p->dofsP, p->el2nP, ntr, h->stream));
        CK(launch_transfer_temperature<double>(static_cast<double*>(p->T0), static_cast<const double*>(t->T0), p->dofsP, p->el2nP, ntr, h->stream));
        if (shear_heating) CK(cudaMemsetAsync(phi_scratch, 0, sizeof(double) * p->nq * p->nels, h->stream));
    } else {
        CK(launch_transfer_temperature<float>(static_cast<float*>(p->T), static_cast<const float*>(t->T), p->dofsP, p->el2nP, ntr, h->stream));
        CK(launch_transfer_temperature<float>(static_cast<float*>(p->T0), static_cast<const float*>(t->T0), p->dofsP, p->el2nP, ntr, h->stream));
        if (shear_heating) CK(cudaMemsetAsync(phi_scratch, 0, sizeof(float) * p->nq * p->nels, h->stream));
    }
    Coupled cp{t, Tref, shear_heating ? phi_scratch : nullptr};
    RC(dispatch<DoSolve>(p, h, p, c, st, &cp));
    return finish_solve(h, c, st);
}

}  // extern "C"

// ---- allocation-free thermal solve (femb200_solve_thermal_noalloc) ----------
//
// For hosts that own all device memory through their own pool, or that cannot
// take the device-wide synchronisation of cudaFree / cudaMallocHost, this solve
// keeps its Dirichlet mask and reduction partials in one fixed array of the
// library's device image instead of handle buffers grown with cudaMalloc. The
// final reduction over blocks runs on the device (one thread per slot, blocks in
// order, the same summation order as fetch_sums), so the host reads back a few
// doubles into a stack buffer and needs no pinned memory.
namespace {

constexpr int64_t NA_MAX_NODES = FEMB200_NOALLOC_MAX_NODES;
constexpr int NA_MAX_BLOCKS = 1024;
constexpr size_t NA_PARTIALS = (size_t)NA_MAX_BLOCKS * RED_SLOTS;   // doubles
constexpr size_t NA_RESULT = 16;                                     // doubles
constexpr size_t NA_BYTES = (NA_PARTIALS + NA_RESULT) * sizeof(double) + (size_t)NA_MAX_NODES;
}  // namespace

// Layout: [block partials | reduced slots | one mask byte per node]. In host code
// the name is only a handle for cudaGetSymbolAddress, never a device address.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

namespace {

struct NoallocScratch {
    double* partials;
    double* result;
    uint8_t* mask;
};

// Device address of the scratch array, looked up by the first call on a handle
// (with the handle's device current; it must not fall inside a capture) and kept
// in the handle. A handle made after cudaDeviceReset looks it up again, in the
// reloaded module.
int noalloc_scratch(femb200_handle* h, NoallocScratch& s) {
    int dev = -1;
    CK(cudaGetDevice(&dev));
    if (dev != h->device) {
        h->err = "femb200_solve_thermal_noalloc: the current device (" + std::to_string(dev) +
                 ") is not the handle's device (" + std::to_string(h->device) + ")";
        return FEMB200_EINVAL;
    }
    if (!h->noalloc_base) {
        void* p = nullptr;
        CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        h->noalloc_base = static_cast<unsigned char*>(p);
    }
    s.partials = reinterpret_cast<double*>(h->noalloc_base);
    s.result = s.partials + NA_PARTIALS;
    s.mask = reinterpret_cast<uint8_t*>(s.result + NA_RESULT);
    return FEMB200_OK;
}

// result[s] = Σ_b partials[b][s] (mode 0, s < nslots) or, for the λmax check
// (mode 1), result[0] = max_b partials[b][0] and result[1] = 1 if any block
// flagged a NaN. One thread per slot, blocks in ascending order.
__global__ void noalloc_finalize_kernel(const double* partials, int blocks, int nslots, int mode, double* result) {
    const int s = threadIdx.x;
    if (s >= nslots) return;
    if (mode == 0) {
        double t = 0;
        for (int b = 0; b < blocks; ++b) t += partials[(size_t)b * RED_SLOTS + s];
        result[s] = t;
    } else if (s == 0) {
        double m = -INFINITY, f = 0;
        for (int b = 0; b < blocks; ++b) {
            m = fmax(m, partials[(size_t)b * RED_SLOTS]);
            if (partials[(size_t)b * RED_SLOTS + 1] != 0) f = 1;
        }
        result[0] = m;
        result[1] = f;
    }
}

int noalloc_read(femb200_handle* h, const NoallocScratch& s, int blocks, int nslots, int mode, double* out) {
    count_launch();
    noalloc_finalize_kernel<<<1, 32, 0, h->stream>>>(s.partials, blocks, nslots, mode, s.result);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, s.result, sizeof(double) * nslots, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return FEMB200_OK;
}

// _checked_λmax (src/utils.jl:152-158) on the scratch partials.
int noalloc_lmax(femb200_handle* h, const NoallocScratch& s, const double* J, const double* PC, int64_t n, int blocks,
                 double& out) {
    CK(launch_ratio_max<double>(J, PC, n, s.partials, blocks, h->stream));
    double r[2];
    RC(noalloc_read(h, s, blocks, 2, 1, r));
    double m = r[1] != 0 ? NAN : r[0];
    if (!(std::isfinite(m) && m > 0)) {
        char buf[256];
        std::snprintf(buf, sizeof buf, "thermal diffusion preconditioner produced invalid λmax = %g; check for zero or non-finite preconditioner entries", m);
        h->err = buf;
        return FEMB200_ELAMBDA;
    }
    out = m;
    return FEMB200_OK;
}

}  // namespace

extern "C" {

// solve_dynamic_relaxation! for the thermal DR (src/dynamic_relaxation/solver.jl:61-122),
// step for step as femb200_solve_thermal, with all scratch in g_noalloc_scratch.
int femb200_solve_thermal_noalloc(femb200_handle* h, const femb200_thermal_problem* t, const femb200_thermal_controls* c,
                                  femb200_thermal_stats* st) {
    if (!h || !t || !c || !st) return FEMB200_EINVAL;
    if (t->dtype != FEMB200_F64 || t->geo_dtype != FEMB200_F64) { h->err = "the thermal solver runs in FP64"; return FEMB200_EUNSUPPORTED; }
    if (t->nnodes < 1 || t->nnodes > NA_MAX_NODES) {
        h->err = "femb200_solve_thermal_noalloc: nnodes = " + std::to_string((long long)t->nnodes) +
                 " is outside 1:" + std::to_string((long long)NA_MAX_NODES) +
                 " (the fixed scratch size; use femb200_solve_thermal for larger meshes)";
        return FEMB200_EINVAL;
    }
    if (c->check_interval < 1) { h->err = "check_interval must be positive"; return FEMB200_EINVAL; }
    using T = double;
    NoallocScratch s;
    RC(noalloc_scratch(h, s));
    RC(upload_thermal_material(h, t));
    const int64_t n = t->nnodes;
    // the mask region keeps the previous call's bits: clear it before setting this call's
    CK(cudaMemsetAsync(s.mask, 0, (size_t)n, h->stream));
    if (t->bc_n > 0) CK(launch_build_mask(s.mask, t->bc_dofs, t->bc_n, 0, h->stream));
    // the block split of femb200_solve_thermal (4 per SM) must fit the scratch
    // partials, or the sums would be ordered differently from that solve's
    const int nbk = red_blocks(h, n);
    if (nbk > NA_MAX_BLOCKS) {
        h->err = "femb200_solve_thermal_noalloc: " + std::to_string(nbk) + " reduction blocks (4 per SM) exceed the " +
                 std::to_string(NA_MAX_BLOCKS) + " the fixed scratch holds";
        return FEMB200_EUNSUPPORTED;
    }
    double a = 0, b = 0, nr0 = 0, last = NAN, lmax = 0;
    for (int64_t it = 1; it <= c->max_iterations; ++it) {
        const bool dj = (it % c->check_interval == 0) || it == 1;
        if (dj) CK(launch_copy<T>(static_cast<T*>(t->R0), static_cast<const T*>(t->R), n, h->stream));
        RC((thermal_assemble<T, T>(h, t, c->dt, c->Tref, dj, t->source_ip)));
        if (dj) RC(noalloc_lmax(h, s, static_cast<const T*>(t->dRdT), static_cast<const T*>(t->PC), n, nbk, lmax));
        CK(launch_thermal_update<T>(static_cast<T*>(t->T), static_cast<T*>(t->rate), static_cast<T*>(t->R),
                                    static_cast<const T*>(t->PC), s.mask, n, a, b, h->stream));
        if (t->bc_n > 0) CK(launch_dirichlet<T>(static_cast<T*>(t->T), t->bc_dofs, static_cast<const T*>(t->bc_vals), t->bc_n, h->stream));
        if (dj) {
            const double dtau = 2 / std::sqrt(lmax) * t->cfl;
            CK(launch_lmin_sums<T>(static_cast<const T*>(t->rate), static_cast<const T*>(t->R), static_cast<const T*>(t->R0),
                                   static_cast<const T*>(t->PC), n, dtau, s.partials, nbk, h->stream));
            double r[3];
            RC(noalloc_read(h, s, nbk, 3, 0, r));
            const double nr = std::sqrt(r[2]);
            if (it == 1) nr0 = std::max(nr, julia_eps(nr));
            if (std::isnan(nr / nr0)) { char bb[64]; std::snprintf(bb, sizeof bb, "NaNs at PT iter %lld", (long long)it); h->err = bb; return FEMB200_ENAN; }
            const double lmin = (it == 1 || r[0] == 0) ? 0.0 : std::fabs(r[1]) / r[0];
            cheb(dtau, lmin, t->c_fact, a, b);
            last = nr / nr0;
            if (last < c->tolerance) { st->converged = 1; st->iterations = it; st->residual = last; return FEMB200_OK; }
        }
    }
    st->converged = 0; st->iterations = c->max_iterations; st->residual = last;
    if (c->throw_on_failure) {
        char bb[256];
        std::snprintf(bb, sizeof bb, "Thermal diffusion DR solver did not converge after %lld pseudo-transient iterations (relative residual = %g)",
                      (long long)c->max_iterations, last);
        h->err = bb;
        return FEMB200_ENOTCONV;
    }
    return FEMB200_OK;
}

}  // extern "C"
