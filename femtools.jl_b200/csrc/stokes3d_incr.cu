// stokes3d_incr.cu — thread-per-element FP32 incremental sweep of the mixed-precision solve.
//
// The sweep computes, for every Hex27/P1-disc element, the increments of the
// pressure residual, of the element-local Pnum and of the visco-elasto-plastic
// momentum residual between the FP64 base state x_k and x_k + δ
// (pressure_residual.jl:132-158, momentum_residuals.jl:209-258, rheology.jl:413-472),
// with the base trial stress and yield value of every integration point read
// from the tiled FP32 base data written by the FP64 base sweep.
//
// Mapping: one thread owns one element. Its 81 velocity increments and its 81
// residual accumulators live in thread-private shared-memory slots (bank = lane,
// conflict-free); the quadrature runs plane by plane (ζ): per plane the thread
// contracts the ζ-direction into 2 × 27 more private slots (W0, W1), per row (η)
// into 27 registers, evaluates the 3 points of the row with fully unrolled 1-D
// contractions whose Gauss-rule coefficients are compile-time constants (zero
// coefficients of the middle point drop out), and accumulates the transposed
// contraction of the fluxes into 2 × 27 + 9 registers that are expanded into the
// residual slots once per plane.
// No shared-memory exchange between threads and no idle lanes: the per-element
// instruction count is about a third of the warp-cooperative sweep's.
//
// Pnum enters the momentum residual only through −Pnum·I in the stress, which is
// linear in the four element-local Pnum values, so its contribution is added in
// the scatter from the constant table K[p][d][a] = Σ_q w_q N^P_p(q) ∂_d N_a(q):
// the element's pressure residual (which Pnum needs) and its momentum residual
// come out of one pass over the quadrature points.
#include <algorithm>
#include <cmath>
#include <mutex>
#include "kernels.cuh"
#include "rheology.cuh"

namespace femb {
namespace {

constexpr int IN_THREADS = 128;     // 4 warps; two blocks per SM
constexpr int IN_WARPS = IN_THREADS / 32;
constexpr int IN_SLOTS = 216;       // thread-private shared words: δv (81), residual (81), plane (54)

// 1-D quadratic Lagrange basis on (−1, 0, 1) at the 3-point Gauss rule ±√(3/5), 0
// (Hex27: src/elements/shape_functions.jl:404-446, Gauss rule integration_points.jl:321).
constexpr float GA = 0.774596669241483377f;
FEMB_HD constexpr float gx(int q) { return q == 0 ? -GA : (q == 1 ? 0.0f : GA); }
FEMB_HD constexpr float gw(int q) { return q == 1 ? 8.0f / 9.0f : 5.0f / 9.0f; }
FEMB_HD constexpr float Lb(int q, int i) {
    return i == 0 ? gx(q) * (gx(q) - 1.0f) * 0.5f : (i == 1 ? 1.0f - gx(q) * gx(q) : gx(q) * (gx(q) + 1.0f) * 0.5f);
}
FEMB_HD constexpr float Ld(int q, int i) { return i == 0 ? gx(q) - 0.5f : (i == 1 ? -2.0f * gx(q) : gx(q) + 0.5f); }

// fma with a coefficient that is a compile-time constant after unrolling: zero
// coefficients (middle Gauss point) fold away
FEMB_D float cfma(float c, float x, float acc) { return c != 0.0f ? fmaf(c, x, acc) : acc; }

}  // namespace

// K[p][d][a] = Σ_q w_q N^P_p(q) ∂N_a/∂ξ_d(q), a in tensor order.
__constant__ float c_inc_K[4][3][27];

namespace {

void host_pnum_table(float K[4][3][27]) {
    const double ga = std::sqrt(3.0 / 5.0);
    const double x[3] = {-ga, 0.0, ga}, w[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
    auto l = [&](int q, int i) { return i == 0 ? x[q] * (x[q] - 1) * 0.5 : (i == 1 ? 1 - x[q] * x[q] : x[q] * (x[q] + 1) * 0.5); };
    auto dl = [&](int q, int i) { return i == 0 ? x[q] - 0.5 : (i == 1 ? -2 * x[q] : x[q] + 0.5); };
    for (int p = 0; p < 4; ++p)
        for (int d = 0; d < 3; ++d)
            for (int a = 0; a < 27; ++a) {
                const int ia[3] = {a % 3, (a / 3) % 3, a / 9};
                double s = 0;
                for (int q = 0; q < 27; ++q) {
                    const int iq[3] = {q % 3, (q / 3) % 3, q / 9};
                    const double np = p == 0 ? 1 - x[iq[0]] - x[iq[1]] - x[iq[2]] : x[iq[p - 1]];
                    double dn = 1;
                    for (int r = 0; r < 3; ++r) dn *= r == d ? dl(iq[r], ia[r]) : l(iq[r], ia[r]);
                    s += w[iq[0]] * w[iq[1]] * w[iq[2]] * np * dn;
                }
                K[p][d][a] = (float)s;
            }
}

// Phase of an element for the sweep: the common phase of its nodes (or DoFs) in
// any of the three layouts (src/utils.jl:70-74), 0-based; -1 when they differ.
__device__ int uniform_phase(const int32_t* ph, int layout, const int32_t* ids, int n, int64_t e) {
    if (!ph) return 0;
    if (layout == FEMB200_PHASE_CELL) return ph[e] - 1;
    int p0 = -2;
    for (int i = 0; i < n; ++i) {
        const int p = (layout == FEMB200_PHASE_ELEMENT_NODE ? ph[(int64_t)n * e + i] : ph[ids[(int64_t)n * e + i] - 1]) - 1;
        if (p0 == -2) p0 = p;
        else if (p != p0) return -1;
    }
    return p0;
}

__global__ void incr_tiles_kernel(const IncrTileSrc src, int64_t nels, int64_t nslots, IncrArgs dst, int* flags) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nslots) return;
    const int64_t tile = e >> 5;
    const int lane = (int)(e & 31);
    const bool act = e < nels;
    int32_t* el2n_t = const_cast<int32_t*>(dst.el2n_t);
    int32_t* dofs_t = const_cast<int32_t*>(dst.dofs_t);
    float* geo_t = const_cast<float*>(dst.geo_t);
    float* pscale_t = const_cast<float*>(dst.pscale_t);
    for (int t = 0; t < 27; ++t) el2n_t[(tile * 27 + t) * 32 + lane] = act ? src.el2n[27 * e + c_tab.tn3[t]] - 1 : 0;
    bool linear = true;
    for (int p = 0; p < 4; ++p) {
        const int32_t d = act ? src.dofsP[4 * e + p] - 1 : 0;
        linear = linear && (!act || d == 4 * e + p);
        dofs_t[(tile * 4 + p) * 32 + lane] = d;
        pscale_t[(tile * 4 + p) * 32 + lane] = act ? src.gP[d] / src.MP[d] : 0.0f;
    }
    if (!linear) atomicOr(flags, INCR_DOFS_GENERAL);
    bool offdiag = false;
    for (int r = 0; r < 10; ++r) {
        const float gv = act ? src.geo_c[10 * e + r] : 0.0f;
        offdiag = offdiag || (r < 9 && r % 4 != 0 && gv != 0.0f);
        geo_t[(tile * 10 + r) * 32 + lane] = gv;
    }
    if (offdiag) atomicOr(flags, INCR_GEOMETRY_FULL);
    if (src.eta) {
        float* eta_t = const_cast<float*>(dst.eta_t);
        for (int q = 0; q < 27; ++q) eta_t[(tile * 27 + q) * 32 + lane] = act ? src.eta[27 * e + q] : 1.0f;
    }
    int pv = 0, pp = 0;
    if (act) {
        pv = uniform_phase(src.phv, src.phv_layout, src.el2n, 27, e);
        pp = uniform_phase(src.php, src.php_layout, src.dofsP, 4, e);
        if (pv < 0 || pp < 0 || pv >= src.nphases || pp >= src.nphases) {
            atomicOr(flags, INCR_MIXED_PHASES);
            pv = pp = 0;
        }
    }
    int32_t* phase_t = const_cast<int32_t*>(dst.phase_t);
    phase_t[e] = pv;
    phase_t[nslots + e] = pp;
}

FEMB_D void cp_async4(float* dst, const float* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
FEMB_D void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
FEMB_D void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Bulk copies (sm_90+ cp.async.bulk, one thread issues, completion counted in bytes on an
// mbarrier) of the contiguous per-tile blocks: this GPU's global memory to the CTA's own
// shared memory, no multicast.
FEMB_D uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
FEMB_D void mbar_init(uint32_t m) { asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(m) : "memory"); }
// orders this thread's earlier shared-memory accesses before later bulk-copy writes
FEMB_D void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
FEMB_D void mbar_expect(uint32_t m, unsigned bytes) {
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}" ::"r"(m), "r"(bytes)
                 : "memory");
}
FEMB_D void bulk_load(uint32_t dst, const void* src, unsigned bytes, uint32_t m) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(m)
                 : "memory");
}
// Waits until the barrier's phase `parity` has completed: at most 2^20 try_wait rounds,
// each suspended for a bounded, implementation-defined time; false when it gave up.
FEMB_D bool mbar_wait(uint32_t m, unsigned parity) {
    uint32_t done = 0;
    for (int it = 0; it < (1 << 20) && !done; ++it)
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                     : "=r"(done)
                     : "r"(m), "r"(parity)
                     : "memory");
    return done != 0;
}

// Inputs and output of the FP64 return near the yield-surface apex, passed by value
// so that the caller's arrays stay in registers on the common (FP32) path.
struct ApexIn {
    float tb[6], dtt[6], Fk, Pq, twoe, sphi, inv_den;
};
struct ApexOut {
    float tau[6];
};
__device__ __noinline__ ApexOut apex_increment_f64(const ApexIn in) {
    double tbd[6], dtd[6], outd[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) { tbd[c] = in.tb[c]; dtd[c] = in.dtt[c]; }
    dp_increment<double>(tbd, (double)in.Fk, dtd, (double)in.Pq, (double)in.twoe, (double)in.sphi, (double)in.inv_den,
                         eps2<double>(), outd);
    ApexOut o;
#pragma unroll
    for (int c = 0; c < 6; ++c) o.tau[c] = (float)outd[c];
    return o;
}

// The base data is read once per sweep and is larger than L2: it is loaded with an
// evict-first L2 policy so that the node arrays (δv gathers, residual atomics, the node
// update) stay resident across sweeps.
FEMB_D uint64_t l2_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
FEMB_D float ldg_stream(const float* ptr, uint64_t pol) {
    float v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(ptr), "l"(pol));
    return v;
}

// Yield values F of the base state at the three points of one quadrature row (field
// 6 of each point in the tiled layout: one 128-byte line per point and warp).
FEMB_D void load_row_F(float (&F)[3], const float* row, uint64_t pol) {
#pragma unroll
    for (int j = 0; j < 3; ++j) F[j] = ldg_stream(row + (j * BASE_FIELDS + 6) * 32, pol);
}

// Per-element data of a tile, loaded one tile ahead (during the previous tile's
// scatter) so that its latency is hidden.
struct ElemData {
    float Ji[9];
    float detJ;
    float dP[4];
    int ph, phP;
};

FEMB_D int elem_dof(const IncrArgs& a, int64_t tile, int lane, int p) {
    // padding lanes (past the last element) read the first element's DoFs
    const int64_t e = tile * 32 + lane;
    return a.dofs_linear ? (int)(4 * (e < a.nels ? e : 0) + p) : __ldg(a.dofs_t + (tile * 4 + p) * 32 + lane);
}

template <bool DIAG>
FEMB_D void load_elem(const IncrArgs& a, int64_t tile, int lane, int64_t nslots, ElemData& d) {
    const int64_t e = tile * 32 + lane;
    const float* gt = a.geo_t + tile * 10 * 32 + lane;
#pragma unroll
    for (int r = 0; r < 9; ++r) d.Ji[r] = (!DIAG || r % 4 == 0) ? __ldg(gt + r * 32) : 0.0f;
    d.detJ = __ldg(gt + 9 * 32);   // 0 on padding lanes
#pragma unroll
    for (int p = 0; p < 4; ++p) d.dP[p] = __ldg(a.dP + elem_dof(a, tile, lane, p));
    d.ph = __ldg(a.phase_t + e);
    d.phP = __ldg(a.phase_t + nslots + e);
}

// The next tile's per-element data in a thread's slots 31.. (slot s at S[s * 32]): the
// tile's ten geometry rows (J⁻¹ column-major, then |det J|) at 31..40 and its two phase
// rows at 41, 42 arrive by bulk copy; for linear pressure numbering δP at the element's
// four pressure DoFs goes to 43..46 by per-thread cp.async (its rows are element-major).
FEMB_D void load_elem_dP_async(const IncrArgs& a, int64_t tile, int lane, float* S) {
    if (a.dofs_linear) {
#pragma unroll
        for (int p = 0; p < 4; ++p) cp_async4(S + (43 + p) * 32, a.dP + elem_dof(a, tile, lane, p));
    }
}

template <bool DIAG>
FEMB_D void read_elem(const IncrArgs& a, int64_t tile, int lane, const float* S, ElemData& d) {
#pragma unroll
    for (int r = 0; r < 9; ++r) d.Ji[r] = (!DIAG || r % 4 == 0) ? S[(31 + r) * 32] : 0.0f;
    d.detJ = S[40 * 32];
    d.ph = __float_as_int(S[41 * 32]);
    d.phP = __float_as_int(S[42 * 32]);
#pragma unroll
    for (int p = 0; p < 4; ++p) d.dP[p] = a.dofs_linear ? S[(43 + p) * 32] : __ldg(a.dP + elem_dof(a, tile, lane, p));
}

// DIAG: every element's J⁻¹ is diagonal (axis-aligned boxes, the structured
// generators' meshes), so the gradient and flux transforms are one product per entry.
template <bool DIAG, bool PRE>
__global__ void __launch_bounds__(IN_THREADS, 2) hex27_incr_kernel(const IncrArgs a) {
    extern __shared__ __align__(128) float in_smem[];
    __shared__ IncrPhase PT[MAXPH];
    __shared__ __align__(8) uint64_t mbar_all[IN_WARPS];
    pdl_enter();
    for (int t = threadIdx.x; t < MAXPH; t += blockDim.x) PT[t] = a.ph[t];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t mbar = smem_addr(mbar_all + warp);
    if (lane == 0) mbar_init(mbar);
    fence_proxy_async();
    __syncthreads();
    unsigned mphase = 0;   // parity of the warp's barrier phase the next wait completes
    // shared addresses of the warp's slot 0 (lane 0 first) and of its plane slots
    const uint32_t sV = smem_addr(in_smem) + (uint32_t)(warp * IN_SLOTS * 32 * 4);
    const uint32_t sWS = sV + 162 * 32 * 4;
    float* V = in_smem + (size_t)warp * IN_SLOTS * 32 + lane;   // slot s at V[s * 32]
    int* Vi = reinterpret_cast<int*>(V);
    float* RS = V + 81 * 32;
    float* WS = V + 162 * 32;
    // the incremental sweep models the FP64 problem: its ε² is FP64's
    const float EPS2 = (float)eps2<double>();
    const int64_t ntiles = (a.nels + 31) >> 5;
    const int64_t nslots = ntiles * 32;
    const int tstride = (int)gridDim.x * IN_WARPS;
    const bool plastic = a.plastic != 0;
    // work item wk is tile wk, or the wk-th tile of the launch's list (32-bit: 2^31 tiles
    // would be 2^36 elements, more than a GPU's memory holds connectivity for)
    const int nwork = (int)(a.tile_list ? a.tile_count : ntiles);
    int wk = (int)blockIdx.x * IN_WARPS + warp;
    if (wk >= nwork) return;
    int64_t tile = a.tile_list ? __ldg(a.tile_list + wk) : wk;

    // Software pipeline across tiles: the next tile's connectivity (cp.async) and
    // δv gather (cp.async, indexed by it) run during the last quadrature plane, its
    // per-element data loads during this tile's scatter, and the base data of the
    // next quadrature row is loaded into registers while the current row computes.
    {
        const int32_t* nd = a.el2n_t + tile * 27 * 32 + lane;
#pragma unroll 9
        for (int k = 0; k < 27; ++k) {
            const int n = __ldg(nd + k * 32);
            cp_async4(V + (0 * 27 + k) * 32, a.dv[0] + n);
            cp_async4(V + (1 * 27 + k) * 32, a.dv[1] + n);
            cp_async4(V + (2 * 27 + k) * 32, a.dv[2] + n);
        }
        cp_async_commit();
    }
    // yield values of the next row's points, loaded one row ahead; the trial stress of a
    // point is read only where the elastic bound below does not settle the point
    float preF[3] = {0.0f, 0.0f, 0.0f};
    unsigned stress_reads = 0;
    unsigned needed = 0;
    // PRE (regions that yield): the trial stresses of the current row's points, loaded a
    // row ahead like the yield values; without PRE they are read on demand where the
    // elastic bound fails
    float preT[3][6] = {};
    const uint64_t pol = l2_evict_first();
    if constexpr (PRE) {
        if (plastic) {
            const float* row0 = a.base_t + tile * 27 * BASE_FIELDS * 32 + lane;
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int c = 0; c < 6; ++c) preT[j][c] = ldg_stream(row0 + (j * BASE_FIELDS + c) * 32, pol);
            stress_reads += tile * 32 + lane < a.nels ? 3u : 0u;
        }
    }
    if (plastic) load_row_F(preF, a.base_t + tile * 27 * BASE_FIELDS * 32 + lane, pol);
    ElemData cur;
    load_elem<DIAG>(a, tile, lane, nslots, cur);

    for (; wk < nwork; wk += tstride) {
        const int64_t e = tile * 32 + lane;
        const bool act = e < a.nels;
        const bool has_next = wk + tstride < nwork;
        const int64_t tnext = !has_next ? 0 : a.tile_list ? __ldg(a.tile_list + wk + tstride) : wk + tstride;
        const IncrPhase M = PT[cur.ph];
        // storage term of the continuity residual: the phase of the pressure DoFs
        const float invbulkdt = PT[cur.phP].invbulkdt;
        const float* etq = a.eta_t ? a.eta_t + tile * 27 * 32 + lane : nullptr;
        float rp[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        cp_async_wait_all();

#pragma unroll 1
        for (int qz = 0; qz < 3; ++qz) {
            const float bz[3] = {Lb(qz, 0), Lb(qz, 1), Lb(qz, 2)};
            const float dz[3] = {Ld(qz, 0), Ld(qz, 1), Ld(qz, 2)};
            const float ze = gx(qz), wz = gw(qz);
            // ζ-contraction of the plane into the thread's W slots:
            // W0 = Σ_k L_k(ζ) v_ijk, W1 = Σ_k L'_k(ζ) v_ijk
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int ij = 0; ij < 9; ++ij) {
                    const float v0 = V[(c * 27 + ij) * 32], v1 = V[(c * 27 + ij + 9) * 32], v2 = V[(c * 27 + ij + 18) * 32];
                    WS[(c * 9 + ij) * 32] = fmaf(bz[0], v0, fmaf(bz[1], v1, bz[2] * v2));
                    WS[(27 + c * 9 + ij) * 32] = fmaf(dz[0], v0, fmaf(dz[1], v1, dz[2] * v2));
                }
            // the δv slots are free from here on: the next tile's connectivity goes
            // into the first 27 of them
            if (qz == 2 && has_next) {
                // every lane has read its δv slots: one bulk copy of the next tile's 27
                // connectivity rows (3 456 B) into slots 0..26 of the warp
                fence_proxy_async();
                __syncwarp();
                if (lane == 0) {
                    mbar_expect(mbar, 27 * 32 * 4);
                    bulk_load(sV, a.el2n_t + tnext * 27 * 32, 27 * 32 * 4, mbar);
                }
            }
            // plane accumulators; the body-force term −g_c β carries the same L_k(ζ)
            // factor as the ξ/η fluxes and is folded into U0
            float U0[3][9], U1[3][9];
#pragma unroll
            for (int ij = 0; ij < 9; ++ij)
#pragma unroll
                for (int c = 0; c < 3; ++c) { U0[c][ij] = 0.0f; U1[c][ij] = 0.0f; }
#pragma unroll 1
            for (int qy = 0; qy < 3; ++qy) {
                if (qz == 2 && qy == 1 && has_next) {
                    // the connectivity has landed: gather the next tile's δv (slot k is
                    // read before the copy that overwrites it is issued)
                    if (!__all_sync(0xffffffffu, mbar_wait(mbar, mphase))) {
                        if (lane == 0) atomicExch(a.err_flag, 1);
                        return;
                    }
                    mphase ^= 1u;
#pragma unroll 9
                    for (int k = 0; k < 27; ++k) {
                        const int n = Vi[k * 32];
                        cp_async4(V + (2 * 27 + k) * 32, a.dv[2] + n);
                        cp_async4(V + (1 * 27 + k) * 32, a.dv[1] + n);
                        cp_async4(V + (0 * 27 + k) * 32, a.dv[0] + n);
                    }
                    cp_async_commit();
                }
                const float by[3] = {Lb(qy, 0), Lb(qy, 1), Lb(qy, 2)};
                const float dy[3] = {Ld(qy, 0), Ld(qy, 1), Ld(qy, 2)};
                const float et = gx(qy), wyz = gw(qy) * wz;
                // base data of this row and of the next one (rows in (qz, qy) order, then
                // the next tile's first row): each point's F register is refilled as soon
                // as the point has read it
                const float* cur_row = a.base_t + (tile * 27 + 3 * (3 * qz + qy)) * BASE_FIELDS * 32 + lane;
                const int rnext = 3 * qz + qy + 1;
                const float* next_row = rnext < 9 ? a.base_t + (tile * 27 + 3 * rnext) * BASE_FIELDS * 32 + lane
                                                  : (has_next ? a.base_t + tnext * 27 * BASE_FIELDS * 32 + lane : nullptr);
                const bool fetch = PRE && plastic && next_row;
                // η-contraction of the row: X = Σ_j L_j(η) W0, Y = Σ_j L'_j(η) W0, Z = Σ_j L_j(η) W1
                float X[3][3], Y[3][3], Z[3][3];
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        float x = 0.0f, y = 0.0f, z = 0.0f;
#pragma unroll
                        for (int j = 0; j < 3; ++j) {
                            const float w0 = WS[(c * 9 + i + 3 * j) * 32], w1 = WS[(27 + c * 9 + i + 3 * j) * 32];
                            x = fmaf(by[j], w0, x);
                            y = fmaf(dy[j], w0, y);
                            z = fmaf(by[j], w1, z);
                        }
                        X[c][i] = x; Y[c][i] = y; Z[c][i] = z;
                    }
                // the row's fluxes, contracted over ξ: A = Σ_qx L'_i F_ξ, B = Σ_qx L_i F_η,
                // C = Σ_qx L_i F_ζ, Ab = Σ_qx L_i β
                float A[3][3], Bf[3][3], Cf[3][3], Ab[3];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    Ab[i] = 0.0f;
#pragma unroll
                    for (int c = 0; c < 3; ++c) { A[c][i] = 0.0f; Bf[c][i] = 0.0f; Cf[c][i] = 0.0f; }
                }
#pragma unroll
                for (int qx = 0; qx < 3; ++qx) {
                    const int q = qx + 3 * qy + 9 * qz;
                    // reference gradient gr[c][d] = ∂δv_c/∂ξ_d at the point
                    float gr[3][3];
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f;
#pragma unroll
                        for (int i = 0; i < 3; ++i) {
                            s0 = cfma(Ld(qx, i), X[c][i], s0);
                            s1 = cfma(Lb(qx, i), Y[c][i], s1);
                            s2 = cfma(Lb(qx, i), Z[c][i], s2);
                        }
                        gr[c][0] = s0; gr[c][1] = s1; gr[c][2] = s2;
                    }
                    if (qz == 2 && qy == 2 && qx == 1) {
                        // the plane slots were last read by this row's η-contraction, whose
                        // values the first point consumed: the scatter's node indices and
                        // pressure scales go there, in flight during the last two points
                        // bulk copies: the tile's connectivity (slots 0..26) and pressure
                        // scales (27..30), the next tile's geometry rows (31..40) and phase
                        // rows (41, 42); δP per thread
                        fence_proxy_async();
                        __syncwarp();
                        if (lane == 0) {
                            mbar_expect(mbar, (27 + 4) * 32 * 4 + (has_next ? 12 * 32 * 4 : 0));
                            bulk_load(sWS, a.el2n_t + tile * 27 * 32, 27 * 32 * 4, mbar);
                            bulk_load(sWS + 27 * 128, a.pscale_t + tile * 4 * 32, 4 * 32 * 4, mbar);
                            if (has_next) {
                                bulk_load(sWS + 31 * 128, a.geo_t + tnext * 10 * 32, 10 * 32 * 4, mbar);
                                bulk_load(sWS + 41 * 128, a.phase_t + tnext * 32, 32 * 4, mbar);
                                bulk_load(sWS + 42 * 128, a.phase_t + nslots + tnext * 32, 32 * 4, mbar);
                            }
                        }
                        if (has_next) load_elem_dP_async(a, tnext, lane, WS);
                        cp_async_commit();
                    }
                    // physical gradient ∂δv_c/∂x_k = Σ_d gr[c][d] ∂ξ_d/∂x_k
                    float gq[3][3];
#pragma unroll
                    for (int c = 0; c < 3; ++c)
#pragma unroll
                        for (int k = 0; k < 3; ++k)
                            gq[c][k] = DIAG ? gr[c][k] * cur.Ji[4 * k]
                                            : fmaf(gr[c][0], cur.Ji[3 * k], fmaf(gr[c][1], cur.Ji[1 + 3 * k], gr[c][2] * cur.Ji[2 + 3 * k]));
                    const float div = gq[0][0] + gq[1][1] + gq[2][2];
                    const float xi = gx(qx);
                    const float NP0 = 1.0f - xi - et - ze;
                    const float dO = cur.detJ * gw(qx) * wyz;
                    const float Pq = fmaf(NP0, cur.dP[0], cfma(xi, cur.dP[1], fmaf(et, cur.dP[2], ze * cur.dP[3])));
                    // continuity: −∇·δv − δP/(bulk·Δt) (pressure_residual.jl:132-158)
                    const float f = (-div - Pq * invbulkdt) * dO;
                    rp[0] = fmaf(NP0, f, rp[0]);
                    rp[1] = cfma(xi, f, rp[1]);
                    rp[2] = fmaf(et, f, rp[2]);
                    rp[3] = fmaf(ze, f, rp[3]);
                    // deviatoric strain-rate increment and the stress increment
                    const float tr = div * (1.0f / 3.0f);
                    const float ed[6] = {gq[0][0] - tr, gq[1][1] - tr, gq[2][2] - tr, 0.5f * (gq[0][1] + gq[1][0]),
                                         0.5f * (gq[0][2] + gq[2][0]), 0.5f * (gq[1][2] + gq[2][1])};
                    float twoe = M.twoe, inv_den = M.inv_den;
                    if (etq) {
                        const float eq = act ? __ldg(etq + q * 32) : 1.0f;
                        const float etave = 1.0f / (1.0f / eq + M.invG_dt);
                        twoe = 2.0f * etave;
                        inv_den = 1.0f / (etave + M.den_rest);
                    }
                    float dtt[6], tau[6];
#pragma unroll
                    for (int c = 0; c < 6; ++c) dtt[c] = twoe * ed[c];
                    if (plastic) {
                        const float Fk = preF[qx];
                        if (next_row) preF[qx] = ldg_stream(next_row + (qx * BASE_FIELDS + 6) * 32, pol);
                        float tbp[6];
#pragma unroll
                        for (int c = 0; c < 6; ++c) tbp[c] = preT[qx][c];
                        if (fetch) {
#pragma unroll
                            for (int c = 0; c < 6; ++c) preT[qx][c] = ldg_stream(next_row + (qx * BASE_FIELDS + c) * 32, pol);
                            stress_reads += act ? 1u : 0u;
                        }
                        // Elastic bound: τII = sqrt(‖τ‖² + ε²) is 1-Lipschitz in the J2 norm
                        // ‖τ‖² = ½Σ τ_ii² + Σ_{i<j} τ_ij², so the trial yield value satisfies
                        // F(τb + δτ) ≤ F_k + ‖δτ‖ + sinϕ·|δP|. Where that bound (with a 1e-3
                        // relative margin over the rounding of either path) stays negative,
                        // base and trial are both elastic, the return leaves the increment
                        // unchanged (dp_increment gives δτ exactly), and the base trial
                        // stress is not needed.
                        const float dd = 0.5f * (dtt[0] * dtt[0] + dtt[1] * dtt[1] + dtt[2] * dtt[2]) + dtt[3] * dtt[3] +
                                         dtt[4] * dtt[4] + dtt[5] * dtt[5];
                        // (sqrt(dd) + |sinϕ·δP|)·1.001 + 1e-20 < −F_k, compared on squares
                        const float lim = -(Fk + 1e-20f) * 0.999000999f - fabsf(M.sphi * Pq);
                        if (lim > 0.0f && dd < lim * lim) {
#pragma unroll
                            for (int c = 0; c < 6; ++c) tau[c] = dtt[c];
                        } else {
                        needed += act ? 1u : 0u;
                        float tb[6];
                        if constexpr (PRE) {
#pragma unroll
                            for (int c = 0; c < 6; ++c) tb[c] = tbp[c];
                        } else {
                            stress_reads += act ? 1u : 0u;
#pragma unroll
                            for (int c = 0; c < 6; ++c) tb[c] = ldg_stream(cur_row + (qx * BASE_FIELDS + c) * 32, pol);
                        }
                        const float Jk = 0.5f * (tb[0] * tb[0] + tb[1] * tb[1] + tb[2] * tb[2]) + tb[3] * tb[3] +
                                         tb[4] * tb[4] + tb[5] * tb[5];
                        if (Jk < 1e-6f * M.cC * M.cC) {
                            // within 1e-3·C·cosϕ of the yield-surface apex the return direction
                            // is ill-conditioned: this point's increment is formed in FP64 (out of
                            // line, so that the rare branch does not raise the register count)
                            ApexIn in;
#pragma unroll
                            for (int c = 0; c < 6; ++c) { in.tb[c] = tb[c]; in.dtt[c] = dtt[c]; }
                            in.Fk = Fk; in.Pq = Pq; in.twoe = twoe; in.sphi = M.sphi; in.inv_den = inv_den;
                            const ApexOut o = apex_increment_f64(in);
#pragma unroll
                            for (int c = 0; c < 6; ++c) tau[c] = o.tau[c];
                        } else {
                            dp_increment<float, true>(tb, Fk, dtt, Pq, twoe, M.sphi, inv_den, EPS2, tau);
                        }
                        }
                    } else {
#pragma unroll
                        for (int c = 0; c < 6; ++c) tau[c] = dtt[c];
                    }
                    // reference-frame fluxes F[c][d] = dΩ Σ_k ∂ξ_d/∂x_k σ_kc, σ = δτ − δP·I
                    const float sg[3][3] = {{tau[0] - Pq, tau[3], tau[4]}, {tau[3], tau[1] - Pq, tau[5]}, {tau[4], tau[5], tau[2] - Pq}};
                    // EOS density increment ρ0·δP/K (momentum_residuals.jl:11-16)
                    const float bq = M.rho0beta * Pq * dO;
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        float F[3];
#pragma unroll
                        for (int d = 0; d < 3; ++d)
                            F[d] = DIAG ? dO * cur.Ji[4 * d] * sg[d][c]
                                        : dO * fmaf(cur.Ji[d], sg[0][c], fmaf(cur.Ji[d + 3], sg[1][c], cur.Ji[d + 6] * sg[2][c]));
#pragma unroll
                        for (int i = 0; i < 3; ++i) {
                            A[c][i] = cfma(Ld(qx, i), F[0], A[c][i]);
                            Bf[c][i] = cfma(Lb(qx, i), F[1], Bf[c][i]);
                            Cf[c][i] = cfma(Lb(qx, i), F[2], Cf[c][i]);
                        }
                    }
#pragma unroll
                    for (int i = 0; i < 3; ++i) Ab[i] = cfma(Lb(qx, i), bq, Ab[i]);
                }
                // contract the row over η: U0 += L_j(η) (A − g_c Ab) + L'_j(η) B, U1 += L_j(η) C
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        const float ag = fmaf(-a.g[c], Ab[i], A[c][i]);
#pragma unroll
                        for (int j = 0; j < 3; ++j) {
                            U0[c][i + 3 * j] = fmaf(by[j], ag, fmaf(dy[j], Bf[c][i], U0[c][i + 3 * j]));
                            U1[c][i + 3 * j] = fmaf(by[j], Cf[c][i], U1[c][i + 3 * j]);
                        }
                    }
            }
            // expand the plane: R_c(ijk) += L_k(ζ) U0 + L'_k(ζ) U1
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int k = 0; k < 3; ++k)
#pragma unroll
                    for (int ij = 0; ij < 9; ++ij) {
                        const float r = fmaf(bz[k], U0[c][ij], dz[k] * U1[c][ij]);
                        float* slot = RS + (c * 27 + ij + 9 * k) * 32;
                        *slot = qz == 0 ? r : *slot + r;
                    }
        }
        // ---- pressure residual and Pnum increments (element-local) ----
        cp_async_wait_all();
        if (!__all_sync(0xffffffffu, mbar_wait(mbar, mphase))) {
            if (lane == 0) atomicExch(a.err_flag, 1);
            return;
        }
        mphase ^= 1u;
        float Pn[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            Pn[p] = WS[(27 + p) * 32] * rp[p];
            if (act) a.RPinc[elem_dof(a, tile, lane, p)] = rp[p];
        }
        const float* Ji = cur.Ji;
        const float detJ = cur.detJ;
        // ---- scatter, with the Pnum term −|det J| Σ_d ∂ξ_d/∂x_c Σ_p Pn_p K[p][d][a] ----
        // nodes (ξ, η, ζ) = (i, j, k) in groups of one (j, k) line
#pragma unroll 1
        for (int jk = 0; jk < 9; ++jk) {
            float val[3][3];
            int n[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int t = 3 * jk + i;
                float S[3];
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    S[d] = fmaf(Pn[0], c_inc_K[0][d][t], fmaf(Pn[1], c_inc_K[1][d][t], fmaf(Pn[2], c_inc_K[2][d][t], Pn[3] * c_inc_K[3][d][t])));
                n[i] = __float_as_int(WS[t * 32]);
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    val[i][c] = RS[(c * 27 + t) * 32] -
                                detJ * (DIAG ? Ji[4 * c] * S[c] : fmaf(Ji[3 * c], S[0], fmaf(Ji[3 * c + 1], S[1], Ji[3 * c + 2] * S[2])));
            }
            // when the next lane's element shares this line's ξ = +1 node as its ξ = −1
            // node (tiles that run along ξ), its contribution is added here and one
            // atomic per component is saved; any shared node folds correctly
            const int n0n = __shfl_down_sync(0xffffffffu, n[0], 1);
            const int actn = __shfl_down_sync(0xffffffffu, (int)act, 1);
            const bool fold = lane < 31 && actn && n0n == n[2];
            const bool folded = __shfl_up_sync(0xffffffffu, (int)fold, 1) && lane > 0;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float v0n = __shfl_down_sync(0xffffffffu, val[0][c], 1);
                if (fold) val[2][c] += v0n;
            }
            if (act) {
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    if (!folded) atomicAdd(a.R[c] + n[0], val[0][c]);
                    atomicAdd(a.R[c] + n[1], val[1][c]);
                    atomicAdd(a.R[c] + n[2], val[2][c]);
                }
            }
        }
        if (has_next) read_elem<DIAG>(a, tnext, lane, WS, cur);
        tile = tnext;
    }
    cp_async_wait_all();
    if (a.stress_reads) {
        unsigned n = stress_reads;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) n += __shfl_down_sync(0xffffffffu, n, o);
        if (lane == 0 && n) atomicAdd(a.stress_reads, (unsigned long long)n);
    }
    if (a.bound_failures) {
        unsigned n = needed;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) n += __shfl_down_sync(0xffffffffu, n, o);
        if (lane == 0 && n) atomicAdd(a.bound_failures, (unsigned long long)n);
    }
}

std::mutex g_inc_mutex;
bool g_inc_ready[64] = {};

}  // namespace

cudaError_t launch_incr_tiles(const IncrTileSrc& src, int64_t nels, const IncrArgs& dst, int32_t* flags,
                              cudaStream_t st) {
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    {
        // the Pnum table and the kernel's shared-memory limit, once per device
        std::lock_guard<std::mutex> lk(g_inc_mutex);
        if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
        if (!g_inc_ready[dev]) {
            static float K[4][3][27];
            host_pnum_table(K);
            err = cudaMemcpyToSymbol(c_inc_K, K, sizeof(K));
            if (err != cudaSuccess) return err;
            for (auto fn : {hex27_incr_kernel<false, false>, hex27_incr_kernel<true, false>, hex27_incr_kernel<false, true>,
                            hex27_incr_kernel<true, true>}) {
                err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           IN_WARPS * IN_SLOTS * 32 * (int)sizeof(float));
                if (err != cudaSuccess) return err;
            }
            g_inc_ready[dev] = true;
        }
    }
    const int64_t nslots = (nels + 31) / 32 * 32;
    count_launch();
    incr_tiles_kernel<<<(unsigned)((nslots + 255) / 256), 256, 0, st>>>(src, nels, nslots, dst, flags);
    return cudaGetLastError();
}

namespace {
__global__ void add_f32_kernel(float* out, const float* x, const float* y, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = x[i] + y[i];
}
}  // namespace

cudaError_t launch_add_f32(float* out, const float* x, const float* y, int64_t n, cudaStream_t st) {
    count_launch();
    const int64_t blocks = std::min<int64_t>((n + 255) / 256, 148 * 8);
    add_f32_kernel<<<(unsigned)std::max<int64_t>(blocks, 1), 256, 0, st>>>(out, x, y, n);
    return cudaGetLastError();
}

int64_t incr_warp_slots(int num_sms) {
    int per_sm = 2;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hex27_incr_kernel<true, false>, IN_THREADS,
                                                  (size_t)IN_WARPS * IN_SLOTS * 32 * sizeof(float));
    return (int64_t)num_sms * std::max(per_sm, 1) * IN_WARPS;
}

cudaError_t launch_hex27_incr(const IncrArgs& a, int num_sms, cudaStream_t st, bool pdl) {
    const size_t smem = (size_t)IN_WARPS * IN_SLOTS * 32 * sizeof(float);
    const int64_t ntiles = a.tile_list ? a.tile_count : (a.nels + 31) / 32;
    if (ntiles < 1) return cudaSuccess;
    auto fn = a.diag_geometry ? (a.prefetch_stress ? hex27_incr_kernel<true, true> : hex27_incr_kernel<true, false>)
                              : (a.prefetch_stress ? hex27_incr_kernel<false, true> : hex27_incr_kernel<false, false>);
    int per_sm = 2;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, IN_THREADS, smem);
    if (per_sm < 1) per_sm = 1;
    int64_t blocks = (ntiles + IN_WARPS - 1) / IN_WARPS;
    blocks = std::min<int64_t>(blocks, (int64_t)num_sms * per_sm);
    if (blocks < 1) blocks = 1;
    count_launch();
    return launch_pdl(pdl, fn, dim3((unsigned)blocks), dim3(IN_THREADS), smem, st, a);
}

}  // namespace femb
