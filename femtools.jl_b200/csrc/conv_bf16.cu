// conv_bf16.cu — BF16 tensor-core 3×3 convolutions (FP32 accumulation) for the learned
// warm-start network, and its training kernels (loss, Adam). No reference counterpart:
// FEMTools.jl has no learned component; this is the network that predicts the next
// time step's v/P from the solver's own converged history.
//
// Layout: activations NHWC BF16 with C ∈ {16, 32} channels (unused channels zero);
// weights [co][9·ci + 8] BF16 (k = tap·ci + c, tap = 3·ky + kx; eight padding entries
// per row).
//
// Both contractions run on the sm_100a tensor cores (tcgen05.mma, kind::f16, BF16
// operands from shared memory, FP32 accumulators in tensor memory), on tiles of four output
// rows × 128 pixels: the six staged input rows of a tile serve all four, which halves the
// bytes moved from L2 into shared memory per output pixel against one-row tiles.
//
// * convolution (forward, and the data gradient on the flipped transposed weights): an
//   implicit GEMM per output row with M = 128 pixels, N = co and K = 9·ci. The staged rows
//   keep 8 channels per 16-byte row of a core matrix, so that the A operand of tap (ky, kx)
//   is the staged block shifted by (u + ky)·130 + kx pixels: a start address in the
//   descriptor, no im2col copy. One thread issues the MMAs of the tile's four rows.
// * weight gradient: per tap an MMA with M = channel, N = co, K = the 128 pixels of one
//   row, both operands MN-major, reading the staged rows directly; the accumulators stay in
//   tensor memory over all the tiles a CTA visits, and each CTA adds its sums to dw once.
// Both kernels are persistent and stage the next tiles with cp.async while the current
// one's MMAs and epilogue run.
#include <cuda_bf16.h>
#include <algorithm>
#include <mutex>
#include "kernels.cuh"
#include "tc05.cuh"

namespace femb {
namespace {

using tc05::smem_u32;

FEMB_D uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}
FEMB_D float bf16_lo(uint32_t w) { return __bfloat162float(__ushort_as_bfloat16((unsigned short)(w & 0xffffu))); }
FEMB_D float bf16_hi(uint32_t w) { return __bfloat162float(__ushort_as_bfloat16((unsigned short)(w >> 16))); }

constexpr int SEG = 128;                     // output pixels of one image-row segment (the MMA's M)
constexpr int HALO = SEG + 2;                // staged input pixels per row
constexpr int FROWS = 4;                     // output rows of a convolution tile
constexpr int FSLAB = (FROWS + 2) * HALO * 16;   // bytes of one 8-channel slab of its staged rows
constexpr int FWD_THREADS = 256;             // 8 warps: warp w reads TMEM lanes 32·(w mod 4)..

FEMB_D void cp_async16(void* dst, const void* src, bool valid) {
    // 16 bytes global → shared; zero-filled where `valid` is false (src is then not read)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}
FEMB_D void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> FEMB_D void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// A tile: rows [y, y + ROWS) × pixels [x0, x0 + 128) of image b; tiles are numbered row
// block by row block (tile indices fit in 32 bits, checked on the host).
struct Seg {
    int b, y, x0;
};
template <int ROWS>
FEMB_D Seg seg_of(int t, int nseg, int nrb) {
    const int rb = t / nseg;
    return Seg{rb / nrb, (rb % nrb) * ROWS, (t - rb * nseg) * SEG};
}

// Stages the NR input rows y − 1 .. y + NR − 2 of a tile with their halo columns: 8-channel
// slab s, row r, pixel xx (input column x0 − 1 + xx) at ((s·NR + r)·HALO + xx)·16 bytes,
// zero outside the grid. Consecutive threads copy consecutive 16-byte chunks of an input
// row (the slabs of a pixel, then the next pixel), so each warp reads whole sectors.
template <int CI, int NR, int NTH>
FEMB_D void stage_halo(uint8_t* dst, const __nv_bfloat16* in, Seg g, int H, int W, int tid) {
    constexpr int NS = CI / 8, LOG = NS == 4 ? 2 : 1, PER_ROW = HALO * NS;
    static_assert(NS == 2 || NS == 4, "16 or 32 channels");
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        const int gy = g.y - 1 + r;
        const bool row = gy >= 0 && gy < H;
        const __nv_bfloat16* rowp = in + ((int64_t)g.b * H + (row ? gy : 0)) * W * CI;
#pragma unroll
        for (int k = 0; k < (PER_ROW + NTH - 1) / NTH; ++k) {
            const int i = tid + k * NTH;
            if (i < PER_ROW) {
                const int sl = i & (NS - 1), xx = i >> LOG;
                const int gx = g.x0 - 1 + xx;
                const bool v = row && gx >= 0 && gx < W;
                cp_async16(dst + ((sl * NR + r) * HALO + xx) * 16, v ? rowp + (int64_t)gx * CI + 8 * sl : in, v);
            }
        }
    }
}

// Shared memory of the convolution: the weights (16-byte chunk j of row co at
// (j·co_n + co)·16), NSTAGE halo stages of FROWS + 2 rows, the bias, the mbarrier and the
// TMEM address slot.
constexpr int NSTAGE = 3;
template <int CI, int CO> struct ConvSmem {
    static constexpr int A = CI / 8 * FSLAB;
    static constexpr int B = 9 * CI / 8 * CO * 16;
    static constexpr int BIAS = B + NSTAGE * A;
    static constexpr int BAR = BIAS + CO * 4;
    static constexpr int BYTES = BAR + 32;
};

// MODE 0: out = ReLU(conv + bias), BF16.  MODE 1: out = conv + bias, FP32.
// MODE 2: out = conv where mask > 0 else 0, BF16 (data gradient through a ReLU; no bias).
// A tile is FROWS output rows × 128 pixels: FROWS + 2 staged input rows serve all of them
// (1.5 staged rows per output row instead of 3). Output row u of the tile accumulates in
// TMEM columns u·co.., from A blocks that start ((u + ky)·HALO + kx) staged pixels into
// the stage. Persistent: the CTA visits tiles blockIdx.x, blockIdx.x + gridDim.x, ...; the
// halos of the next two tiles are in flight (cp.async into the other stages) while the
// current one's MMAs and epilogue run. Warps w and w + 4 share TMEM lane quadrant w and
// write rows 0, 1 and 2, 3 of the tile.
template <int CI, int CO, int MODE>
__global__ void __launch_bounds__(FWD_THREADS) conv3x3_tc_kernel(const __nv_bfloat16* __restrict__ in,
                                                                const __nv_bfloat16* __restrict__ wt,
                                                                const float* __restrict__ bias,
                                                                const __nv_bfloat16* __restrict__ mask, void* out, int B,
                                                                int H, int W, int* err) {
    using S = ConvSmem<CI, CO>;
    constexpr uint32_t TCOLS = FROWS * CO <= 64 ? 64 : 128;
    static_assert(FROWS * CO <= 128 && FWD_THREADS == 2 * 128 && FROWS == 4, "two rows per warp");
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t* sB = smem;
    uint8_t* sA = smem + S::B;   // stage k at sA + k·S::A
    float* sbias = reinterpret_cast<float*>(smem + S::BIAS);
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + S::BAR);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + S::BAR + 16);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int quad = warp & 3, half = warp >> 2;   // TMEM lanes 32·quad.., tile rows 2·half, 2·half + 1
    const int nseg = (W + SEG - 1) / SEG, nrb = (H + FROWS - 1) / FROWS;
    const int ntile = B * nrb * nseg;
    if (warp == 0) tc05::tmem_alloc(smem_u32(tslot), TCOLS);
    if (tid == 0) {
        tc05::mbar_init(smem_u32(mbar));
        tc05::fence_mbar_init();
    }
    if (tid < CO) sbias[tid] = MODE == 2 ? 0.0f : __ldg(bias + tid);
    {
        constexpr int KP8 = (9 * CI + 8) / 8;   // 16-byte chunks of a weight row
        for (int i = tid; i < 9 * CI / 8 * CO; i += FWD_THREADS) {
            const int co = i % CO, j = i / CO;
            cp_async16(sB + (j * CO + co) * 16, wt + (co * KP8 + j) * 8, true);
        }
    }
    const int G = (int)gridDim.x;
    int t = blockIdx.x;
    // prologue: the halos of the first two tiles (the weights travel in the first group)
#pragma unroll
    for (int k = 0; k < NSTAGE - 1; ++k) {
        if (t + k * G < ntile)
            stage_halo<CI, FROWS + 2, FWD_THREADS>(sA + k * S::A, in, seg_of<FROWS>(t + k * G, nseg, nrb), H, W, tid);
        cp_async_commit();
    }
    tc05::fence_before_sync();
    __syncthreads();
    tc05::fence_after_sync();
    const uint32_t tbase = *tslot;
    constexpr uint32_t idesc = tc05::idesc_bf16_f32<SEG, CO>();
    // descriptors of stage 0 and of the weights; offsets are added in 16-byte units to the
    // start-address field (shared addresses stay below 2^18 bytes)
    const uint64_t adesc0 = tc05::smem_desc(smem_u32(sA), FSLAB, 128);
    const uint64_t bdesc0 = tc05::smem_desc(smem_u32(sB), CO * 16, 128);
    uint32_t phase = 0u;
    int st = 0;   // stage of tile t
    for (; t < ntile; t += G, st = st == NSTAGE - 1 ? 0 : st + 1) {
        cp_async_wait<NSTAGE - 2>();   // every group but the newest: this tile's halo
        tc05::fence_async_smem();
        tc05::fence_before_sync();
        __syncthreads();
        tc05::fence_after_sync();
        if (tid == 0) {
            const uint64_t ab = adesc0 + (uint64_t)(st * S::A / 16);
#pragma unroll
            for (int tap = 0; tap < 9; ++tap)
#pragma unroll
                for (int c0 = 0; c0 < CI; c0 += 16)
#pragma unroll
                    for (int u = 0; u < FROWS; ++u) {
                        // rows m of output row u, tap (ky, kx): staged pixels (u + ky)·HALO + kx + m
                        // of slabs c0/8, c0/8 + 1
                        const uint64_t ad = ab + (uint64_t)((c0 / 8) * (FSLAB / 16) + (u + tap / 3) * HALO + tap % 3);
                        const uint64_t bd = bdesc0 + (uint64_t)((tap * CI + c0) / 8 * CO);
                        tc05::mma_bf16(tbase + u * CO, ad, bd, idesc, tap > 0 || c0 > 0);
                    }
            tc05::commit(smem_u32(mbar));
        }
        // while the MMAs run: the tile two ahead goes into the stage the previous tile's
        // (completed) MMAs read
        const int ta = t + (NSTAGE - 1) * G;
        const int sa = st == 0 ? NSTAGE - 1 : st - 1;
        if (ta < ntile) stage_halo<CI, FROWS + 2, FWD_THREADS>(sA + sa * S::A, in, seg_of<FROWS>(ta, nseg, nrb), H, W, tid);
        cp_async_commit();
        const bool ok = __syncthreads_and(tid != 0 || tc05::mbar_poll(smem_u32(mbar), phase)) != 0;
        phase ^= 1u;
        if (!ok) {
            if (tid == 0) atomicExch(err, 1);
            break;
        }
        tc05::fence_after_sync();
        const Seg cur = seg_of<FROWS>(t, nseg, nrb);
        const int gx = cur.x0 + quad * 32 + lane;
#pragma unroll
        for (int uu = 0; uu < 2; ++uu) {
            const int u = 2 * half + uu;
            float acc[CO / 16][16];
#pragma unroll
            for (int c = 0; c < CO / 16; ++c)
                tc05::tmem_ld16(tbase + ((uint32_t)(quad * 32) << 16) + u * CO + c * 16, acc[c]);
            const int gy = cur.y + u;
            if (gx >= W || gy >= H) continue;
            const int64_t pix = ((int64_t)cur.b * H + gy) * W + gx;
            {
            if constexpr (MODE == 1) {
                float4* o = reinterpret_cast<float4*>(static_cast<float*>(out) + pix * CO);
#pragma unroll
                for (int q = 0; q < CO / 4; ++q) {
                    const int c = 4 * q;
                    o[q] = make_float4(acc[c / 16][c % 16] + sbias[c], acc[c / 16][c % 16 + 1] + sbias[c + 1],
                                       acc[c / 16][c % 16 + 2] + sbias[c + 2], acc[c / 16][c % 16 + 3] + sbias[c + 3]);
                }
            } else {
                uint4* o = reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(out) + pix * CO);
                const uint4* mk = MODE == 2 ? reinterpret_cast<const uint4*>(mask + pix * CO) : nullptr;
#pragma unroll
                for (int q = 0; q < CO / 8; ++q) {
                    uint32_t w[4];
                    uint4 m4 = make_uint4(0u, 0u, 0u, 0u);
                    if constexpr (MODE == 2) m4 = __ldg(mk + q);
                    const uint32_t mw[4] = {m4.x, m4.y, m4.z, m4.w};
#pragma unroll
                    for (int h = 0; h < 4; ++h) {
                        const int c = 8 * q + 2 * h;
                        float v0 = acc[c / 16][c % 16], v1 = acc[c / 16][c % 16 + 1];
                        if constexpr (MODE == 0) {
                            v0 = fmaxf(v0 + sbias[c], 0.0f);
                            v1 = fmaxf(v1 + sbias[c + 1], 0.0f);
                        }
                        if constexpr (MODE == 2) {
                            if (!(bf16_lo(mw[h]) > 0.0f)) v0 = 0.0f;
                            if (!(bf16_hi(mw[h]) > 0.0f)) v1 = 0.0f;
                        }
                        w[h] = pack2(__float2bfloat16(v0), __float2bfloat16(v1));
                    }
                    o[q] = make_uint4(w[0], w[1], w[2], w[3]);
                }
            }
            }
        }
        // every thread's TMEM reads are done before the next tile's MMAs overwrite them
        tc05::fence_before_sync();
    }
    cp_async_wait<0>();
    tc05::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc05::tmem_dealloc(tbase, TCOLS);
}

// Weight gradient: dW[co][(3·ky + kx)·ci + c] = Σ_p X[p + (ky−1, kx−1)][c]·dY[p][co] over
// the pixels of tiles of FROWS rows × 128. The MMA is MN-major on both operands. A
// (M = 128 rows, K = pixel) is the staged input itself, stored row-major by slabs — staged
// row r, slab s, pixel xx at ((r·ns + s)·HALO + xx)·16 — so that consecutive 8-channel groups
// lie one staged row apart (HALO·16 bytes): an A block that starts at output row u's first
// input row and column kx holds, in rows ky·ci + c, the input of kernel row ky for every ky
// at once. B (N = co, K = pixel) is the staged output gradient of row u,
// ((u·co/8 + s)·SEG + p)·16. One MMA per (row, kx, K step) thus accumulates all three kernel
// rows of column kx into TMEM columns kx·co + n, lanes ky·ci + c; rows 3·ci.. of the block
// read further into the stage (inside the CTA's allocation) and fill accumulator rows that
// are never read. The accumulators stay in tensor memory over every tile the CTA visits.
constexpr int WG_THREADS = 256;
template <int CI, int CO> struct WgradSmem {
    static constexpr int NS = CI / 8, NSO = CO / 8, NR = FROWS + 2;
    static constexpr int A = NR * NS * HALO * 16;            // staged input rows
    static constexpr int BY = FROWS * NSO * SEG * 16;        // staged output gradient
    static constexpr int STAGE = A + BY;
    // last byte an A block can reach from its stage's start, plus one
    static constexpr int REACH = ((FROWS - 1) * NS * HALO + 2 + SEG - 16) * 16 + 15 * HALO * 16 + 256;
    static constexpr int TAIL = REACH > STAGE ? REACH - STAGE : 0;
    static constexpr int BYTES = 2 * STAGE + TAIL + 32;
    static constexpr int COLS = 3 * CO;
    static constexpr int TCOLS = COLS <= 64 ? 64 : 128;
    static_assert(3 * CI <= 128, "the three kernel rows of a column in one M = 128 block");
};

// Stages the input rows of a tile for the weight gradient (row-major slabs, see above).
template <int CI>
FEMB_D void stage_rows_wg(uint8_t* dst, const __nv_bfloat16* in, Seg g, int H, int W, int tid) {
    constexpr int NS = CI / 8, LOG = NS == 4 ? 2 : 1, PER_ROW = HALO * NS;
#pragma unroll
    for (int r = 0; r < FROWS + 2; ++r) {
        const int gy = g.y - 1 + r;
        const bool row = gy >= 0 && gy < H;
        const __nv_bfloat16* rowp = in + ((int64_t)g.b * H + (row ? gy : 0)) * W * CI;
#pragma unroll
        for (int k = 0; k < (PER_ROW + WG_THREADS - 1) / WG_THREADS; ++k) {
            const int i = tid + k * WG_THREADS;
            if (i < PER_ROW) {
                const int sl = i & (NS - 1), xx = i >> LOG;
                const int gx = g.x0 - 1 + xx;
                const bool v = row && gx >= 0 && gx < W;
                cp_async16(dst + ((r * NS + sl) * HALO + xx) * 16, v ? rowp + (int64_t)gx * CI + 8 * sl : in, v);
            }
        }
    }
}

template <int CI, int CO>
__global__ void __launch_bounds__(WG_THREADS) conv3x3_wgrad_tc_kernel(const __nv_bfloat16* __restrict__ x,
                                                                     const __nv_bfloat16* __restrict__ dy, float* dw,
                                                                     int B, int H, int W, int* err) {
    using S = WgradSmem<CI, CO>;
    extern __shared__ __align__(128) uint8_t smem[];
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + 2 * S::STAGE + S::TAIL);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + 2 * S::STAGE + S::TAIL + 16);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nseg = (W + SEG - 1) / SEG, nrb = (H + FROWS - 1) / FROWS;
    const int ntile = B * nrb * nseg;
    if (warp == 0) tc05::tmem_alloc(smem_u32(tslot), S::TCOLS);
    if (tid == 0) {
        tc05::mbar_init(smem_u32(mbar));
        tc05::mbar_init(smem_u32(mbar + 1));
        tc05::fence_mbar_init();
    }
    // input rows and the output gradient of a tile (consecutive threads: consecutive chunks)
    auto stage = [&](Seg g, uint8_t* dst) {
        stage_rows_wg<CI>(dst, x, g, H, W, tid);
        constexpr int LOG = S::NSO == 4 ? 2 : 1;
#pragma unroll
        for (int u = 0; u < FROWS; ++u) {
            const bool row = g.y + u < H;
            const __nv_bfloat16* rowp = dy + (((int64_t)g.b * H + (row ? g.y + u : 0)) * W + g.x0) * CO;
#pragma unroll
            for (int k = 0; k < SEG * S::NSO / WG_THREADS; ++k) {
                const int i = tid + k * WG_THREADS;
                const int sl = i & (S::NSO - 1), p = i >> LOG;
                const bool v = row && g.x0 + p < W;
                cp_async16(dst + S::A + ((u * S::NSO + sl) * SEG + p) * 16, v ? rowp + p * CO + 8 * sl : dy, v);
            }
        }
    };
    int t = blockIdx.x;
    if (t < ntile) stage(seg_of<FROWS>(t, nseg, nrb), smem);
    cp_async_commit();
    tc05::fence_before_sync();
    __syncthreads();
    tc05::fence_after_sync();
    const uint32_t tbase = *tslot;
    // A and B both MN-major (bits 15 and 16 of the instruction descriptor)
    constexpr uint32_t idesc = tc05::idesc_bf16_f32<128, CO>() | (1u << 15) | (1u << 16);
    const uint64_t adesc0 = tc05::smem_desc(smem_u32(smem), 128, HALO * 16);
    const uint64_t bdesc0 = tc05::smem_desc(smem_u32(smem + S::A), 128, SEG * 16);
    uint32_t phases = 0u;   // bit k: parity of the next completion of mbarrier k
    bool ok = true, any = false;
    for (int it = 0; t < ntile; ++it, t += gridDim.x) {
        const int buf = it & 1;
        cp_async_wait<0>();   // this tile's rows
        tc05::fence_async_smem();
        tc05::fence_before_sync();
        __syncthreads();
        tc05::fence_after_sync();
        if (tid == 0) {
            const uint64_t ab = adesc0 + (uint64_t)(buf * S::STAGE / 16), bb = bdesc0 + (uint64_t)(buf * S::STAGE / 16);
            // consecutive MMAs accumulate into different kernel columns' accumulators
#pragma unroll 1
            for (int ks = 0; ks < SEG / 16; ++ks)
#pragma unroll
                for (int u = 0; u < FROWS; ++u)
#pragma unroll
                    for (int kx = 0; kx < 3; ++kx)
                        tc05::mma_bf16(tbase + kx * CO, ab + (uint64_t)(u * S::NS * HALO + kx + 16 * ks),
                                       bb + (uint64_t)(u * S::NSO * SEG + 16 * ks), idesc, any || ks > 0 || u > 0);
            tc05::commit(smem_u32(mbar + buf));
        }
        // while the MMAs run: the next tile goes into the other stage, whose MMAs (the
        // previous tile's) have completed
        const int tn = t + (int)gridDim.x;
        if (tn < ntile) stage(seg_of<FROWS>(tn, nseg, nrb), smem + (buf ^ 1) * S::STAGE);
        cp_async_commit();
        any = true;
        // the stage is re-filled only after the MMAs that read it completed
        ok = __syncthreads_and(tid != 0 || tc05::mbar_poll(smem_u32(mbar + buf), (phases >> buf) & 1u)) != 0;
        phases ^= 1u << buf;
        if (!ok) break;
    }
    cp_async_wait<0>();
    if (ok && any) {
        tc05::fence_after_sync();
        // accumulator row m = ky·ci + c sits in TMEM lane m: warp w < 4 reads lanes 32w..
        const int m = warp * 32 + lane, ky = m / CI, ch = m % CI;
        if (warp < 4 && warp * 32 < 3 * CI) {
            constexpr int KP = 9 * CI + 8;
#pragma unroll 1
            for (int kx = 0; kx < 3; ++kx)
#pragma unroll
                for (int c = 0; c < CO / 16; ++c) {
                    float v[16];
                    tc05::tmem_ld16(tbase + ((uint32_t)(warp * 32) << 16) + kx * CO + c * 16, v);
                    if (ky < 3) {
#pragma unroll
                        for (int i = 0; i < 16; ++i)
                            atomicAdd(dw + (int64_t)(c * 16 + i) * KP + (3 * ky + kx) * CI + ch, v[i]);
                    }
                }
        }
    } else if (!ok && tid == 0) {
        atomicExch(err, 1);
    }
    tc05::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc05::tmem_dealloc(tbase, S::TCOLS);
}

// db[co] += Σ_p dY[p][co]
template <int CO>
__global__ void bias_grad_kernel(const __nv_bfloat16* __restrict__ dy, float* db, int64_t npix) {
    __shared__ float red[CO];
    if (threadIdx.x < CO) red[threadIdx.x] = 0.0f;
    __syncthreads();
    float acc = 0.0f;
    const int c = threadIdx.x % CO;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npix * CO; i += (int64_t)gridDim.x * blockDim.x)
        acc += __bfloat162float(dy[i]);
    atomicAdd(&red[c], acc);
    __syncthreads();
    if (threadIdx.x < CO) atomicAdd(db + threadIdx.x, red[threadIdx.x]);
}

// W'[ci][tap'·co + c] = W[c][tap·ci + ci] with tap' = 8 − tap (the data-gradient weights)
__global__ void flip_weights_kernel(const __nv_bfloat16* __restrict__ w, __nv_bfloat16* wT, int ci, int co) {
    const int kp = 9 * ci + 8, kpT = 9 * co + 8;
    const int n = ci * kpT;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int r = i / kpT, k = i % kpT;   // r: output channel of the gradient (= ci), k = tap'·co + c
        __nv_bfloat16 v = __float2bfloat16(0.0f);
        if (k < 9 * co) {
            const int tapT = k / co, c = k % co;
            v = w[c * kp + (8 - tapT) * ci + r];
        }
        wT[i] = v;
    }
}

// MSE over the first nt channels of an FP32 output (channels co) against an FP32
// target (channels nt): dY = 2·scale·(out − target) as BF16 (other channels 0) and
// block partials of Σ (out − target)².
__global__ void mse_kernel(const float* __restrict__ out, const float* __restrict__ target, int nt, int co, float scale,
                           __nv_bfloat16* dy, int64_t npix, double* partials) {
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npix * co; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = i / co;
        const int c = (int)(i % co);
        float g = 0.0f;
        if (c < nt) {
            const float d = out[i] - target[p * nt + c];
            acc += (double)d * d;
            g = 2.0f * scale * d;
        }
        dy[i] = __float2bfloat16(g);
    }
    __shared__ double red[256 / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
        partials[(size_t)blockIdx.x * RED_SLOTS] = t;
    }
}

// Adam on FP32 master parameters with a BF16 copy (Kingma & Ba, 2015):
// m = β1 m + (1−β1) g; v = β2 v + (1−β2) g²; w −= lr·m̂/(√v̂ + ε).
__global__ void adam_kernel(float* w, float* m, float* v, const float* g, __nv_bfloat16* wb, int64_t n, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        if (wb) wb[i] = __float2bfloat16(wi);
    }
}

__global__ void f32_to_bf16_kernel(const float* x, __nv_bfloat16* y, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = __float2bfloat16(x[i]);
}

// Dynamic shared memory above 48 KB needs the kernel attribute (a host-side setting, made on
// every call so that it survives a context reset); the resident blocks per SM that the
// attributes give are queried once per kernel and device.
struct LaunchCache {
    const void* fn;
    int dev, per_sm;
};
std::mutex g_launch_mutex;
LaunchCache g_launch_cache[128];
int g_launch_entries = 0;

template <class... KArgs>
cudaError_t prepare_kernel(void (*fn)(KArgs...), int threads, int smem, int& per_sm) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(g_launch_mutex);
    for (int i = 0; i < g_launch_entries; ++i)
        if (g_launch_cache[i].fn == (const void*)fn && g_launch_cache[i].dev == dev) {
            per_sm = g_launch_cache[i].per_sm;
            return cudaSuccess;
        }
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
    if (e != cudaSuccess) return e;
    per_sm = std::max(per_sm, 1);
    if (g_launch_entries < 128) g_launch_cache[g_launch_entries++] = LaunchCache{(const void*)fn, dev, per_sm};
    return cudaSuccess;
}

template <int CI, int CO, int MODE>
cudaError_t conv_launch(const void* in, const void* wt, const float* bias, const void* mask, void* out, int B, int H,
                        int W, int num_sms, int* err, cudaStream_t st) {
    constexpr int smem = ConvSmem<CI, CO>::BYTES;
    auto fn = conv3x3_tc_kernel<CI, CO, MODE>;
    int per_sm = 1;
    cudaError_t e = prepare_kernel(fn, FWD_THREADS, smem, per_sm);
    if (e != cudaSuccess) return e;
    const int64_t ntile = (int64_t)B * ((H + FROWS - 1) / FROWS) * ((W + SEG - 1) / SEG);
    if (ntile >= ((int64_t)1 << 31)) return cudaErrorInvalidValue;
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>(ntile, (int64_t)num_sms * std::max(per_sm, 1)));
    count_launch();
    fn<<<(unsigned)blocks, FWD_THREADS, smem, st>>>(static_cast<const __nv_bfloat16*>(in),
                                                   static_cast<const __nv_bfloat16*>(wt), bias,
                                                   static_cast<const __nv_bfloat16*>(mask), out, B, H, W, err);
    return cudaGetLastError();
}

template <int CI, int CO>
cudaError_t conv_mode(int mode, const void* in, const void* wt, const float* bias, const void* mask, void* out, int B,
                      int H, int W, int num_sms, int* err, cudaStream_t st) {
    if (mode == 0) return conv_launch<CI, CO, 0>(in, wt, bias, mask, out, B, H, W, num_sms, err, st);
    if (mode == 1) return conv_launch<CI, CO, 1>(in, wt, bias, mask, out, B, H, W, num_sms, err, st);
    return conv_launch<CI, CO, 2>(in, wt, bias, mask, out, B, H, W, num_sms, err, st);
}

template <int CI, int CO>
cudaError_t wgrad_launch(const void* x, const void* dy, float* dw, float* db, int B, int H, int W, int num_sms, int* err,
                         cudaStream_t st) {
    using S = WgradSmem<CI, CO>;
    int per_sm = 1;
    cudaError_t e = prepare_kernel(conv3x3_wgrad_tc_kernel<CI, CO>, WG_THREADS, S::BYTES, per_sm);
    if (e != cudaSuccess) return e;
    const int64_t ntile = (int64_t)B * ((H + FROWS - 1) / FROWS) * ((W + SEG - 1) / SEG);
    if (ntile >= ((int64_t)1 << 31)) return cudaErrorInvalidValue;
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>(ntile, (int64_t)num_sms * std::max(per_sm, 1)));
    count_launch();
    conv3x3_wgrad_tc_kernel<CI, CO><<<(unsigned)blocks, WG_THREADS, S::BYTES, st>>>(
        static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(dy), dw, B, H, W, err);
    e = cudaGetLastError();
    if (e != cudaSuccess || !db) return e;
    const int64_t npix = (int64_t)B * H * W;
    count_launch();
    bias_grad_kernel<CO><<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((npix * CO + 255) / 256, num_sms * 8)), 256, 0,
                          st>>>(static_cast<const __nv_bfloat16*>(dy), db, npix);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_conv3x3(int ci, int co, int mode, const void* in, const void* wt, const float* bias,
                           const void* mask, void* out, int B, int H, int W, int num_sms, int* err, cudaStream_t st) {
    if (ci == 16 && co == 16) return conv_mode<16, 16>(mode, in, wt, bias, mask, out, B, H, W, num_sms, err, st);
    if (ci == 16 && co == 32) return conv_mode<16, 32>(mode, in, wt, bias, mask, out, B, H, W, num_sms, err, st);
    if (ci == 32 && co == 16) return conv_mode<32, 16>(mode, in, wt, bias, mask, out, B, H, W, num_sms, err, st);
    if (ci == 32 && co == 32) return conv_mode<32, 32>(mode, in, wt, bias, mask, out, B, H, W, num_sms, err, st);
    return cudaErrorInvalidValue;
}

cudaError_t launch_conv3x3_wgrad(int ci, int co, const void* x, const void* dy, float* dw, float* db, int B, int H, int W,
                                 int num_sms, int* err, cudaStream_t st) {
    if (ci == 16 && co == 16) return wgrad_launch<16, 16>(x, dy, dw, db, B, H, W, num_sms, err, st);
    if (ci == 16 && co == 32) return wgrad_launch<16, 32>(x, dy, dw, db, B, H, W, num_sms, err, st);
    if (ci == 32 && co == 16) return wgrad_launch<32, 16>(x, dy, dw, db, B, H, W, num_sms, err, st);
    if (ci == 32 && co == 32) return wgrad_launch<32, 32>(x, dy, dw, db, B, H, W, num_sms, err, st);
    return cudaErrorInvalidValue;
}

cudaError_t launch_flip_weights(const void* w, void* wT, int ci, int co, cudaStream_t st) {
    count_launch();
    flip_weights_kernel<<<64, 256, 0, st>>>(static_cast<const __nv_bfloat16*>(w), static_cast<__nv_bfloat16*>(wT), ci, co);
    return cudaGetLastError();
}

cudaError_t launch_mse(const float* out, const float* target, int nt, int co, float scale, void* dy, int64_t npix,
                       double* partials, int blocks, cudaStream_t st) {
    count_launch();
    mse_kernel<<<blocks, 256, 0, st>>>(out, target, nt, co, scale, static_cast<__nv_bfloat16*>(dy), npix, partials);
    return cudaGetLastError();
}

cudaError_t launch_adam(float* w, float* m, float* v, const float* g, void* wb, int64_t n, float lr, float b1, float b2,
                        float eps, int64_t step, cudaStream_t st) {
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    count_launch();
    adam_kernel<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 1184)), 256, 0, st>>>(
        w, m, v, g, static_cast<__nv_bfloat16*>(wb), n, lr, b1, b2, eps, c1, c2);
    return cudaGetLastError();
}

cudaError_t launch_f32_to_bf16(const float* x, void* y, int64_t n, cudaStream_t st) {
    count_launch();
    f32_to_bf16_kernel<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 1184)), 256, 0, st>>>(
        x, static_cast<__nv_bfloat16*>(y), n);
    return cudaGetLastError();
}

}  // namespace femb
