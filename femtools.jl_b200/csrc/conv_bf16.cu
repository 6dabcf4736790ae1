// conv_bf16.cu — BF16 tensor-core 3×3 convolutions (FP32 accumulation) for the learned
// warm-start network, and its training kernels (loss, Adam). No reference counterpart:
// FEMTools.jl has no learned component; this is the network that predicts the next
// time step's v/P from the solver's own converged history.
//
// Layout: activations NHWC BF16 with C ∈ {16, 32} channels (unused channels zero);
// weights [co][9·ci + 8] BF16 (k = tap·ci + c, tap = 3·ky + kx; 8 padding entries per
// row keep the B-fragment loads bank-conflict-free).
//
// The convolution is an implicit GEMM on mma.sync.m16n8k16 (BF16 in, FP32 accumulate):
// a 128-thread block owns an 8 × 16 output tile; the input tile with its one-pixel
// halo (zero outside the grid) and the whole weight matrix are staged in shared
// memory, each warp owns two output rows (two 16-pixel M tiles) and all output
// channels, and the reduction runs over the 9 taps × ci. The data gradient is the
// same kernel on the flipped, transposed weights with the ReLU mask of the layer
// below applied in the epilogue; the weight gradient contracts the input patches
// with the output gradient over the pixels (per block, then one atomic add per
// weight and block).
#include <cuda_bf16.h>
#include <algorithm>
#include "kernels.cuh"

namespace femb {
namespace {

constexpr int CT_X = 16, CT_Y = 8, CONV_THREADS = 128;
constexpr int HALO_X = CT_X + 2, HALO_Y = CT_Y + 2;

template <int C> constexpr int kpad() { return 9 * C + 8; }

FEMB_D void mma16816(float c[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

FEMB_D uint32_t lds32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }
FEMB_D uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// MODE 0: out = ReLU(conv + bias), BF16.  MODE 1: out = conv + bias, FP32.
// MODE 2: out = conv where mask > 0 else 0, BF16 (data gradient through a ReLU; no bias).
template <int CI, int CO, int MODE>
__global__ void __launch_bounds__(CONV_THREADS) conv3x3_kernel(const __nv_bfloat16* __restrict__ in,
                                                             const __nv_bfloat16* __restrict__ wt,
                                                             const float* __restrict__ bias,
                                                             const __nv_bfloat16* __restrict__ mask, void* out, int H,
                                                             int W) {
    constexpr int K = 9 * CI, KP = kpad<CI>(), PS = CI + 8;
    __shared__ __align__(16) __nv_bfloat16 s_in[HALO_Y * HALO_X * PS];
    __shared__ __align__(16) __nv_bfloat16 s_w[CO * KP];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gid = lane >> 2, tig = lane & 3;
    const int x0 = blockIdx.x * CT_X, y0 = blockIdx.y * CT_Y, b = blockIdx.z;
    {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(wt);
        uint32_t* dst = reinterpret_cast<uint32_t*>(s_w);
        for (int i = tid; i < CO * KP / 2; i += CONV_THREADS) dst[i] = src[i];
    }
    {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(in);
        uint32_t* dst = reinterpret_cast<uint32_t*>(s_in);
        for (int i = tid; i < HALO_Y * HALO_X * (CI / 2); i += CONV_THREADS) {
            const int pix = i / (CI / 2), cp = i % (CI / 2);
            const int gy = y0 - 1 + pix / HALO_X, gx = x0 - 1 + pix % HALO_X;
            uint32_t v = 0;
            if (gy >= 0 && gy < H && gx >= 0 && gx < W) v = src[(((int64_t)b * H + gy) * W + gx) * (CI / 2) + cp];
            dst[pix * (PS / 2) + cp] = v;
        }
    }
    __syncthreads();
    float acc[2][CO / 8][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < CO / 8; ++nt)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[mt][nt][r] = 0.0f;
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
        const int ky = tap / 3, kx = tap % 3;
#pragma unroll
        for (int c0 = 0; c0 < CI; c0 += 16) {
            uint32_t a[2][4];
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                const int row = 2 * warp + mt;
                const __nv_bfloat16* lo = s_in + ((row + ky) * HALO_X + gid + kx) * PS + c0 + tig * 2;
                const __nv_bfloat16* hi = lo + 8 * PS;
                a[mt][0] = lds32(lo);
                a[mt][1] = lds32(hi);
                a[mt][2] = lds32(lo + 8);
                a[mt][3] = lds32(hi + 8);
            }
#pragma unroll
            for (int nt = 0; nt < CO / 8; ++nt) {
                const __nv_bfloat16* wp = s_w + (nt * 8 + gid) * KP + tap * CI + c0 + tig * 2;
                const uint32_t b0 = lds32(wp), b1 = lds32(wp + 8);
                mma16816(acc[0][nt], a[0], b0, b1);
                mma16816(acc[1][nt], a[1], b0, b1);
            }
        }
    }
    static_assert(K % 16 == 0, "9·ci must be a multiple of 16");
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        const int gy = y0 + 2 * warp + mt;
        if (gy >= H) continue;
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int gx = x0 + gid + 8 * half;
            if (gx >= W) continue;
            const int64_t pix = ((int64_t)b * H + gy) * W + gx;
#pragma unroll
            for (int nt = 0; nt < CO / 8; ++nt) {
                const int co = nt * 8 + tig * 2;
                float v0 = acc[mt][nt][2 * half], v1 = acc[mt][nt][2 * half + 1];
                if constexpr (MODE == 0 || MODE == 1) { v0 += bias[co]; v1 += bias[co + 1]; }
                if constexpr (MODE == 0) { v0 = fmaxf(v0, 0.0f); v1 = fmaxf(v1, 0.0f); }
                if constexpr (MODE == 2) {
                    const uint32_t m = *reinterpret_cast<const uint32_t*>(mask + pix * CO + co);
                    if (!(__bfloat162float(__ushort_as_bfloat16((unsigned short)(m & 0xffffu))) > 0.0f)) v0 = 0.0f;
                    if (!(__bfloat162float(__ushort_as_bfloat16((unsigned short)(m >> 16))) > 0.0f)) v1 = 0.0f;
                }
                if constexpr (MODE == 1) {
                    *reinterpret_cast<float2*>(static_cast<float*>(out) + pix * CO + co) = make_float2(v0, v1);
                } else {
                    *reinterpret_cast<uint32_t*>(static_cast<__nv_bfloat16*>(out) + pix * CO + co) =
                        pack2(__float2bfloat16(v0), __float2bfloat16(v1));
                }
            }
        }
    }
}

// dW[co][tap·ci + c] += Σ_p X[p + (ky−1, kx−1)][c]·dY[p][co] over the grid (batch
// included), on mma.sync with the pixels as the reduction dimension: tiles are
// staged channel-major (X_T[c][iy][ix], dY_T[co][py][px]) so that consecutive pixels
// are adjacent; the block accumulates in registers over all the tiles it visits and
// adds its partial sums once.
template <int CI, int CO>
__global__ void __launch_bounds__(CONV_THREADS) conv3x3_wgrad_kernel(const __nv_bfloat16* __restrict__ x,
                                                                   const __nv_bfloat16* __restrict__ dy, float* dw,
                                                                   int B, int H, int W) {
    constexpr int XS = 20, YS = 20;   // row strides of the staged tiles (halo width 18, tile width 16)
    constexpr int MT = 9 * CI / 16, NT = CO / 8;
    constexpr int MT_W = (MT + 3) / 4;   // M tiles per warp
    constexpr int KP = kpad<CI>();
    __shared__ __align__(16) __nv_bfloat16 s_x[CI * HALO_Y * XS];
    __shared__ __align__(16) __nv_bfloat16 s_dy[CO * CT_Y * YS];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gid = lane >> 2, tig = lane & 3;
    float acc[MT_W][NT][4];
#pragma unroll
    for (int i = 0; i < MT_W; ++i)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[i][nt][r] = 0.0f;
    const int tx_n = (W + CT_X - 1) / CT_X, ty_n = (H + CT_Y - 1) / CT_Y;
    const int64_t ntile = (int64_t)B * tx_n * ty_n;
    for (int64_t t = blockIdx.x; t < ntile; t += gridDim.x) {
        const int b = (int)(t / ((int64_t)tx_n * ty_n));
        const int rem = (int)(t % ((int64_t)tx_n * ty_n));
        const int x0 = (rem % tx_n) * CT_X, y0 = (rem / tx_n) * CT_Y;
        __syncthreads();
        for (int i = tid; i < HALO_Y * HALO_X * CI; i += CONV_THREADS) {
            const int pix = i / CI, c = i % CI;
            const int iy = pix / HALO_X, ix = pix % HALO_X;
            const int gy = y0 - 1 + iy, gx = x0 - 1 + ix;
            __nv_bfloat16 v = __float2bfloat16(0.0f);
            if (gy >= 0 && gy < H && gx >= 0 && gx < W) v = x[(((int64_t)b * H + gy) * W + gx) * CI + c];
            s_x[(c * HALO_Y + iy) * XS + ix] = v;
        }
        for (int i = tid; i < CT_Y * CT_X * CO; i += CONV_THREADS) {
            const int pix = i / CO, c = i % CO;
            const int py = pix / CT_X, px = pix % CT_X;
            const int gy = y0 + py, gx = x0 + px;
            __nv_bfloat16 v = __float2bfloat16(0.0f);
            if (gy < H && gx < W) v = dy[(((int64_t)b * H + gy) * W + gx) * CO + c];
            s_dy[(c * CT_Y + py) * YS + px] = v;
        }
        __syncthreads();
#pragma unroll 1
        for (int py = 0; py < CT_Y; ++py) {
            uint32_t bf[NT][2];
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) {
                const __nv_bfloat16* p = s_dy + ((nt * 8 + gid) * CT_Y + py) * YS + tig * 2;
                bf[nt][0] = lds32(p);
                bf[nt][1] = lds32(p + 8);
            }
#pragma unroll
            for (int i = 0; i < MT_W; ++i) {
                const int mt = warp + 4 * i;
                if (mt >= MT) break;
                const int tap = (mt * 16) / CI, c0 = (mt * 16) % CI;
                const int ky = tap / 3, kx = tap % 3;
                uint32_t a[4];
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    const int c = c0 + gid + ((r & 1) ? 8 : 0);
                    const int px = tig * 2 + ((r & 2) ? 8 : 0);
                    const __nv_bfloat16* p = s_x + (c * HALO_Y + py + ky) * XS + px + kx;
                    a[r] = pack2(p[0], p[1]);
                }
#pragma unroll
                for (int nt = 0; nt < NT; ++nt) mma16816(acc[i][nt], a, bf[nt][0], bf[nt][1]);
            }
        }
    }
    // D rows: k = mt·16 + gid (+8); columns: co = nt·8 + tig·2 (+1)
#pragma unroll
    for (int i = 0; i < MT_W; ++i) {
        const int mt = warp + 4 * i;
        if (mt >= MT) break;
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
            const int k0 = mt * 16 + gid, co = nt * 8 + tig * 2;
            atomicAdd(dw + (int64_t)co * KP + k0, acc[i][nt][0]);
            atomicAdd(dw + (int64_t)(co + 1) * KP + k0, acc[i][nt][1]);
            atomicAdd(dw + (int64_t)co * KP + k0 + 8, acc[i][nt][2]);
            atomicAdd(dw + (int64_t)(co + 1) * KP + k0 + 8, acc[i][nt][3]);
        }
    }
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

template <int CI, int CO, int MODE>
cudaError_t conv_launch(const void* in, const void* wt, const float* bias, const void* mask, void* out, int B, int H,
                        int W, cudaStream_t st) {
    dim3 grid((W + CT_X - 1) / CT_X, (H + CT_Y - 1) / CT_Y, B);
    count_launch();
    conv3x3_kernel<CI, CO, MODE><<<grid, CONV_THREADS, 0, st>>>(static_cast<const __nv_bfloat16*>(in),
                                                                static_cast<const __nv_bfloat16*>(wt), bias,
                                                                static_cast<const __nv_bfloat16*>(mask), out, H, W);
    return cudaGetLastError();
}

template <int CI, int CO>
cudaError_t conv_mode(int mode, const void* in, const void* wt, const float* bias, const void* mask, void* out, int B,
                      int H, int W, cudaStream_t st) {
    if (mode == 0) return conv_launch<CI, CO, 0>(in, wt, bias, mask, out, B, H, W, st);
    if (mode == 1) return conv_launch<CI, CO, 1>(in, wt, bias, mask, out, B, H, W, st);
    return conv_launch<CI, CO, 2>(in, wt, bias, mask, out, B, H, W, st);
}

template <int CI, int CO>
cudaError_t wgrad_launch(const void* x, const void* dy, float* dw, float* db, int B, int H, int W, int num_sms,
                         cudaStream_t st) {
    const int64_t ntile = (int64_t)B * ((W + CT_X - 1) / CT_X) * ((H + CT_Y - 1) / CT_Y);
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>(ntile, (int64_t)num_sms * 8));
    count_launch();
    conv3x3_wgrad_kernel<CI, CO><<<(unsigned)blocks, CONV_THREADS, 0, st>>>(static_cast<const __nv_bfloat16*>(x),
                                                                           static_cast<const __nv_bfloat16*>(dy), dw, B,
                                                                           H, W);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || !db) return e;
    const int64_t npix = (int64_t)B * H * W;
    count_launch();
    bias_grad_kernel<CO><<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((npix * CO + 255) / 256, num_sms * 8)), 256, 0,
                          st>>>(static_cast<const __nv_bfloat16*>(dy), db, npix);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_conv3x3(int ci, int co, int mode, const void* in, const void* wt, const float* bias,
                           const void* mask, void* out, int B, int H, int W, cudaStream_t st) {
    if (ci == 16 && co == 16) return conv_mode<16, 16>(mode, in, wt, bias, mask, out, B, H, W, st);
    if (ci == 16 && co == 32) return conv_mode<16, 32>(mode, in, wt, bias, mask, out, B, H, W, st);
    if (ci == 32 && co == 16) return conv_mode<32, 16>(mode, in, wt, bias, mask, out, B, H, W, st);
    if (ci == 32 && co == 32) return conv_mode<32, 32>(mode, in, wt, bias, mask, out, B, H, W, st);
    return cudaErrorInvalidValue;
}

cudaError_t launch_conv3x3_wgrad(int ci, int co, const void* x, const void* dy, float* dw, float* db, int B, int H, int W,
                                 int num_sms, cudaStream_t st) {
    if (ci == 16 && co == 16) return wgrad_launch<16, 16>(x, dy, dw, db, B, H, W, num_sms, st);
    if (ci == 16 && co == 32) return wgrad_launch<16, 32>(x, dy, dw, db, B, H, W, num_sms, st);
    if (ci == 32 && co == 16) return wgrad_launch<32, 16>(x, dy, dw, db, B, H, W, num_sms, st);
    if (ci == 32 && co == 32) return wgrad_launch<32, 32>(x, dy, dw, db, B, H, W, num_sms, st);
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
