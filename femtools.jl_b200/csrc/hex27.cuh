// hex27.cuh — sum-factorised Hex27/P1-disc element machinery.
//
// Mapping: a warp processes three elements at a time; lanes 0..26 form three
// groups of nine ("line threads"), lanes 27..31 idle. Thread m = m1 + 3·m2 of a
// group owns one tensor line of the 3×3×3 node/quadrature grid, so every 1-D
// contraction of the tensor-product basis runs in registers and only the
// re-orientation between directions goes through shared memory (warp-local,
// ordered by __syncwarp). This replaces the reference's thread-per-element
// loops over 27 quadrature points × 27 nodes (momentum_residuals.jl:231-256)
// with ~1/3 of the floating-point work.
//
// Orientation of the owned line per stage:
//   gather / scatter : x-line (·, m1, m2)  — contiguous node runs in memory
//   after stage Y    : y-line (m1, ·, m2)
//   quadrature stage : z-line (m1, m2, ·)  — quadrature points q = m1 + 3m2 + 9qz
#pragma once
#include <type_traits>
#include "common.cuh"

namespace femb {

constexpr int H27_ELEM_SMEM = 540;   // scalars of stage scratch per element

FEMB_D int tidx(int i, int j, int k) { return i + 3 * j + 9 * k; }

// Ordered scatter of a warp's three elements (lane s·9 + m owns the x-line (·, m1, m2) of
// element s; lanes 27..31 idle): where element s + 1's ξ = −1 node of the line is element
// s's ξ = +1 node (consecutive elements along ξ), lane (s, m) adds that lane's node-0
// values into its node-2 values, so the group adds to such a node once. Returns whether
// this lane's node 0 went to the previous element's lane. Every lane of the warp calls it.
template <class T>
FEMB_D bool fold_next_element(const int node[3], bool act, int s, T (&R)[3][3]) {
    const int lane = threadIdx.x & 31;
    const int n0n = __shfl_down_sync(0xffffffffu, node[0], 9);
    const int actn = __shfl_down_sync(0xffffffffu, (int)act, 9);
    const bool fold = s < 2 && act && actn && n0n == node[2];
    const bool folded = __shfl_up_sync(0xffffffffu, (int)fold, 9) && lane >= 9;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const T v0n = __shfl_down_sync(0xffffffffu, R[c][0], 9);
        if (fold) R[c][2] += v0n;
    }
    return folded;
}

// Layouts of the stage buffers. A buffer holds blocks of one 3×3×3 grid; it is written
// along one line orientation and read along another. Buffers of the first kind (the
// gradient's x-stage, the transpose's y-stage) use l1 in blocks of K1 words, those of
// the second kind (the gradient's y-stage, the transpose's z-stage) l2 in blocks of K2.
// H27Compact is i + 3j + 9k for both. H27Fp64Banked is for FP64 element slots 539
// words apart with the idle lanes on m = 2 of a fourth slot: 3i + 4j + 9k and
// 3i + 2j + 9k, found by exhaustive search over the two access orientations of each
// buffer kind (FP64 shared accesses go as two half-warps over 16 eight-byte banks);
// a gradient and a transpose take 480 wavefronts instead of the compact layout's 807
// (384 is the floor).
struct H27Compact {
    static constexpr int K1 = 27, K2 = 27;
    static constexpr int SLOT = H27_ELEM_SMEM, IDLE_M = 0;
    static FEMB_D int l1(int i, int j, int k) { return i + 3 * j + 9 * k; }
    static FEMB_D int l2(int i, int j, int k) { return i + 3 * j + 9 * k; }
};
struct H27Fp64Banked {
    static constexpr int K1 = 33, K2 = 29;
    static constexpr int SLOT = 539, IDLE_M = 2;
    static FEMB_D int l1(int i, int j, int k) { return 3 * i + 4 * j + 9 * k; }
    static FEMB_D int l2(int i, int j, int k) { return 3 * i + 2 * j + 9 * k; }
};
// words of stage scratch a layout needs per element slot
template <class LY> constexpr int h27_stage_words() {
    return (6 * LY::K1 + 9 * LY::K2) > (10 * LY::K2 + 7 * LY::K1) ? (6 * LY::K1 + 9 * LY::K2)
                                                                   : (10 * LY::K2 + 7 * LY::K1);
}
static_assert(h27_stage_words<H27Compact>() <= H27_ELEM_SMEM, "compact stage layout");
static_assert(h27_stage_words<H27Fp64Banked>() <= H27Fp64Banked::SLOT, "banked stage layout");
// the layout of the four-slot kernels (three elements and the idle lanes per warp)
template <class T> using H27Layout = std::conditional_t<sizeof(T) == 8, H27Fp64Banked, H27Compact>;

// 1-D basis tables read straight from constant memory: every index in the stage
// code is a compile-time constant, so they become constant-bank operands and take
// no registers.
template <class T>
struct Tab1D {
    struct Row {
        int q;
        FEMB_D T operator[](int i) const { return (T)c_tab.B[q][i]; }
    };
    struct RowD {
        int q;
        FEMB_D T operator[](int i) const { return (T)c_tab.Dd[q][i]; }
    };
    struct TabB {
        FEMB_D Row operator[](int q) const { return Row{q}; }
    } B;
    struct TabD {
        FEMB_D RowD operator[](int q) const { return RowD{q}; }
    } Dd;
    FEMB_D void load() {}
};

// Reference gradients of the three velocity components at the three quadrature
// points of the owned z-line. v[c][i]: node values on the owned x-line.
// Output g[c][d][qz], d = ξ, η, ζ.
template <class T, class LY = H27Compact>
FEMB_D void h27_gradient(const Tab1D<T>& t, const T v[3][3], T* E, int m1, int m2, T g[3][3][3], bool wr = true) {
    // stage X: contract x (thread owns x-line (·, m1, m2))
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            T x0 = t.B[q][0] * v[c][0] + t.B[q][1] * v[c][1] + t.B[q][2] * v[c][2];
            T x1 = t.Dd[q][0] * v[c][0] + t.Dd[q][1] * v[c][1] + t.Dd[q][2] * v[c][2];
            if (wr) {
                E[(c * 2 + 0) * LY::K1 + LY::l1(q, m1, m2)] = x0;
                E[(c * 2 + 1) * LY::K1 + LY::l1(q, m1, m2)] = x1;
            }
        }
    __syncwarp();
    // stage Y: thread owns y-line (qx = m1, ·, k = m2)
    T* E1 = E + 6 * LY::K1;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        T X0[3], X1[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            X0[j] = E[(c * 2 + 0) * LY::K1 + LY::l1(m1, j, m2)];
            X1[j] = E[(c * 2 + 1) * LY::K1 + LY::l1(m1, j, m2)];
        }
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const T y0 = t.B[q][0] * X1[0] + t.B[q][1] * X1[1] + t.B[q][2] * X1[2];
            const T y1 = t.Dd[q][0] * X0[0] + t.Dd[q][1] * X0[1] + t.Dd[q][2] * X0[2];
            const T y2 = t.B[q][0] * X0[0] + t.B[q][1] * X0[1] + t.B[q][2] * X0[2];
            if (wr) {
                E1[(c * 3 + 0) * LY::K2 + LY::l2(m1, q, m2)] = y0;
                E1[(c * 3 + 1) * LY::K2 + LY::l2(m1, q, m2)] = y1;
                E1[(c * 3 + 2) * LY::K2 + LY::l2(m1, q, m2)] = y2;
            }
        }
    }
    __syncwarp();
    // stage Z: thread owns z-line (qx = m1, qy = m2, ·)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        T A[3], Bv[3], Cv[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            A[k] = E1[(c * 3 + 0) * LY::K2 + LY::l2(m1, m2, k)];
            Bv[k] = E1[(c * 3 + 1) * LY::K2 + LY::l2(m1, m2, k)];
            Cv[k] = E1[(c * 3 + 2) * LY::K2 + LY::l2(m1, m2, k)];
        }
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            g[c][0][q] = t.B[q][0] * A[0] + t.B[q][1] * A[1] + t.B[q][2] * A[2];
            g[c][1][q] = t.B[q][0] * Bv[0] + t.B[q][1] * Bv[1] + t.B[q][2] * Bv[2];
            g[c][2][q] = t.Dd[q][0] * Cv[0] + t.Dd[q][1] * Cv[1] + t.Dd[q][2] * Cv[2];
        }
    }
    __syncwarp();
}

// Transposed contraction: nodal residual R[c][ix] on the owned x-line from the
// reference-frame fluxes F[c][d][qz] and the body-force density beta[qz]
// (R_c(a) = Σ_q Σ_d ∂_d N_a(q) F_cd(q) − g_c Σ_q N_a(q) β(q)).
template <class T, bool BODY = true, class LY = H27Compact>
FEMB_D void h27_transpose(const Tab1D<T>& t, const T F[3][3][3], const T beta[3], const T gvec[3], T* E,
                          int m1, int m2, T R[3][3], bool wr = true) {
    // Z^T: thread owns z-line (qx = m1, qy = m2)
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int iz = 0; iz < 3; ++iz) {
            const T z0 = t.B[0][iz] * F[c][0][0] + t.B[1][iz] * F[c][0][1] + t.B[2][iz] * F[c][0][2];
            const T z1 = t.B[0][iz] * F[c][1][0] + t.B[1][iz] * F[c][1][1] + t.B[2][iz] * F[c][1][2];
            const T z2 = t.Dd[0][iz] * F[c][2][0] + t.Dd[1][iz] * F[c][2][1] + t.Dd[2][iz] * F[c][2][2];
            if (wr) {
                E[(c * 3 + 0) * LY::K2 + LY::l2(m1, m2, iz)] = z0;
                E[(c * 3 + 1) * LY::K2 + LY::l2(m1, m2, iz)] = z1;
                E[(c * 3 + 2) * LY::K2 + LY::l2(m1, m2, iz)] = z2;
            }
        }
    if constexpr (BODY) {
#pragma unroll
        for (int iz = 0; iz < 3; ++iz) {
            const T zb = t.B[0][iz] * beta[0] + t.B[1][iz] * beta[1] + t.B[2][iz] * beta[2];
            if (wr) E[9 * LY::K2 + LY::l2(m1, m2, iz)] = zb;
        }
    }
    __syncwarp();
    // Y^T: thread owns y-line (qx = m1, ·, iz = m2)
    T* E1 = E + 10 * LY::K2;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        T TA[3], TB[3], TC[3];
#pragma unroll
        for (int qy = 0; qy < 3; ++qy) {
            TA[qy] = E[(c * 3 + 0) * LY::K2 + LY::l2(m1, qy, m2)];
            TB[qy] = E[(c * 3 + 1) * LY::K2 + LY::l2(m1, qy, m2)];
            TC[qy] = E[(c * 3 + 2) * LY::K2 + LY::l2(m1, qy, m2)];
        }
#pragma unroll
        for (int iy = 0; iy < 3; ++iy) {
            const T u0 = t.B[0][iy] * TA[0] + t.B[1][iy] * TA[1] + t.B[2][iy] * TA[2];
            const T u1 = (t.Dd[0][iy] * TB[0] + t.Dd[1][iy] * TB[1] + t.Dd[2][iy] * TB[2]) +
                         (t.B[0][iy] * TC[0] + t.B[1][iy] * TC[1] + t.B[2][iy] * TC[2]);
            if (wr) {
                E1[(c * 2 + 0) * LY::K1 + LY::l1(m1, iy, m2)] = u0;
                E1[(c * 2 + 1) * LY::K1 + LY::l1(m1, iy, m2)] = u1;
            }
        }
    }
    if constexpr (BODY) {
        T TD[3];
#pragma unroll
        for (int qy = 0; qy < 3; ++qy) TD[qy] = E[9 * LY::K2 + LY::l2(m1, qy, m2)];
#pragma unroll
        for (int iy = 0; iy < 3; ++iy) {
            const T ub = t.B[0][iy] * TD[0] + t.B[1][iy] * TD[1] + t.B[2][iy] * TD[2];
            if (wr) E1[6 * LY::K1 + LY::l1(m1, iy, m2)] = ub;
        }
    }
    __syncwarp();
    // X^T: thread owns x-line (·, iy = m1, iz = m2)
    T body[3] = {T(0), T(0), T(0)};
    if constexpr (BODY) {
        T UD[3];
#pragma unroll
        for (int qx = 0; qx < 3; ++qx) UD[qx] = E1[6 * LY::K1 + LY::l1(qx, m1, m2)];
#pragma unroll
        for (int ix = 0; ix < 3; ++ix) body[ix] = t.B[0][ix] * UD[0] + t.B[1][ix] * UD[1] + t.B[2][ix] * UD[2];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        T UA[3], UB[3];
#pragma unroll
        for (int qx = 0; qx < 3; ++qx) {
            UA[qx] = E1[(c * 2 + 0) * LY::K1 + LY::l1(qx, m1, m2)];
            UB[qx] = E1[(c * 2 + 1) * LY::K1 + LY::l1(qx, m1, m2)];
        }
#pragma unroll
        for (int ix = 0; ix < 3; ++ix)
            R[c][ix] = (t.Dd[0][ix] * UA[0] + t.Dd[1][ix] * UA[1] + t.Dd[2][ix] * UA[2]) +
                       (t.B[0][ix] * UB[0] + t.B[1][ix] * UB[1] + t.B[2][ix] * UB[2]) - (BODY ? gvec[c] * body[ix] : T(0));
    }
    __syncwarp();
}

// Per-element material at one quadrature point, interpolated with the velocity
// shape functions over the element's node phases (interp2ip_phase, utils.jl:37).
template <class T>
struct QpMat {
    T eta, invG, alpha, rho0, beta;
    T cphi, sphi, spsi, C, ereg, Kb;
};

template <class T>
FEMB_D void interp_material(QpMat<T>& m, bool uniform, int p0, const int* PH, int qx, int qy, int qz,
                            bool plastic, const T* eta_override) {
    if (uniform) {
        const T s = (T)c_tab.sumN3[tidx(qx, qy, qz)];
        m.eta = (T)c_mat.eta[p0] * s;
        m.invG = (T)c_mat.invG[p0] * s;
        m.alpha = (T)c_mat.alpha[p0] * s;
        m.rho0 = (T)c_mat.rho0[p0] * s;
        m.beta = (T)c_mat.beta[p0] * s;
        if (plastic) {
            m.cphi = (T)c_mat.cos_phi[p0] * s; m.sphi = (T)c_mat.sin_phi[p0] * s; m.spsi = (T)c_mat.sin_psi[p0] * s;
            m.C = (T)c_mat.C[p0] * s; m.ereg = (T)c_mat.eta_reg[p0] * s; m.Kb = (T)c_mat.Kb[p0] * s;
        }
    } else {
        m.eta = m.invG = m.alpha = m.rho0 = m.beta = T(0);
        m.cphi = m.sphi = m.spsi = m.C = m.ereg = m.Kb = T(0);
        for (int k = 0; k < 3; ++k)
            for (int j = 0; j < 3; ++j)
                for (int i = 0; i < 3; ++i) {
                    const T N = (T)c_tab.B[qx][i] * (T)c_tab.B[qy][j] * (T)c_tab.B[qz][k];
                    const int p = PH[tidx(i, j, k)];
                    m.eta += N * (T)c_mat.eta[p];
                    m.invG += N * (T)c_mat.invG[p];
                    m.alpha += N * (T)c_mat.alpha[p];
                    m.rho0 += N * (T)c_mat.rho0[p];
                    m.beta += N * (T)c_mat.beta[p];
                    if (plastic) {
                        m.cphi += N * (T)c_mat.cos_phi[p]; m.sphi += N * (T)c_mat.sin_phi[p];
                        m.spsi += N * (T)c_mat.sin_psi[p]; m.C += N * (T)c_mat.C[p];
                        m.ereg += N * (T)c_mat.eta_reg[p]; m.Kb += N * (T)c_mat.Kb[p];
                    }
                }
    }
    if (eta_override) m.eta = *eta_override;
}


}  // namespace femb
