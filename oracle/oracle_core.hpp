// oracle_core.hpp — TEST INFRASTRUCTURE ONLY. CPU restatement of the FEMTools.jl
// matrix-free dynamic-relaxation hot path, used as the parity checker and as the
// timed CPU baseline. Nothing in the product library links or calls this code.
//
// Every routine below restates one reference function; the citation is the file
// and line of the Julia source inside the FEMTools.jl repository (v0.2.0).
// Arithmetic is FP64 and follows the reference's order of operations where the
// order is visible in the source. The scalar type S is templated so that a
// forward-mode dual number reproduces the ForwardDiff Jacobian diagnostics of
// momentum_residuals.jl:781 and heat_diffusion/assembly/residual.jl:39.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <limits>

namespace orc {

// ---------------------------------------------------------------------------
// Forward-mode dual number with N partials (the ForwardDiff.Dual analogue).
// ---------------------------------------------------------------------------
template <int N>
struct Dual {
    double v;
    double d[N];
    Dual() : v(0) { for (int i = 0; i < N; ++i) d[i] = 0; }
    Dual(double x) : v(x) { for (int i = 0; i < N; ++i) d[i] = 0; }
};
template <int N> inline Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) { Dual<N> r; r.v = a.v + b.v; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i]; return r; }
template <int N> inline Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) { Dual<N> r; r.v = a.v - b.v; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i]; return r; }
template <int N> inline Dual<N> operator-(const Dual<N>& a) { Dual<N> r; r.v = -a.v; for (int i = 0; i < N; ++i) r.d[i] = -a.d[i]; return r; }
template <int N> inline Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) { Dual<N> r; r.v = a.v * b.v; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i]; return r; }
template <int N> inline Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) { Dual<N> r; r.v = a.v / b.v; double ib2 = 1.0 / (b.v * b.v); for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] * b.v - a.v * b.d[i]) * ib2; return r; }
template <int N> inline Dual<N> operator+(const Dual<N>& a, double b) { Dual<N> r = a; r.v += b; return r; }
template <int N> inline Dual<N> operator+(double b, const Dual<N>& a) { Dual<N> r = a; r.v += b; return r; }
template <int N> inline Dual<N> operator-(const Dual<N>& a, double b) { Dual<N> r = a; r.v -= b; return r; }
template <int N> inline Dual<N> operator-(double b, const Dual<N>& a) { Dual<N> r; r.v = b - a.v; for (int i = 0; i < N; ++i) r.d[i] = -a.d[i]; return r; }
template <int N> inline Dual<N> operator*(const Dual<N>& a, double b) { Dual<N> r; r.v = a.v * b; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b; return r; }
template <int N> inline Dual<N> operator*(double b, const Dual<N>& a) { return a * b; }
template <int N> inline Dual<N> operator/(const Dual<N>& a, double b) { Dual<N> r; r.v = a.v / b; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] / b; return r; }
template <int N> inline Dual<N> operator/(double a, const Dual<N>& b) { Dual<N> r; r.v = a / b.v; double f = -a / (b.v * b.v); for (int i = 0; i < N; ++i) r.d[i] = f * b.d[i]; return r; }
template <int N> inline Dual<N> sqrt(const Dual<N>& a) { Dual<N> r; r.v = std::sqrt(a.v); double f = 0.5 / r.v; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * f; return r; }
template <int N> inline Dual<N>& operator+=(Dual<N>& a, const Dual<N>& b) { a = a + b; return a; }
template <int N> inline Dual<N>& operator-=(Dual<N>& a, const Dual<N>& b) { a = a - b; return a; }

inline double val(double x) { return x; }
template <int N> inline double val(const Dual<N>& x) { return x.v; }
using std::sqrt;

// ---------------------------------------------------------------------------
// Reference-element tables.
// ---------------------------------------------------------------------------
// Hex27 local node reference coordinates (src/elements/shape_functions.jl:414-442).
static const int HEX27_NODES[27][3] = {
    {-1, -1, -1}, {+1, -1, -1}, {+1, +1, -1}, {-1, +1, -1},
    {-1, -1, +1}, {+1, -1, +1}, {+1, +1, +1}, {-1, +1, +1},
    {0, -1, -1}, {+1, 0, -1}, {0, +1, -1}, {-1, 0, -1},
    {0, -1, +1}, {+1, 0, +1}, {0, +1, +1}, {-1, 0, +1},
    {-1, -1, 0}, {+1, -1, 0}, {+1, +1, 0}, {-1, +1, 0},
    {0, 0, -1}, {0, -1, 0}, {+1, 0, 0}, {0, +1, 0}, {-1, 0, 0}, {0, 0, +1}, {0, 0, 0}};
// Q9 local node reference coordinates (src/elements/shape_functions.jl:268-278).
static const int Q9_NODES[9][2] = {{-1, -1}, {+1, -1}, {+1, +1}, {-1, +1}, {0, -1}, {+1, 0}, {0, +1}, {-1, 0}, {0, 0}};

// 1-D quadratic Lagrange basis on nodes (-1, 0, +1) (shape_functions.jl:173-196).
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

struct Tables {
    int dim, nv, np, nq;
    double N[27][27];        // N[q][a]
    double dN[27][27][3];    // ∂N_a/∂ξ_j at q
    double NP[27][4];        // pressure basis at velocity quadrature points
    double w[27];            // quadrature weights
    int prow[4];             // local velocity nodes carrying the pressure DoFs (0-based)
};

// Hex27 with the 3×3×3 Gauss rule (integration_points.jl:321-337) and the P1
// pressure basis (1-ξ-η-ζ, ξ, η, ζ) of LinearElement{3,4} at those points
// (shape_functions.jl:288-298); pressure rows (27,23,24,26) (mixed_mesh.jl:415).
inline Tables hex27_tables() {
    Tables t; std::memset(&t, 0, sizeof(t));
    t.dim = 3; t.nv = 27; t.np = 4; t.nq = 27;
    const double a = std::sqrt(3.0 / 5.0);
    const double pts[3] = {-a, 0.0, +a};
    const double wts[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
    for (int q = 0; q < 27; ++q) {
        int qx = q % 3, qy = (q / 3) % 3, qz = q / 9;
        double x[3] = {pts[qx], pts[qy], pts[qz]};
        t.w[q] = wts[qx] * wts[qy] * wts[qz];
        for (int n = 0; n < 27; ++n) {
            const int* nd = HEX27_NODES[n];
            double l[3], dl[3];
            for (int d = 0; d < 3; ++d) { l[d] = line_N(x[d], nd[d]); dl[d] = line_dN(x[d], nd[d]); }
            t.N[q][n] = l[0] * l[1] * l[2];
            t.dN[q][n][0] = dl[0] * l[1] * l[2];
            t.dN[q][n][1] = l[0] * dl[1] * l[2];
            t.dN[q][n][2] = l[0] * l[1] * dl[2];
        }
        t.NP[q][0] = 1 - x[0] - x[1] - x[2];
        t.NP[q][1] = x[0]; t.NP[q][2] = x[1]; t.NP[q][3] = x[2];
    }
    t.prow[0] = 26; t.prow[1] = 22; t.prow[2] = 23; t.prow[3] = 25;
    return t;
}

// Q9 with the 3×3 Gauss rule (integration_points.jl:223-242) and the P1 basis
// (1-ξ-η, ξ, η) of LinearElement{2,3} (shape_functions.jl:231-239); pressure rows
// (9,6,7) (mixed_mesh.jl:409).
inline Tables q9_tables() {
    Tables t; std::memset(&t, 0, sizeof(t));
    t.dim = 2; t.nv = 9; t.np = 3; t.nq = 9;
    const double a = std::sqrt(3.0 / 5.0);
    const double pts[3] = {-a, 0.0, +a};
    const double wq[9] = {25.0 / 81, 40.0 / 81, 25.0 / 81, 40.0 / 81, 64.0 / 81, 40.0 / 81, 25.0 / 81, 40.0 / 81, 25.0 / 81};
    for (int q = 0; q < 9; ++q) {
        int qx = q % 3, qy = q / 3;
        double x[2] = {pts[qx], pts[qy]};
        t.w[q] = wq[q];
        for (int n = 0; n < 9; ++n) {
            const int* nd = Q9_NODES[n];
            double l[2], dl[2];
            for (int d = 0; d < 2; ++d) { l[d] = line_N(x[d], nd[d]); dl[d] = line_dN(x[d], nd[d]); }
            t.N[q][n] = l[0] * l[1];
            t.dN[q][n][0] = dl[0] * l[1];
            t.dN[q][n][1] = l[0] * dl[1];
        }
        t.NP[q][0] = 1 - x[0] - x[1];
        t.NP[q][1] = x[0]; t.NP[q][2] = x[1];
    }
    t.prow[0] = 8; t.prow[1] = 5; t.prow[2] = 6;
    return t;
}

inline const Tables& tables_for(int dim) {
    static const Tables h = hex27_tables();
    static const Tables q = q9_tables();
    return dim == 3 ? h : q;
}

// ---------------------------------------------------------------------------
// Structured meshes and geometry.
// ---------------------------------------------------------------------------
// generate_element2node(Hex27) (src/mesh/connectivity.jl:273-322); nodes on the
// refined (2nx+1)(2ny+1)(2nz+1) grid, x fastest; 1-based output.
inline void hex27_el2n(int nx, int ny, int nz, int32_t* el2n) {
    const int64_t sy = 2 * nx + 1, sz = (int64_t)(2 * nx + 1) * (2 * ny + 1);
    auto node = [&](int64_t ix, int64_t iy, int64_t iz) { return (int32_t)(iz * sz + iy * sy + ix + 1); };
    int64_t iel = 0;
    for (int ez = 0; ez < nz; ++ez)
        for (int ey = 0; ey < ny; ++ey)
            for (int ex = 0; ex < nx; ++ex, ++iel) {
                int ix = 2 * ex, iy = 2 * ey, iz = 2 * ez;
                int32_t* e = el2n + 27 * iel;
                for (int a = 0; a < 27; ++a)
                    e[a] = node(ix + 1 + HEX27_NODES[a][0], iy + 1 + HEX27_NODES[a][1], iz + 1 + HEX27_NODES[a][2]);
            }
}

// generate_element2node(Q9) (src/mesh/connectivity.jl, tensor ordering as Q9_NODES).
inline void q9_el2n(int nx, int ny, int32_t* el2n) {
    const int64_t sy = 2 * nx + 1;
    int64_t iel = 0;
    for (int ey = 0; ey < ny; ++ey)
        for (int ex = 0; ex < nx; ++ex, ++iel) {
            int32_t* e = el2n + 9 * iel;
            for (int a = 0; a < 9; ++a)
                e[a] = (int32_t)((2 * ey + 1 + Q9_NODES[a][1]) * sy + (2 * ex + 1 + Q9_NODES[a][0]) + 1);
        }
}

// Inverse Jacobian and |det J|·ω at every quadrature point
// (precompute_geometry_kernel!, src/mesh/mesh.jl:674-682; _geometry_entry :550).
// coords is dim × nnodes (AoS, one SVector per node).
inline void geometry(int dim, int64_t nels, const double* coords, const int32_t* el2n,
                     double* geo_v, double* geo_P) {
    const Tables& t = tables_for(dim);
    const int D = dim, NV = t.nv, NQ = t.nq, S = D * D + 1;
    for (int64_t e = 0; e < nels; ++e) {
        for (int q = 0; q < NQ; ++q) {
            double J[3][3] = {{0}};
            for (int a = 0; a < NV; ++a) {
                const double* x = coords + (int64_t)D * (el2n[NV * e + a] - 1);
                for (int i = 0; i < D; ++i)
                    for (int j = 0; j < D; ++j) J[i][j] += x[i] * t.dN[q][a][j];
            }
            double inv[3][3], det;
            if (D == 3) {
                det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                      J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
                inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
                inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
                inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
                inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
                inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
                inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
                inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
                inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
                inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
            } else {
                det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
                inv[0][0] = J[1][1] / det; inv[0][1] = -J[0][1] / det;
                inv[1][0] = -J[1][0] / det; inv[1][1] = J[0][0] / det;
            }
            double* g = geo_v + ((int64_t)e * NQ + q) * S;
            for (int c = 0; c < D; ++c)
                for (int r = 0; r < D; ++r) g[r + D * c] = inv[r][c];   // column-major
            g[D * D] = std::fabs(det) * t.w[q];
            if (geo_P) geo_P[(int64_t)e * NQ + q] = std::fabs(det) * t.w[q];
        }
    }
}

}  // namespace orc
