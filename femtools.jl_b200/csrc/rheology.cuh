// rheology.cuh — pointwise visco-elasto-plastic stress updates shared by the sweeps.
#pragma once
#include "common.cuh"

namespace femb {

// Stress increment of the Drucker–Prager radial return (rheology.jl:441-472)
// between the base trial stress tb (yield value Fk) and the trial stress tb + dtt,
// with pressure increment dPeq. Written in increments (J2 difference through the
// cross term, f' − f through δλ and δτII), so that no two nearly equal stresses
// are subtracted and the FP32 error scales with the increment, not the stress.
// The return is τ = τtr − f·M·τtr with M = ½ on the normal and 1 on the shear
// components and f = 2ηve·λ/(τII + ε²), λ = F/den.
// Square root and quotient of the increment formula: IEEE-rounded by default; with
// FAST (the FP32 sweep away from the apex, where every argument is a normal
// positive number) the hardware approximations of about 2 ulp.
template <class U, bool FAST> struct DpOps {
    static FEMB_D U root(U x) { return sqrt(x); }
    static FEMB_D U quot(U a, U b) { return a / b; }
};
template <> struct DpOps<float, true> {
    static FEMB_D float root(float x) {
        float r;
        asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
        return r;
    }
    static FEMB_D float quot(float a, float b) { return __fdividef(a, b); }
};

template <class U, bool FAST = false>
FEMB_D void dp_increment(const U tb[6], U Fk, const U dtt[6], U dPeq, U twoe, U sphi, U inv_den, U eps2, U out[6]) {
    using O = DpOps<U, FAST>;
    const U Jk = U(0.5) * (tb[0] * tb[0] + tb[1] * tb[1] + tb[2] * tb[2]) + tb[3] * tb[3] + tb[4] * tb[4] + tb[5] * tb[5];
    const U cross = tb[0] * dtt[0] + tb[1] * dtt[1] + tb[2] * dtt[2] + U(2) * (tb[3] * dtt[3] + tb[4] * dtt[4] + tb[5] * dtt[5]);
    const U dd = U(0.5) * (dtt[0] * dtt[0] + dtt[1] * dtt[1] + dtt[2] * dtt[2]) + dtt[3] * dtt[3] + dtt[4] * dtt[4] + dtt[5] * dtt[5];
    const U tIIk = O::root(Jk + eps2);
    const U tIIn = O::root(Jk + eps2 + (cross + dd));
    const U dtII = O::quot(cross + dd, tIIn + tIIk);
    const U dF = dtII - sphi * dPeq;
    const U Fn = Fk + dF;
    const bool pk = Fk > U(0), pn = Fn > U(0);
    const U lamk = pk ? Fk * inv_den : U(0);
    U fn = U(0), df = U(0);
    if (pn) {
        fn = O::quot(twoe * (Fn * inv_den), tIIn + eps2);
        df = pk ? O::quot(twoe * (dF * inv_den * (tIIk + eps2) - lamk * dtII), (tIIn + eps2) * (tIIk + eps2)) : fn;
    } else if (pk) {
        df = -O::quot(twoe * lamk, tIIk + eps2);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) out[c] = dtt[c] - U(0.5) * (fn * dtt[c] + df * tb[c]);
#pragma unroll
    for (int c = 3; c < 6; ++c) out[c] = dtt[c] - (fn * dtt[c] + df * tb[c]);
}


// Tiled layout of the per-point base data of the mixed-precision solve (the FP32
// trial stress τ_xx, τ_yy, τ_zz, τ_xy, τ_xz, τ_yz and the yield value F of every
// integration point at the FP64 base state): elements in tiles of 32, so that 32
// consecutive elements read one point's component as one 128-byte line.
constexpr int BASE_FIELDS = 7;
FEMB_HD int64_t base_index(int64_t e, int q, int c) {
    return (((e >> 5) * 27 + q) * BASE_FIELDS + c) * 32 + (e & 31);
}

}  // namespace femb
