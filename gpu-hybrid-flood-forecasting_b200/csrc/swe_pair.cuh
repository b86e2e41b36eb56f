// Paired-lane arithmetic for the step kernel (sm_100a).
//
// A lane owns two neighbouring cells and carries their fields as float2.  In
// the fast policy every add/multiply/fma of a pair is one packed sm_100
// instruction (__fadd2_rn / __fmul2_rn / __ffma2_rn).  The exact policy keeps
// the scalar __fadd_rn / __fmul_rn per component: those are documented never
// to be merged into a fused multiply-add, a guarantee the packed forms do not
// state (measured: packed exact arithmetic drifted by ulps from the reference
// on a lake at rest, the scalar form is bit-identical).  Divisions, square
// roots, compares and selects are per component in both policies.
#pragma once

#include <cuda_runtime.h>

#include "swe_math.cuh"

namespace swe {

struct B2 {
    bool x, y;
};
__device__ __forceinline__ B2 operator&(B2 a, B2 b) { return {a.x && b.x, a.y && b.y}; }
__device__ __forceinline__ B2 operator|(B2 a, B2 b) { return {a.x || b.x, a.y || b.y}; }
__device__ __forceinline__ B2 operator!(B2 a) { return {!a.x, !a.y}; }

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 splat(float a) { return make_float2(a, a); }

__device__ __forceinline__ bool gt(float a, float b) { return a > b; }
__device__ __forceinline__ B2 gt(float2 a, float2 b) { return {a.x > b.x, a.y > b.y}; }
__device__ __forceinline__ bool ge(float a, float b) { return a >= b; }
__device__ __forceinline__ B2 ge(float2 a, float2 b) { return {a.x >= b.x, a.y >= b.y}; }
__device__ __forceinline__ bool le(float a, float b) { return a <= b; }
__device__ __forceinline__ B2 le(float2 a, float2 b) { return {a.x <= b.x, a.y <= b.y}; }
__device__ __forceinline__ float sel(bool p, float a, float b) { return p ? a : b; }
__device__ __forceinline__ float2 sel(B2 p, float2 a, float2 b) { return {p.x ? a.x : b.x, p.y ? a.y : b.y}; }
__device__ __forceinline__ float vmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ float2 vmax(float2 a, float2 b) { return {fmaxf(a.x, b.x), fmaxf(a.y, b.y)}; }
__device__ __forceinline__ float vmin(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ float2 vmin(float2 a, float2 b) { return {fminf(a.x, b.x), fminf(a.y, b.y)}; }
// Three-input minimum / maximum (one sm_100 instruction each; NaN inputs are
// ignored as by fminf / fmaxf).
__device__ __forceinline__ float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float vmin3(float a, float b, float c) { return min3f(a, b, c); }
__device__ __forceinline__ float2 vmin3(float2 a, float2 b, float2 c) { return {min3f(a.x, b.x, c.x), min3f(a.y, b.y, c.y)}; }
__device__ __forceinline__ float vmax3(float a, float b, float c) { return max3f(a, b, c); }
__device__ __forceinline__ float2 vmax3(float2 a, float2 b, float2 c) { return {max3f(a.x, b.x, c.x), max3f(a.y, b.y, c.y)}; }
__device__ __forceinline__ float vabs(float a) { return fabsf(a); }
__device__ __forceinline__ float2 vabs(float2 a) { return {fabsf(a.x), fabsf(a.y)}; }
__device__ __forceinline__ float neg(float a) { return -a; }
__device__ __forceinline__ float2 neg(float2 a) { return {-a.x, -a.y}; }
__device__ __forceinline__ bool act_of(float nm) { return !signbit(nm); }
__device__ __forceinline__ B2 act_of(float2 nm) { return {!signbit(nm.x), !signbit(nm.y)}; }
template <class T>
__device__ __forceinline__ auto all_true();
template <>
__device__ __forceinline__ auto all_true<float>() { return true; }
template <>
__device__ __forceinline__ auto all_true<float2>() { return B2{true, true}; }

// Arithmetic of one policy, overloaded for a scalar and a pair.
template <class M>
struct P;

template <>
struct P<ExactMath> {
    static constexpr bool kExact = true;
    __device__ static __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    __device__ static __forceinline__ float2 add(float2 a, float2 b) {
        return {__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y)};
    }
    __device__ static __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    __device__ static __forceinline__ float2 sub(float2 a, float2 b) {
        return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y)};
    }
    __device__ static __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    __device__ static __forceinline__ float2 mul(float2 a, float2 b) {
        return {__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)};
    }
    __device__ static __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
    __device__ static __forceinline__ float2 div(float2 a, float2 b) {
        return {__fdiv_rn(a.x, b.x), __fdiv_rn(a.y, b.y)};
    }
    __device__ static __forceinline__ float sqrt(float a) { return __fsqrt_rn(a); }
    __device__ static __forceinline__ float2 sqrt(float2 a) { return {__fsqrt_rn(a.x), __fsqrt_rn(a.y)}; }
    __device__ static __forceinline__ float hypot(float a, float b) { return ExactMath::hypot(a, b); }
    __device__ static __forceinline__ float2 hypot(float2 a, float2 b) {
        return {ExactMath::hypot(a.x, b.x), ExactMath::hypot(a.y, b.y)};
    }
    __device__ static __forceinline__ float pow73(float x, float e) { return powf(x, e); }
    __device__ static __forceinline__ float2 pow73(float2 x, float e) { return {powf(x.x, e), powf(x.y, e)}; }
};

template <>
struct P<FastMath> {
    static constexpr bool kExact = false;
    __device__ static __forceinline__ float add(float a, float b) { return a + b; }
    __device__ static __forceinline__ float2 add(float2 a, float2 b) { return __fadd2_rn(a, b); }
    __device__ static __forceinline__ float sub(float a, float b) { return a - b; }
    __device__ static __forceinline__ float2 sub(float2 a, float2 b) { return __fadd2_rn(a, neg(b)); }
    __device__ static __forceinline__ float mul(float a, float b) { return a * b; }
    __device__ static __forceinline__ float2 mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
    __device__ static __forceinline__ float fma(float a, float b, float c) { return fmaf(a, b, c); }
    __device__ static __forceinline__ float2 fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
    __device__ static __forceinline__ float rcp(float a) { return FastMath::rcp(a); }
    __device__ static __forceinline__ float2 rcp(float2 a) { return {FastMath::rcp(a.x), FastMath::rcp(a.y)}; }
    __device__ static __forceinline__ float sqrt(float a) { return FastMath::sqrt(a); }
    __device__ static __forceinline__ float2 sqrt(float2 a) { return {FastMath::sqrt(a.x), FastMath::sqrt(a.y)}; }
    __device__ static __forceinline__ float lg2(float a) {
        float r;
        asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
        return r;
    }
    __device__ static __forceinline__ float2 lg2(float2 a) { return {lg2(a.x), lg2(a.y)}; }
    __device__ static __forceinline__ float ex2(float a) {
        float r;
        asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
        return r;
    }
    __device__ static __forceinline__ float2 ex2(float2 a) { return {ex2(a.x), ex2(a.y)}; }
};

template <class T>
struct CellT {
    T h, hu, hv, z, nm;  // nm: n^2 with the mask in the sign bit
    T u, v;              // velocities from the unreconstructed depth
};

template <class T>
struct FaceT {
    T f0, f1, f2;        // HLL flux (mass, x-momentum, y-momentum), zero if irrelevant
    T corr_lo, corr_hi;  // normal-momentum pressure corrections of the two sides
};

// Step constants as scalars and as splatted pairs.
struct KPair {
    float2 g, half_g, dry, eps, zero, one, tiny;
};

__device__ __forceinline__ KPair make_kpair(const Consts& k) {
    return {splat(k.g), splat(k.half_g), splat(k.dry), splat(k.eps), splat(0.f), splat(1.f),
            splat(1.0e-30f)};
}

// Velocities of a cell or a pair of cells (numpy_solver/shallow_water_2d.py:60-63).
template <class M, class T, class KP>
__device__ __forceinline__ void set_vel_t(CellT<T>& c, const KP& kp) {
    using A = P<M>;
    const auto wet = gt(c.h, kp.dry);
    if constexpr (A::kExact) {
        c.u = sel(wet, A::div(c.hu, c.h), kp.zero);
        c.v = sel(wet, A::div(c.hv, c.h), kp.zero);
    } else {
        const T r = sel(wet, A::rcp(c.h), kp.zero);
        c.u = A::mul(c.hu, r);
        c.v = A::mul(c.hv, r);
    }
}

// One face (or a pair of faces): wall mirroring at active/inactive faces,
// hydrostatic reconstruction, HLL, side-specific pressure corrections
// (numpy_solver/shallow_water_2d.py:66-239).  AXIS 1 = x-face, 0 = y-face.
//
// Exact policy: the reference's operation order, including the velocity
// recomputed from the reconstructed momentum and the three-way flux select.
// Fast policy: (H*u)/H = u, and the HLL flux in its clamped-speed form
// (s- = min(sL, 0), s+ = max(sR, 0)), which equals the select form exactly in
// real arithmetic and needs no compares.
template <int AXIS, class M, bool MASKED, class T, class KP>
__device__ __forceinline__ FaceT<T> face_t(const CellT<T>& lo, const CellT<T>& hi, const KP& kp) {
    using A = P<M>;
    T hL = lo.h, zL = lo.z, hR = hi.h, zR = hi.z;
    T uL = lo.u, vL = lo.v, uR = hi.u, vR = hi.v;
    auto relevant = all_true<T>();
    if constexpr (MASKED) {
        const auto a_lo = act_of(lo.nm), a_hi = act_of(hi.nm);
        relevant = a_lo | a_hi;
        const auto hi_wall = a_lo & !a_hi;
        const auto lo_wall = !a_lo & a_hi;
        hL = sel(lo_wall, hi.h, lo.h);
        zL = sel(lo_wall, hi.z, lo.z);
        hR = sel(hi_wall, lo.h, hi.h);
        zR = sel(hi_wall, lo.z, hi.z);
        if constexpr (AXIS == 1) {
            uL = sel(lo_wall, neg(hi.u), lo.u);
            vL = sel(lo_wall, hi.v, lo.v);
            uR = sel(hi_wall, neg(lo.u), hi.u);
            vR = sel(hi_wall, lo.v, hi.v);
        } else {
            uL = sel(lo_wall, hi.u, lo.u);
            vL = sel(lo_wall, neg(hi.v), lo.v);
            uR = sel(hi_wall, lo.u, hi.u);
            vR = sel(hi_wall, neg(lo.v), hi.v);
        }
    }
    const T zf = vmax(zL, zR);
    const T HL = vmax(A::sub(A::add(hL, zL), zf), kp.zero);
    const T HR = vmax(A::sub(A::add(hR, zR), zf), kp.zero);
    const T XL = A::mul(HL, uL), YL = A::mul(HL, vL);
    const T XR = A::mul(HR, uR), YR = A::mul(HR, vR);
    const auto wL = gt(HL, kp.dry), wR = gt(HR, kp.dry);
    T unL, unR, tL, tR;  // normal velocity; tangential factor of the third flux
    if constexpr (A::kExact) {
        unL = sel(wL, A::div(AXIS == 1 ? XL : YL, HL), kp.zero);
        unR = sel(wR, A::div(AXIS == 1 ? XR : YR, HR), kp.zero);
        if constexpr (AXIS == 1) {
            tL = sel(wL, A::div(YL, HL), kp.zero);
            tR = sel(wR, A::div(YR, HR), kp.zero);
        }
    } else {
        unL = sel(wL, AXIS == 1 ? uL : vL, kp.zero);
        unR = sel(wR, AXIS == 1 ? uR : vR, kp.zero);
        if constexpr (AXIS == 1) {
            tL = sel(wL, vL, kp.zero);
            tR = sel(wR, vR, kp.zero);
        }
    }
    const T cL = A::sqrt(A::mul(kp.g, HL));
    const T cR = A::sqrt(A::mul(kp.g, HR));
    const T pL = A::mul(kp.half_g, A::mul(HL, HL));
    const T pR = A::mul(kp.half_g, A::mul(HR, HR));
    T fL0, fL1, fL2, fR0, fR1, fR2;
    if constexpr (AXIS == 1) {
        fL0 = XL;
        fR0 = XR;
        fL2 = A::mul(XL, tL);
        fR2 = A::mul(XR, tR);
        if constexpr (A::kExact) {
            fL1 = A::add(A::mul(XL, unL), pL);
            fR1 = A::add(A::mul(XR, unR), pR);
        } else {
            fL1 = A::fma(XL, unL, pL);
            fR1 = A::fma(XR, unR, pR);
        }
    } else {
        fL0 = YL;
        fR0 = YR;
        fL1 = A::mul(XL, unL);
        fR1 = A::mul(XR, unR);
        if constexpr (A::kExact) {
            fL2 = A::add(A::mul(YL, unL), pL);
            fR2 = A::add(A::mul(YR, unR), pR);
        } else {
            fL2 = A::fma(YL, unL, pL);
            fR2 = A::fma(YR, unR, pR);
        }
    }
    FaceT<T> f;
    if constexpr (A::kExact) {
        const T sL = vmin(A::sub(unL, cL), A::sub(unR, cR));
        const T sR = vmax(A::add(unL, cL), A::add(unR, cR));
        const T spread = A::sub(sR, sL);
        const T den = sel(gt(spread, kp.eps), spread, kp.one);
        const T s01 = A::mul(sL, sR);
        const T m0 = A::div(A::add(A::sub(A::mul(sR, fL0), A::mul(sL, fR0)), A::mul(s01, A::sub(HR, HL))), den);
        const T m1 = A::div(A::add(A::sub(A::mul(sR, fL1), A::mul(sL, fR1)), A::mul(s01, A::sub(XR, XL))), den);
        const T m2 = A::div(A::add(A::sub(A::mul(sR, fL2), A::mul(sL, fR2)), A::mul(s01, A::sub(YR, YL))), den);
        const auto take_l = ge(sL, kp.zero), take_r = le(sR, kp.zero);
        f.f0 = sel(relevant, sel(take_l, fL0, sel(take_r, fR0, m0)), kp.zero);
        f.f1 = sel(relevant, sel(take_l, fL1, sel(take_r, fR1, m1)), kp.zero);
        f.f2 = sel(relevant, sel(take_l, fL2, sel(take_r, fR2, m2)), kp.zero);
        f.corr_lo = sel(relevant, A::mul(kp.half_g, A::sub(A::mul(hL, hL), A::mul(HL, HL))), kp.zero);
        f.corr_hi = sel(relevant, A::mul(kp.half_g, A::sub(A::mul(hR, hR), A::mul(HR, HR))), kp.zero);
    } else {
        // Clamped speeds: sL >= 0 gives fL, sR <= 0 gives fR, otherwise the HLL
        // middle state.  s- = min(sL, 0) and s+ = max(sR, 0) are each one
        // three-input instruction; s+ - s- >= 0, and the tiny term keeps the
        // reciprocal finite where both speeds are zero (a still, dry face, whose
        // flux terms are then all zero).
        const T sm = vmin3(A::sub(unL, cL), A::sub(unR, cR), kp.zero);
        const T sp = vmax3(A::add(unL, cL), A::add(unR, cR), kp.zero);
        const T rden = A::rcp(A::add(A::sub(sp, sm), kp.tiny));
        const T smp = A::mul(sm, sp);
        const T nsm = neg(sm);
        T m0 = A::fma(smp, A::sub(HR, HL), A::fma(nsm, fR0, A::mul(sp, fL0)));
        T m1 = A::fma(smp, A::sub(XR, XL), A::fma(nsm, fR1, A::mul(sp, fL1)));
        T m2 = A::fma(smp, A::sub(YR, YL), A::fma(nsm, fR2, A::mul(sp, fL2)));
        m0 = A::mul(m0, rden);
        m1 = A::mul(m1, rden);
        m2 = A::mul(m2, rden);
        const T cl = A::mul(kp.half_g, A::fma(hL, hL, neg(A::mul(HL, HL))));
        const T ch = A::mul(kp.half_g, A::fma(hR, hR, neg(A::mul(HR, HR))));
        if constexpr (MASKED) {
            f.f0 = sel(relevant, m0, kp.zero);
            f.f1 = sel(relevant, m1, kp.zero);
            f.f2 = sel(relevant, m2, kp.zero);
            f.corr_lo = sel(relevant, cl, kp.zero);
            f.corr_hi = sel(relevant, ch, kp.zero);
        } else {
            f.f0 = m0;
            f.f1 = m1;
            f.f2 = m2;
            f.corr_lo = cl;
            f.corr_hi = ch;
        }
    }
    return f;
}

}  // namespace swe
