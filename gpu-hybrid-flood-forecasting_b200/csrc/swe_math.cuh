// Arithmetic policies for the shallow-water step kernels (sm_100a).
//
// ExactMath rounds every operation on its own, in the order the reference
// NumPy solver performs it (src/hybrid_flood/numpy_solver/shallow_water_2d.py):
// explicit __fadd_rn/__fmul_rn/__fdiv_rn/__fsqrt_rn intrinsics, which the
// compiler never contracts into FMA whatever the -fmad setting.  Its only
// deliberate difference from the reference is powf in the friction term.
// hypot is evaluated as glibc's hypotf does (double products, one double sqrt,
// one rounding to float), which NumPy's float32 hypot reproduces.
//
// FastMath keeps the same algorithm but lets the compiler fuse multiply-adds,
// uses the hardware approximate reciprocal / square root / log2 / exp2
// (MUFU), divides the three HLL middle-state components by one reciprocal,
// and uses the identity (H*u)/H == u for the reconstructed velocities.  Its
// results are checked against the oracle with the tolerance the tests state.
#pragma once

#include <cuda_runtime.h>

namespace swe {

struct ExactMath {
    static constexpr bool kExact = true;
    __device__ static __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    __device__ static __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    __device__ static __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    __device__ static __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
    __device__ static __forceinline__ float sqrt(float a) { return __fsqrt_rn(a); }
    // Reciprocal of the HLL denominator; exact mode divides each component instead.
    __device__ static __forceinline__ float recip(float a) { return a; }
    __device__ static __forceinline__ float over(float num, float den_or_recip) {
        return __fdiv_rn(num, den_or_recip);
    }
    // m / max(h, dry) where h > dry, else 0 (shallow_water_2d.py:60-63).
    __device__ static __forceinline__ float vel(float m, float h, float dry) {
        return h > dry ? __fdiv_rn(m, h) : 0.0f;
    }
    // Both velocities of a cell from one depth.
    __device__ static __forceinline__ void vel2(float mx, float my, float h, float dry, float& u,
                                                float& v) {
        const bool wet = h > dry;
        u = wet ? __fdiv_rn(mx, h) : 0.0f;
        v = wet ? __fdiv_rn(my, h) : 0.0f;
    }
    // Velocity recomputed from a reconstructed momentum H*u (shallow_water_2d.py:76-79).
    __device__ static __forceinline__ float recon_vel(float m, float H, float dry, float /*u*/) {
        return H > dry ? __fdiv_rn(m, H) : 0.0f;
    }
    __device__ static __forceinline__ float hypot(float a, float b) {
        const double da = (double)a, db = (double)b;
        return __double2float_rn(__dsqrt_rn(__dadd_rn(__dmul_rn(da, da), __dmul_rn(db, db))));
    }
    // max(h, dry) ** (7/3) with the exponent rounded to float as NumPy does.
    __device__ static __forceinline__ float pow73(float x, float expo) { return powf(x, expo); }
};

struct FastMath {
    static constexpr bool kExact = false;
    __device__ static __forceinline__ float add(float a, float b) { return a + b; }
    __device__ static __forceinline__ float sub(float a, float b) { return a - b; }
    __device__ static __forceinline__ float mul(float a, float b) { return a * b; }
    __device__ static __forceinline__ float rcp(float a) {
        float r;
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
        return r;
    }
    __device__ static __forceinline__ float div(float a, float b) { return a * rcp(b); }
    __device__ static __forceinline__ float sqrt(float a) {
        float r;
        asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
        return r;
    }
    __device__ static __forceinline__ float recip(float a) { return rcp(a); }
    __device__ static __forceinline__ float over(float num, float recip_den) { return num * recip_den; }
    __device__ static __forceinline__ float vel(float m, float h, float dry) {
        return h > dry ? m * rcp(h) : 0.0f;
    }
    __device__ static __forceinline__ void vel2(float mx, float my, float h, float dry, float& u,
                                                float& v) {
        const float r = h > dry ? rcp(h) : 0.0f;
        u = mx * r;
        v = my * r;
    }
    __device__ static __forceinline__ float recon_vel(float /*m*/, float H, float dry, float u) {
        return H > dry ? u : 0.0f;
    }
    __device__ static __forceinline__ float hypot(float a, float b) { return sqrt(a * a + b * b); }
    __device__ static __forceinline__ float pow73(float x, float expo) {
        float l, r;
        asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(l) : "f"(x));
        asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(l * expo));
        return r;
    }
};

}  // namespace swe
