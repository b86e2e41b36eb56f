// Physics-AI coupling kernels (sm_100a): network features and the
// volume-preserving residual correction of the hybrid rollout
// (src/hybrid_flood/hybrid/coupled_forecast.py:49-120).
#pragma once

#include <cuda_bf16.h>

#include "swe_step.cuh"

namespace swe {

// Feature layouts.
//   kFeatRef6   the reference's six channels (coupled_forecast.py:53-79):
//               (h, u, v) standardised by mean/std and zeroed off-mask, the rain
//               rate in mm/h over its scale, standardised terrain, roughness.
//   kFeatState5 (h, hu, hv, z, rain rate in mm/h), each standardised by
//               mean/std, off-mask cells zero.
constexpr int kFeatRef6 = 0;
constexpr int kFeatState5 = 1;

struct FeatureArgs {
    int rows, cols;
    StateView s;
    const float* nm;    // n^2 with the mask in the sign bit (pitch spitch)
    const float* bed;   // pitch spitch
    int64_t spitch;
    const float* terrain;    // rows*cols (kFeatRef6), may be null
    const float* roughness;  // rows*cols (kFeatRef6), may be null
    float mean[5], stdv[5];
    float rain_feature;      // the rain channel's value for this call
    float dry;
    int layout;              // kFeatRef6 / kFeatState5
    int channels;            // 6 or 5
    void* out;               // [rows][cols][channels] (channels-last)
    int out_bf16;            // 1: bfloat16, 0: float32
};

__global__ void features_kernel(const FeatureArgs a) {
    for_cells(0, a.rows, a.cols, [&](int r, int c) {
        const int64_t i = (int64_t)r * a.cols + c;
        const int64_t so = (int64_t)r * a.s.pitch + c, zo = (int64_t)r * a.spitch + c;
        const float h = a.s.h[so], hu = a.s.hu[so], hv = a.s.hv[so];
        const bool act = active(a.nm[zo]);
        float f[6];
        if (a.layout == kFeatRef6) {
            const bool wet = h > a.dry;
            const float u = wet ? __fdiv_rn(hu, fmaxf(h, a.dry)) : 0.f;
            const float v = wet ? __fdiv_rn(hv, fmaxf(h, a.dry)) : 0.f;
            f[0] = act ? __fdiv_rn(__fsub_rn(h, a.mean[0]), a.stdv[0]) : 0.f;
            f[1] = act ? __fdiv_rn(__fsub_rn(u, a.mean[1]), a.stdv[1]) : 0.f;
            f[2] = act ? __fdiv_rn(__fsub_rn(v, a.mean[2]), a.stdv[2]) : 0.f;
            f[3] = a.rain_feature;
            f[4] = a.terrain ? a.terrain[i] : 0.f;
            f[5] = a.roughness ? a.roughness[i] : 0.f;
        } else {
            const float src[5] = {h, hu, hv, a.bed[zo], a.rain_feature};
            for (int q = 0; q < 5; ++q) f[q] = act ? __fdiv_rn(__fsub_rn(src[q], a.mean[q]), a.stdv[q]) : 0.f;
        }
        if (a.out_bf16) {
            __nv_bfloat16* o = static_cast<__nv_bfloat16*>(a.out) + i * a.channels;
            for (int q = 0; q < a.channels; ++q) o[q] = __float2bfloat16_rn(f[q]);
        } else {
            float* o = static_cast<float*>(a.out) + i * a.channels;
            for (int q = 0; q < a.channels; ++q) o[q] = f[q];
        }
    });
}

struct CorrectionArgs {
    int rows, cols;
    StateView s;          // predicted state (physics result)
    StateOut out;         // corrected state (may alias s)
    float* prov;          // scratch plane for the provisional depth, pitch prov_pitch
    int64_t prov_pitch;
    const float* nm;
    int64_t spitch;
    const void* res;      // residual, element (r, c, ch) at res[r*rs_r + c*rs_c + ch*rs_ch]
    int64_t rs_r, rs_c, rs_ch;
    int res_channels;     // 1 (depth only) or 3 (depth, u, v)
    int res_bf16;         // 1: bfloat16 residual, 0: float32
    float lim[3];         // clip limits per channel (+inf: none), coupled_forecast.py:199-200
    float relax, dry, eps;
    double* sums;         // [2] device: sum of masked predicted h, sum of provisional h
};

// Residual channel ch at (r, c), clipped to [-lim, lim] with NaN kept (jnp.clip).
__device__ __forceinline__ float residual_at(const CorrectionArgs& a, int r, int c, int ch) {
    const int64_t o = (int64_t)r * a.rs_r + (int64_t)c * a.rs_c + (int64_t)ch * a.rs_ch;
    const float x = a.res_bf16 ? __bfloat162float(static_cast<const __nv_bfloat16*>(a.res)[o])
                               : static_cast<const float*>(a.res)[o];
    const float l = a.lim[ch];
    return x < -l ? -l : (x > l ? l : x);
}

// Pass 1: provisional depth max(h + r*res_h, 0) on active cells (into the
// scratch plane) and the two volume sums in float64 (coupled_forecast.py:98-104).
__global__ void correction_sums_kernel(const CorrectionArgs a) {
    double t = 0.0, p = 0.0;
    for_cells(0, a.rows, a.cols, [&](int r, int c) {
        const int64_t so = (int64_t)r * a.s.pitch + c;
        const bool act = active(a.nm[(int64_t)r * a.spitch + c]);
        const float h = a.s.h[so];
        const float rh = residual_at(a, r, c, 0);
        const float prov = act ? fmaxf(__fadd_rn(h, __fmul_rn(a.relax, rh)), 0.f) : 0.f;
        a.prov[(int64_t)r * a.prov_pitch + c] = prov;  // provisional depth, scaled in pass 2
        if (act) t += (double)h;
        p += (double)prov;
    });
    t = warp_sum(t);
    p = warp_sum(p);
    __shared__ double s_t[32], s_p[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        s_t[w] = t;
        s_p[w] = p;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tt = 0.0, pp = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            tt += s_t[k];
            pp += s_p[k];
        }
        atomicAdd(&a.sums[0], tt);
        atomicAdd(&a.sums[1], pp);
    }
}

// Pass 2: project onto the physics volume and rebuild the momenta
// (coupled_forecast.py:105-120).  Reads the predicted momenta before writing.
__global__ void correction_apply_kernel(const CorrectionArgs a) {
    const double target = a.sums[0], provisional = a.sums[1];
    const float scale = provisional > (double)a.eps ? (float)(target / provisional) : 1.f;
    const bool keep = !(target > (double)a.eps);
    for_cells(0, a.rows, a.cols, [&](int r, int c) {
        const int64_t so = (int64_t)r * a.s.pitch + c, oo = (int64_t)r * a.out.pitch + c;
        const bool act = active(a.nm[(int64_t)r * a.spitch + c]);
        const float h = a.s.h[so], hu = a.s.hu[so], hv = a.s.hv[so];
        const bool wet0 = h > a.dry;
        float u = wet0 ? __fdiv_rn(hu, fmaxf(h, a.dry)) : 0.f;
        float v = wet0 ? __fdiv_rn(hv, fmaxf(h, a.dry)) : 0.f;
        const float prov = a.prov[(int64_t)r * a.prov_pitch + c];
        const float ch = keep ? h : __fmul_rn(prov, scale);
        if (a.res_channels >= 3) {
            u = __fadd_rn(u, __fmul_rn(a.relax, residual_at(a, r, c, 1)));
            v = __fadd_rn(v, __fmul_rn(a.relax, residual_at(a, r, c, 2)));
        }
        const bool wet = act && ch > a.dry;
        a.out.h[oo] = ch;
        a.out.hu[oo] = wet ? __fmul_rn(ch, u) : 0.f;
        a.out.hv[oo] = wet ? __fmul_rn(ch, v) : 0.f;
    });
}

// Output schema of a state (conserved_to_xarray, structured_io.py:160-209):
// depth, x/y velocity (momentum / depth where depth > dry, else 0) and speed
// (hypot, evaluated in double and rounded once as float32 hypot is), each NaN
// off the domain mask.  IEEE division, so the fields equal NumPy's bit for bit.
struct SchemaArgs {
    int rows, cols;
    StateView s;
    const float* nm;
    int64_t spitch;
    float dry;
    float *depth, *u, *v, *speed;
    int64_t out_pitch;
};

__global__ void schema_kernel(const SchemaArgs a) {
    const float nan = __int_as_float(0x7fc00000);
    for_cells(0, a.rows, a.cols, [&](int r, int c) {
        const int64_t so = (int64_t)r * a.s.pitch + c, oo = (int64_t)r * a.out_pitch + c;
        const bool act = active(a.nm[(int64_t)r * a.spitch + c]);
        const float h = a.s.h[so];
        const bool wet = h > a.dry;
        const float u = wet ? __fdiv_rn(a.s.hu[so], h) : 0.f;
        const float v = wet ? __fdiv_rn(a.s.hv[so], h) : 0.f;
        a.depth[oo] = act ? h : nan;
        a.u[oo] = act ? u : nan;
        a.v[oo] = act ? v : nan;
        a.speed[oo] = act ? ExactMath::hypot(u, v) : nan;
    });
}

}  // namespace swe
