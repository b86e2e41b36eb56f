// Bias + activation epilogue of the corrector's convolutions, channels-last
// (sm_100a).
//
// The convolutions of the residual U-Net (src/hybrid_flood/benchmark/
// pytorch_residual_net.py:79-170) run through cuDNN in bfloat16 NHWC; for these
// shapes its fastest algorithms carry no bias epilogue, and the framework then
// adds the bias with a broadcasting elementwise pass and applies the ReLU with
// another.  This kernel does both in one pass over the convolution's output,
// in place: y[i] = act(y[i] + bias[i % C]), 16-byte vector accesses.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace swe {

template <bool RELU>
__device__ __forceinline__ float bias_act(float x, float b) {
    const float y = x + b;
    return RELU ? fmaxf(y, 0.f) : y;
}

// bfloat16, C a multiple of 8: eight channels per 16-byte vector.
template <bool RELU>
__global__ void bias_act_bf16x8_kernel(__nv_bfloat16* __restrict__ y, int64_t n_vec, int channels,
                                       const float* __restrict__ bias) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n_vec; v += (int64_t)gridDim.x * blockDim.x) {
        uint4 raw = reinterpret_cast<const uint4*>(y)[v];
        const int c0 = (int)((v * 8) % channels);
        __nv_bfloat162* p = reinterpret_cast<__nv_bfloat162*>(&raw);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float2 f = __bfloat1622float2(p[k]);
            p[k] = __floats2bfloat162_rn(bias_act<RELU>(f.x, __ldg(bias + c0 + 2 * k)),
                                          bias_act<RELU>(f.y, __ldg(bias + c0 + 2 * k + 1)));
        }
        reinterpret_cast<uint4*>(y)[v] = raw;
    }
}

// Any C, bfloat16 or float32, one element per thread step.
template <typename T, bool RELU>
__global__ void bias_act_scalar_kernel(T* __restrict__ y, int64_t n, int channels, const float* __restrict__ bias) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float b = __ldg(bias + (int)(i % channels));
        if constexpr (sizeof(T) == 2) {
            y[i] = __float2bfloat16_rn(bias_act<RELU>(__bfloat162float(y[i]), b));
        } else {
            y[i] = bias_act<RELU>(y[i], b);
        }
    }
}

}  // namespace swe
