// Device generators of the synthetic measurement inputs (sm_100a): the urban
// DEM with its Manning field, the Gamma hyetograph and the smoothed log-normal
// Manning field.
//
// The reference builds its terrain on the host from GIS inputs
// (src/hybrid_flood/dem/synthetic_terrain.py:114 generate_base_terrain,
// src/hybrid_flood/dem/urban_conditioning.py:128 condition_urban_terrain); the
// measured workloads here are seeded synthetic fields of the same kind, and at
// 64 ensemble members or 2048x2048 refined targets their host generation and
// upload cost more than the runs they feed.  These kernels build them in place
// in device memory.
//
// Random numbers come from Philox-4x32-10 (Salmon, Moraes, Dror and Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC 2011), a counter-based
// generator: draw i of a stream is a pure function of (seed, i), so every
// thread draws its own numbers without shared state and the fields do not
// depend on the launch shape.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace swe {

// ---------------------------------------------------------------------------
// Philox-4x32-10
// ---------------------------------------------------------------------------
struct U4 {
    uint32_t x, y, z, w;
};

__device__ __forceinline__ void mulhilo(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
    const uint64_t p = (uint64_t)a * (uint64_t)b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
}

// Ten rounds of the Philox S-box/P-box network on a 128-bit counter with a
// 64-bit key (round multipliers and key increments of the published generator).
__device__ inline U4 philox(U4 c, uint32_t k0, uint32_t k1) {
    constexpr uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    constexpr uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo(M0, c.x, hi0, lo0);
        mulhilo(M1, c.z, hi1, lo1);
        c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
        k0 += W0;
        k1 += W1;
    }
    return c;
}

// Draw `idx` of stream `stream` under `seed`.
__device__ __forceinline__ U4 draw(uint64_t seed, uint32_t stream, uint64_t idx) {
    return philox(U4{(uint32_t)idx, (uint32_t)(idx >> 32), stream, 0u}, (uint32_t)seed, (uint32_t)(seed >> 32));
}

// Uniform double in (0, 1) from two 32-bit words (53 random bits, never 0).
__device__ __forceinline__ double u01(uint32_t a, uint32_t b) {
    const uint64_t m = ((uint64_t)a << 21) ^ (uint64_t)(b >> 11);
    return ((double)(m & ((uint64_t(1) << 53) - 1)) + 0.5) * (1.0 / 9007199254740992.0);
}

// Integer uniform on [lo, hi] (inclusive) by the multiply-shift map of a 32-bit word.
__device__ __forceinline__ int uniform_int(uint32_t r, int lo, int hi) {
    const uint64_t span = (uint64_t)(hi - lo + 1);
    return lo + (int)(((uint64_t)r * span) >> 32);
}

// Standard normal pair by the Box-Muller transform.
__device__ __forceinline__ double2 normal2(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    const double u1 = u01(a, b), u2 = u01(c, d);
    const double r = sqrt(-2.0 * log(u1));
    double s, co;
    sincospi(2.0 * u2, &s, &co);
    return make_double2(r * co, r * s);
}

// ---------------------------------------------------------------------------
// Urban DEM
// ---------------------------------------------------------------------------
// Block rectangles are drawn in order; a cell belongs to the blocks when the
// first rectangle that covers it comes before the stopping index K, the first
// index at which the cells covered so far reach the target fraction.  That is
// the sequential rule "add rectangles until coverage >= target" evaluated in
// parallel: each cell keeps the smallest index of the rectangles covering it
// (atomicMin), a histogram of those indices gives the cells each rectangle
// newly covers, and a prefix sum finds K.
struct Rect {
    int r0, c0, h, w;
};

// Rectangle i of the seeded stream: side lengths uniform on [min_side,
// max_side], the corner uniform over the positions that keep it in the grid.
__global__ void gen_rects_kernel(uint64_t seed, int n, int rows, int cols, int min_side, int max_side, Rect* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const U4 r = draw(seed, 1u, (uint64_t)i);
    Rect q;
    q.h = uniform_int(r.x, min_side, max_side);
    q.w = uniform_int(r.y, min_side, max_side);
    q.r0 = uniform_int(r.z, 0, rows - q.h > 0 ? rows - q.h : 0);
    q.c0 = uniform_int(r.w, 0, cols - q.w > 0 ? cols - q.w : 0);
    out[i] = q;
}

// One CTA per rectangle: first[cell] = min(first[cell], rectangle index).
__global__ void rasterize_rects_kernel(const Rect* rects, int n, int rows, int cols, int* first) {
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        const Rect q = rects[i];
        const int r1 = min(q.r0 + q.h, rows), c1 = min(q.c0 + q.w, cols);
        const int w = c1 - q.c0;
        const int cells = (r1 - q.r0) * w;
        for (int t = threadIdx.x; t < cells; t += blockDim.x) {
            const int r = q.r0 + t / w, c = q.c0 + t % w;
            atomicMin(&first[(int64_t)r * cols + c], i);
        }
    }
}

// Cells newly covered by each rectangle.
__global__ void first_histogram_kernel(const int* first, int64_t n_cells, int n_rects, int* counts) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_cells; i += (int64_t)gridDim.x * blockDim.x) {
        const int f = first[i];
        if (f < n_rects) atomicAdd(&counts[f], 1);
    }
}

// Bed and Manning fields from the block mask: a plane falling toward +x
// (slope * (cols*dx - x), x at the cell centre) plus the block raise or the
// street offset, in float64 and rounded once to float32; Manning n of the
// block or the street times n_scale, likewise.
__global__ void urban_fields_kernel(const int* first, int n_blocks, int rows, int cols, double dx, double slope,
                                    double raise, double street, double n_block, double n_street, double n_scale,
                                    float* bed, float* manning, uint8_t* mask) {
    const int64_t total = (int64_t)rows * cols;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % cols);
        const bool block = first[i] < n_blocks;
        const double x = __dmul_rn(__dadd_rn((double)c, 0.5), dx);
        const double plane = __dmul_rn(slope, __dsub_rn(__dmul_rn((double)cols, dx), x));
        bed[i] = __double2float_rn(__dadd_rn(plane, block ? raise : street));
        manning[i] = __double2float_rn(__dmul_rn(block ? n_block : n_street, n_scale));
        if (mask) mask[i] = block ? 1 : 0;
    }
}

// ---------------------------------------------------------------------------
// Gamma hyetograph
// ---------------------------------------------------------------------------
// Gamma(k, 1) by Marsaglia and Tsang ("A simple method for generating gamma
// variables", ACM TOMS 26(3), 2000): for k >= 1, d = k - 1/3, c = 1/sqrt(9d),
// accept v = (1 + c z)^3 when log u < z^2/2 + d - d v + d log v; for k < 1 a
// Gamma(k + 1) variate is scaled by u^(1/k).  Each attempt uses fresh draws of
// the value's own stream, at most 64 attempts (the acceptance rate is above
// 0.95 for every k).
__device__ inline double gamma_variate(uint64_t seed, uint32_t stream, uint64_t value, double k) {
    const bool boost = k < 1.0;
    const double a = boost ? k + 1.0 : k;
    const double d = a - 1.0 / 3.0;
    const double c = 1.0 / sqrt(9.0 * d);
    double g = d;  // the mode, should every attempt be rejected
    for (int attempt = 0; attempt < 64; ++attempt) {
        const U4 r0 = draw(seed, stream, value * 128u + 2u * (uint64_t)attempt);
        const U4 r1 = draw(seed, stream, value * 128u + 2u * (uint64_t)attempt + 1u);
        const double z = normal2(r0.x, r0.y, r0.z, r0.w).x;
        const double t = 1.0 + c * z;
        if (t <= 0.0) continue;
        const double v = t * t * t;
        const double u = u01(r1.x, r1.y);
        if (log(u) < 0.5 * z * z + d - d * v + d * log(v)) {
            g = d * v;
            break;
        }
    }
    if (boost) {
        const U4 rb = draw(seed, stream ^ 0x5bd1e995u, value);
        g *= pow(u01(rb.x, rb.y), 1.0 / k);
    }
    return g;
}

// n values one step_s apart: times i*step_s, rates Gamma(k, theta) * to_m_s,
// both rounded to float32.
__global__ void gamma_hyetograph_kernel(uint64_t seed, int n, double step_s, double k, double theta,
                                        double to_m_s, float* times, float* rates) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    times[i] = __double2float_rn((double)i * step_s);
    rates[i] = __double2float_rn(gamma_variate(seed, 2u, (uint64_t)i, k) * theta * to_m_s);
}

// ---------------------------------------------------------------------------
// Smoothed log-normal field
// ---------------------------------------------------------------------------
// Standard normal noise per cell (float64).
__global__ void normal_field_kernel(uint64_t seed, int64_t n, double* out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const U4 r = draw(seed, 3u, (uint64_t)i);
        out[i] = normal2(r.x, r.y, r.z, r.w).x;
    }
}

// Index of `i` reflected into [0, n) without repeating the edge (NumPy's
// "reflect" padding: -1 -> 1, n -> n - 2).
__device__ __forceinline__ int reflect_index(int i, int n) {
    if (n == 1) return 0;
    const int period = 2 * (n - 1);
    i %= period;
    if (i < 0) i += period;
    return i < n ? i : period - i;
}

// One pass of the separable Gaussian (taps[0 .. 2*radius]) along rows (axis 1)
// or columns (axis 0), reflect-padded, in float64 with the taps applied in
// order from the lowest index.  A 2-D grid (x: columns, y: rows, both
// grid-strided) gives every thread its row and column without a division, and
// only cells within `radius` of an edge take the reflected indices.
template <int AXIS>
__global__ void smooth_pass_kernel(const double* in, double* out, int rows, int cols, const double* taps, int radius) {
    for (int r = blockIdx.y; r < rows; r += gridDim.y) {
        const double* row = in + (int64_t)r * cols;
        for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < cols; c += gridDim.x * blockDim.x) {
            double acc = 0.0;
            if (AXIS == 1) {
                if (c >= radius && c + radius < cols) {
                    for (int t = -radius; t <= radius; ++t) acc = __fma_rn(row[c + t], taps[t + radius], acc);
                } else {
                    for (int t = -radius; t <= radius; ++t)
                        acc = __fma_rn(row[reflect_index(c + t, cols)], taps[t + radius], acc);
                }
            } else {
                if (r >= radius && r + radius < rows) {
                    const double* p = in + (int64_t)(r - radius) * cols + c;
                    for (int t = 0; t <= 2 * radius; ++t) acc = __fma_rn(p[(int64_t)t * cols], taps[t], acc);
                } else {
                    for (int t = -radius; t <= radius; ++t)
                        acc = __fma_rn(in[(int64_t)reflect_index(r + t, rows) * cols + c], taps[t + radius], acc);
                }
            }
            out[(int64_t)r * cols + c] = acc;
        }
    }
}

// Deterministic float64 sums (a fixed grid, a fixed reduction tree and an
// in-order fold, so the generated fields are the same on every run):
// partials[b] = sum over block b's cells of x, or of (x - mean)^2 when `mean`
// is given; fold_sums_kernel adds the partials in order into *out.
constexpr int kGenSumBlocks = 512;

template <int THREADS>
__global__ void __launch_bounds__(THREADS) block_sums_kernel(const double* x, int64_t n, const double* mean,
                                                            double* partials) {
    __shared__ double s_w[THREADS / 32];
    const double m = mean ? *mean / (double)n : 0.0;
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * THREADS) {
        const double v = mean ? (x[i] - m) * (x[i] - m) : x[i];
        s += v;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < THREADS / 32; ++w) b += s_w[w];
        partials[blockIdx.x] = b;
    }
}

__global__ void fold_sums_kernel(const double* partials, int nb, double* out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < nb; ++b) s += partials[b];
        *out = s;
    }
}

// out = float32(median * exp(sigma_log * x / std(x))), std with divisor n
// (sums[1] = sum of squared deviations from the mean).
__global__ void lognormal_finish_kernel(const double* x, int64_t n, const double* sums, double median,
                                        double sigma_log, float* out) {
    const double var = sums[1] / (double)n;
    const double sd = var > 0.0 ? sqrt(var) : 1.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = __double2float_rn(median * exp(sigma_log * (x[i] / sd)));
}

}  // namespace swe
