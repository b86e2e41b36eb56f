// Fused shallow-water step kernels for sm_100a.
//
// One step of the reference finite-volume scheme
// (src/hybrid_flood/numpy_solver/shallow_water_2d.py:277-327, the same
// arithmetic as src/hybrid_flood/jax_solver/numerics.py:312-369) in ONE kernel:
// ghost ring, wall mirroring, hydrostatic reconstruction, HLL x/y fluxes,
// divergence, rain source, positivity clip, semi-implicit Manning friction,
// wet/dry masking -- and, in run mode, the CFL inverse-dt reduction of the NEW
// state (numerics.py:297-309) plus FP64 mass-ledger sums.  A run step plans
// itself: each warp reads the run position (FP64 clock, next output) and the
// previous step's CFL maximum and computes the same dt, one warp per run
// publishes the advanced position, and each warp ends with an atomic maximum
// and its own ledger slot, so no warp waits for another.
//
// Work decomposition ("column marching"): a warp owns a strip of 32*V columns
// (V consecutive columns per lane, loaded as float2/float4) and marches up a
// chunk of rows.  Every x-face and y-face inside the strip is evaluated once:
// the y-face above row r is carried in registers to row r+1, x-faces between
// lanes travel by warp shuffle.  Only the chunk's bottom y-face row and the
// strip's left x-face column are evaluated twice (once by each neighbour).
// No shared memory and no block-wide barrier is needed inside the march.
//
// HBM traffic per cell-update: h, hu, hv, bed and n^2 (with the domain mask in
// the sign bit of n^2) read once = 20 B, h, hu, hv written once = 12 B.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "swe_math.cuh"

namespace swe {

constexpr int kWarp = 32;

// Float32 constants of the step, rounded from the float64 controls exactly where
// NumPy's weak-scalar rule rounds them in the reference.
struct Consts {
    float g;       // float(g)
    float half_g;  // float(0.5 * g)
    float dry;     // float(dry_tolerance)
    float dx, dy;  // float(dx), float(dy)
    float eps;     // float(1e-12)   HLL denominator guard
    float expo;    // float(7/3)     Manning exponent
    int pow2;      // 1: dx and dy are powers of two, so x / dx == x * (1 / dx) exactly
};

// Per-step float32 scalars: float(dt), float(dt*rate), float(dt*g).
struct StepScalars {
    float dt, dt_rain, dt_g;
};

struct DomainDev {
    int rows, cols;
    int64_t spitch;      // pitch (elements) of the static planes
    const float* bed;    // rows x spitch
    const float* nm;     // n^2 with sign bit set on inactive cells
    const float* mult;   // rain multiplier plane, or nullptr (= domain mask)
    int bnd[4];          // left, right, bottom, top: 0 reflective, 1 open
    Consts k;
    double dx, dy, g, cfl, max_dt, default_rain;
    const double* rain_t;  // hyetograph times (s), float64 copies of the float32 table
    const double* rain_r;  // rates (m/s)
    int n_rain;
    double rain_x0, rain_xn, rain_yn;  // first and last time of the hyetograph, last rate
    double rain_scale;     // multiplies every rate (1 = the hyetograph as given)
    // Rows the step updates and the reductions cover: [upd_lo, upd_hi).  A row
    // strip of a decomposed domain also holds its neighbours' boundary rows
    // (halo rows) outside that range: read as ordinary neighbours, never updated.
    int upd_lo, upd_hi;
    // Strip-boundary columns of the state, kept by the plain run-mode step for
    // the next step's strip edges (null: not kept; the edges are then loaded
    // from the state).  For boundary b (between the kEdgeStrip-column strips
    // b-1 and b) edge[p] holds h, hu, hv of its left cell (column
    // kEdgeStrip*b - 1) and of its right cell (column kEdgeStrip*b) of the
    // state in ping-pong buffer p, and edge_static the bed and n^2 of the same
    // cells: one run of edge_rows floats per boundary, quantity and cell side,
    // rows contiguous, so that a warp reads 32 rows of an edge in one access.
    float* edge[2];
    const float* edge_static;
    int edge_rows;
};

constexpr int kEdgeStrip = 64;  // columns of a warp strip of the paired march (32 lanes x 2 cells)

// Index of row r of quantity q of boundary b: q = 0..2 h, hu, hv of the left
// cell, 3..5 of the right cell (edge); q = 0, 1 bed and n^2 of the left cell,
// 2, 3 of the right cell (edge_static).
__host__ __device__ __forceinline__ int64_t edge_index(const DomainDev& d, int b, int q, int r) {
    return ((int64_t)b * 6 + q) * d.edge_rows + r;
}
__host__ __device__ __forceinline__ int64_t edge_static_index(const DomainDev& d, int b, int q, int r) {
    return ((int64_t)b * 4 + q) * d.edge_rows + r;
}

struct StateView {
    const float* h;
    const float* hu;
    const float* hv;
    int64_t pitch;
};

struct StateOut {
    float* h;
    float* hu;
    float* hv;
    int64_t pitch;
};

// Hyetograph segment [x0, x1) with its rates at both ends, kept between steps
// (lo = -1: none yet).
struct RainSeg {
    double x0, y0, x1, y1;
    double slope;  // (y1 - y0) / (x1 - x0), rounded as np.interp rounds it
    int lo;
};

// The run's position at the start of a step.  There is one copy per step
// parity: step k plans itself from copy k&1, and its lead warp writes copy
// (k+1)&1, so a step never writes what its own warps read.
struct alignas(16) RunPos {
    double t;       // simulated time at the start of the step
    double target;  // output time `idx` in float64 (valid while idx < n_out)
    RainSeg rain;   // the segment of the previous step's rain rate
    int steps;      // steps taken
    int idx;        // next output index to fill
    int done;       // nonzero: all outputs written, step cap reached or failure
    int status;     // 0 ok, else an SWE_ERR_* code
};

// CFL maxima of the steps: per step parity, kMaxStripes words 128 bytes apart,
// each the atomic maximum of (steps of the state << 32 | float bits of its
// largest inverse dt) over the warps that chose it.  The step count in the
// high word makes a newer step's value beat whatever an older step left, so
// the words are never cleared during a run.
constexpr int kMaxStripes = 16;
constexpr int kStripeWords = 16;

// Device-resident run control: output bookkeeping, ledger, the run position
// of each step parity and the CFL maxima.  The fields up to `pos` are the
// host's view, published by the lead warp of every step (and by the run's
// start reduction).
struct Control {
    double t;          // simulated time reached
    double dt;         // dt of the last step taken
    int idx;           // next output index to fill
    int steps;         // steps taken
    int done;          // nonzero: all outputs written, step cap hit or failure
    int status;        // 0 ok, else an SWE_ERR_* code
    float maxinv;      // max inverse CFL dt: of the initial state, or across the strips of a domain
    unsigned counter;  // last-CTA ticket of the start reduction
    int n_out, max_steps;
    double t_start;               // clock value set by the start reduction
    const float* times;           // device copy of the float32 output times
    const double* times64;        // float64 targets instead of `times` (advance_to), or null
    unsigned* done_counter;       // incremented once when this run finishes (ensembles), or null
    double* dt_log;               // dt of every step (index = step number), or null
    float* out_h;                 // n_out x rows x cols snapshots (may be null)
    float* out_hu;
    float* out_hv;
    int64_t out_plane;            // rows * cols
    double ledger[6];             // volume0, volume, rain_in, outflow, clip_gain, mask_loss
    int defer_plan;               // 1: steps plan from `maxinv` (set across strips), not from the stripes
    RunPos pos[2];
    alignas(128) unsigned long long maxk[2][kMaxStripes * kStripeWords];
};

// Bytes of the control block the host reads back (everything before the maxima).
constexpr size_t kControlHead = offsetof(Control, maxk);

// The strip-boundary columns of state `s` into `edge` and, when `stat` is not
// null, of the bed and n^2 into `stat` (the layouts of DomainDev::edge and
// edge_static).  Grid: x over the rows, y over the boundaries.  Cells outside
// the grid (left of boundary 0, right of the last) are left as they are.
__global__ void edge_fill_kernel(const DomainDev d, const StateView s, float* edge, float* stat) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y;
    if (r >= d.rows) return;
    for (int side = 0; side < 2; ++side) {
        const int x = kEdgeStrip * b - 1 + side;
        if (x < 0 || x >= d.cols) continue;
        if (edge) {
            const int64_t so = (int64_t)r * s.pitch + x;
            edge[edge_index(d, b, 3 * side + 0, r)] = s.h[so];
            edge[edge_index(d, b, 3 * side + 1, r)] = s.hu[so];
            edge[edge_index(d, b, 3 * side + 2, r)] = s.hv[so];
        }
        if (stat) {
            const int64_t zo = (int64_t)r * d.spitch + x;
            stat[edge_static_index(d, b, 2 * side + 0, r)] = d.bed[zo];
            stat[edge_static_index(d, b, 2 * side + 1, r)] = d.nm[zo];
        }
    }
}

// A run's control block written from launch parameters: the head as the host
// built it, the stripe maxima zeroed and up to two target times.  Parameters
// are captured when the launch is queued, so the host needs no staging buffer,
// and the queue never waits for the stream as a copy from pageable host memory
// may.
struct ControlHeadImage {
    unsigned long long w[kControlHead / 8];
};
static_assert(kControlHead % 8 == 0 && sizeof(ControlHeadImage) <= 2048, "control head must fit the launch parameters");

constexpr int kInlineTimes = 64;  // output times carried in the launch parameters

struct RunTargets {
    int n;              // entries of t (and of t64, at most 2, when times64 is set) written
    float t[kInlineTimes];
    double t64[2];
    float* times;       // device arrays receiving them (times64 may be null)
    double* times64;
};

__global__ void control_init_kernel(Control* ctl, const ControlHeadImage head, const RunTargets tg) {
    auto* dst = reinterpret_cast<unsigned long long*>(ctl);
    for (int i = threadIdx.x; i < (int)(kControlHead / 8); i += blockDim.x) dst[i] = head.w[i];
    unsigned long long* mk = &ctl->maxk[0][0];
    for (int i = threadIdx.x; i < 2 * kMaxStripes * kStripeWords; i += blockDim.x) mk[i] = 0ull;
    if ((int)threadIdx.x < tg.n) {
        tg.times[threadIdx.x] = tg.t[threadIdx.x];
        if (tg.times64 && threadIdx.x < 2) tg.times64[threadIdx.x] = tg.t64[threadIdx.x];
    }
}

struct Partial {
    float maxinv;
    double vol, rain, outflow, clip, mask;
};

// A warp's ledger slot of a run: its cells' volume after the last step, and
// the rain, outflow, clip and mask terms summed over the run's steps.  The
// first four words are read back at the start of each step (two 16-byte
// copies), so the slot is 16-byte aligned.
struct alignas(16) LedgerSlot {
    double rain, outflow, clip, mask, vol, pad;
};

// ---------------------------------------------------------------------------
// Cells
// ---------------------------------------------------------------------------
struct Cell {
    float h, hu, hv, z, nm;  // nm: n^2, negative (sign bit) = inactive
    float u, v;              // cell velocities (unreconstructed depth)
};

__device__ __forceinline__ bool active(float nm) { return !signbit(nm); }

template <class M>
__device__ __forceinline__ void set_vel(Cell& c, float dry) {
    M::vel2(c.hu, c.hv, c.h, dry, c.u, c.v);
}

// Load V cells of row r starting at column c0 (r in [-1, rows], c0 in [-V, cols]),
// applying the ghost ring: clamp to the nearest interior cell, negate hu on
// reflective left/right ghosts and hv on reflective bottom/top ghosts.
template <int V>
__device__ __forceinline__ void load_cells(const DomainDev& d, const StateView& s, int r, int c0,
                                           Cell (&out)[V]) {
    const int rr = r < 0 ? 0 : (r >= d.rows ? d.rows - 1 : r);
    const bool flip_v = (r < 0 && d.bnd[2] == 0) || (r >= d.rows && d.bnd[3] == 0);
    const int64_t so = (int64_t)rr * s.pitch;
    const int64_t zo = (int64_t)rr * d.spitch;
    if (c0 >= 0 && c0 + V <= d.cols) {
        if constexpr (V == 4) {
            const float4 h = __ldg(reinterpret_cast<const float4*>(s.h + so + c0));
            const float4 hu = __ldg(reinterpret_cast<const float4*>(s.hu + so + c0));
            const float4 hv = __ldg(reinterpret_cast<const float4*>(s.hv + so + c0));
            const float4 z = __ldg(reinterpret_cast<const float4*>(d.bed + zo + c0));
            const float4 nm = __ldg(reinterpret_cast<const float4*>(d.nm + zo + c0));
            out[0] = {h.x, hu.x, hv.x, z.x, nm.x, 0.f, 0.f};
            out[1] = {h.y, hu.y, hv.y, z.y, nm.y, 0.f, 0.f};
            out[2] = {h.z, hu.z, hv.z, z.z, nm.z, 0.f, 0.f};
            out[3] = {h.w, hu.w, hv.w, z.w, nm.w, 0.f, 0.f};
        } else if constexpr (V == 2) {
            const float2 h = __ldg(reinterpret_cast<const float2*>(s.h + so + c0));
            const float2 hu = __ldg(reinterpret_cast<const float2*>(s.hu + so + c0));
            const float2 hv = __ldg(reinterpret_cast<const float2*>(s.hv + so + c0));
            const float2 z = __ldg(reinterpret_cast<const float2*>(d.bed + zo + c0));
            const float2 nm = __ldg(reinterpret_cast<const float2*>(d.nm + zo + c0));
            out[0] = {h.x, hu.x, hv.x, z.x, nm.x, 0.f, 0.f};
            out[1] = {h.y, hu.y, hv.y, z.y, nm.y, 0.f, 0.f};
        } else {
#pragma unroll
            for (int i = 0; i < V; ++i) {
                out[i] = {__ldg(s.h + so + c0 + i), __ldg(s.hu + so + c0 + i),
                          __ldg(s.hv + so + c0 + i), __ldg(d.bed + zo + c0 + i),
                          __ldg(d.nm + zo + c0 + i), 0.f, 0.f};
            }
        }
#pragma unroll
        for (int i = 0; i < V; ++i)
            if (flip_v) out[i].hv = -out[i].hv;
    } else {
#pragma unroll
        for (int i = 0; i < V; ++i) {
            const int c = c0 + i;
            const int cc = c < 0 ? 0 : (c >= d.cols ? d.cols - 1 : c);
            Cell x = {__ldg(s.h + so + cc), __ldg(s.hu + so + cc), __ldg(s.hv + so + cc),
                      __ldg(d.bed + zo + cc), __ldg(d.nm + zo + cc), 0.f, 0.f};
            if ((c < 0 && d.bnd[0] == 0) || (c >= d.cols && d.bnd[1] == 0)) x.hu = -x.hu;
            if (flip_v) x.hv = -x.hv;
            out[i] = x;
        }
    }
}

// ---------------------------------------------------------------------------
// Faces
// ---------------------------------------------------------------------------
// Flux through one face plus the two side-specific pressure corrections
// (shallow_water_2d.py:138-239).  The lower-index cell sees F + corr_lo on the
// normal-momentum component, the higher-index cell F + corr_hi.
struct FaceFlux {
    float f0, f1, f2;
    float corr_lo, corr_hi;
};

// AXIS 1: x-face (normal momentum hu), AXIS 0: y-face (normal momentum hv).
template <int AXIS, class M, bool MASKED = true>
__device__ __forceinline__ FaceFlux face_flux(const Cell& lo, const Cell& hi, const Consts& k) {
    // Without a domain mask every cell is active: no walls, every face relevant.
    const bool a_lo = MASKED ? active(lo.nm) : true, a_hi = MASKED ? active(hi.nm) : true;
    const bool relevant = a_lo | a_hi;
    const bool hi_wall = a_lo & !a_hi;  // mirror lo onto hi
    const bool lo_wall = !a_lo & a_hi;  // mirror hi onto lo
    // Mirrored states: the normal-momentum velocity changes sign, the rest is copied.
    const float hL = lo_wall ? hi.h : lo.h;
    const float zL = lo_wall ? hi.z : lo.z;
    const float hR = hi_wall ? lo.h : hi.h;
    const float zR = hi_wall ? lo.z : hi.z;
    float uL, vL, uR, vR;
    if (AXIS == 1) {
        uL = lo_wall ? -hi.u : lo.u;
        vL = lo_wall ? hi.v : lo.v;
        uR = hi_wall ? -lo.u : hi.u;
        vR = hi_wall ? lo.v : hi.v;
    } else {
        uL = lo_wall ? hi.u : lo.u;
        vL = lo_wall ? -hi.v : lo.v;
        uR = hi_wall ? lo.u : hi.u;
        vR = hi_wall ? -lo.v : hi.v;
    }
    // Hydrostatic reconstruction.
    const float zf = fmaxf(zL, zR);
    const float HL = fmaxf(M::sub(M::add(hL, zL), zf), 0.0f);
    const float HR = fmaxf(M::sub(M::add(hR, zR), zf), 0.0f);
    const float XL = M::mul(HL, uL), YL = M::mul(HL, vL);
    const float XR = M::mul(HR, uR), YR = M::mul(HR, vR);
    // HLL (shallow_water_2d.py:66-135) on the reconstructed states.
    const float unL = AXIS == 1 ? M::recon_vel(XL, HL, k.dry, uL) : M::recon_vel(YL, HL, k.dry, vL);
    const float unR = AXIS == 1 ? M::recon_vel(XR, HR, k.dry, uR) : M::recon_vel(YR, HR, k.dry, vR);
    const float cL = M::sqrt(M::mul(k.g, HL));
    const float cR = M::sqrt(M::mul(k.g, HR));
    const float sL = fminf(M::sub(unL, cL), M::sub(unR, cR));
    const float sR = fmaxf(M::add(unL, cL), M::add(unR, cR));
    const float pL = M::mul(k.half_g, M::mul(HL, HL));
    const float pR = M::mul(k.half_g, M::mul(HR, HR));
    float fL0, fL1, fL2, fR0, fR1, fR2;
    if (AXIS == 1) {
        fL0 = XL;
        fL1 = M::add(M::mul(XL, unL), pL);
        fL2 = M::mul(XL, M::recon_vel(YL, HL, k.dry, vL));
        fR0 = XR;
        fR1 = M::add(M::mul(XR, unR), pR);
        fR2 = M::mul(XR, M::recon_vel(YR, HR, k.dry, vR));
    } else {
        fL0 = YL;
        fL1 = M::mul(XL, unL);
        fL2 = M::add(M::mul(YL, unL), pL);
        fR0 = YR;
        fR1 = M::mul(XR, unR);
        fR2 = M::add(M::mul(YR, unR), pR);
    }
    const float spread = M::sub(sR, sL);
    const float den = spread > k.eps ? spread : 1.0f;
    const float rden = M::recip(den);
    const float s01 = M::mul(sL, sR);
    const float m0 = M::over(M::add(M::sub(M::mul(sR, fL0), M::mul(sL, fR0)), M::mul(s01, M::sub(HR, HL))), rden);
    const float m1 = M::over(M::add(M::sub(M::mul(sR, fL1), M::mul(sL, fR1)), M::mul(s01, M::sub(XR, XL))), rden);
    const float m2 = M::over(M::add(M::sub(M::mul(sR, fL2), M::mul(sL, fR2)), M::mul(s01, M::sub(YR, YL))), rden);
    const bool take_l = sL >= 0.0f, take_r = sR <= 0.0f;
    FaceFlux f;
    f.f0 = relevant ? (take_l ? fL0 : (take_r ? fR0 : m0)) : 0.0f;
    f.f1 = relevant ? (take_l ? fL1 : (take_r ? fR1 : m1)) : 0.0f;
    f.f2 = relevant ? (take_l ? fL2 : (take_r ? fR2 : m2)) : 0.0f;
    f.corr_lo = relevant ? M::mul(k.half_g, M::sub(M::mul(hL, hL), M::mul(HL, HL))) : 0.0f;
    f.corr_hi = relevant ? M::mul(k.half_g, M::sub(M::mul(hR, hR), M::mul(HR, HR))) : 0.0f;
    return f;
}

// ---------------------------------------------------------------------------
// Run-mode helpers
// ---------------------------------------------------------------------------
// np.interp(t, times, rates, left=default, right=default) in float64 with
// separately rounded operations (shallow_water_2d.py:254-264).
// The segment containing t comes from `sg` when the cached one contains it
// (x0 <= t < x1): a run's clock only advances, so a step's segment is nearly
// always the previous step's, and the cache then replaces every load of the
// table.  Otherwise it is found by binary search and `sg` is updated.  For a
// sorted table the non-empty segment containing t is unique, so both ways
// give the same segment and the same value.
__device__ inline double rain_rate_unscaled(const DomainDev& d, double t, RainSeg& sg) {
    const int n = d.n_rain;
    if (n <= 0) return d.default_rain;
    if (t != t) return t;
    if (t < d.rain_x0 || t > d.rain_xn) return d.default_rain;
    if (n == 1 || t == d.rain_xn) return d.rain_yn;
    if (!(sg.lo >= 0 && sg.x0 <= t && t < sg.x1)) {
        int lo = 0, hi = n - 1;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (d.rain_t[mid] <= t) lo = mid; else hi = mid;
        }
        sg.lo = lo;
        sg.x0 = d.rain_t[lo];
        sg.y0 = d.rain_r[lo];
        sg.x1 = d.rain_t[lo + 1];
        sg.y1 = d.rain_r[lo + 1];
        sg.slope = __ddiv_rn(__dsub_rn(sg.y1, sg.y0), __dsub_rn(sg.x1, sg.x0));
    }
    const double xj = sg.x0, yj = sg.y0, xj1 = sg.x1, yj1 = sg.y1, slope = sg.slope;
    if (t == xj) return yj;
    double v = __dadd_rn(__dmul_rn(slope, __dsub_rn(t, xj)), yj);
    if (v != v) {
        v = __dadd_rn(__dmul_rn(slope, __dsub_rn(t, xj1)), yj1);
        if (v != v && yj == yj1) v = yj;
    }
    return v;
}

// Float32 scalars of a step of length dt starting at t.
__device__ inline StepScalars step_scalars(const DomainDev& d, double dt, double t, RainSeg& sg) {
    StepScalars s;
    s.dt = __double2float_rn(dt);
    s.dt_rain = __double2float_rn(__dmul_rn(dt, __dmul_rn(d.rain_scale, rain_rate_unscaled(d, t, sg))));
    s.dt_g = __double2float_rn(__dmul_rn(dt, d.g));
    return s;
}

// CFL dt from the largest inverse dt (shallow_water_2d.py:274; in float64).
__device__ inline double cfl_dt_from(const DomainDev& d, float maxinv) {
    const double m = (double)maxinv;
    if (m > 0.0) {
        const double c = __ddiv_rn(d.cfl, m);
        return c < d.max_dt ? c : d.max_dt;
    }
    return d.max_dt;
}

// A step's plan, computed from its run position and the CFL maximum of the
// state it starts from (run loop of shallow_water_2d.py:402-412): dt =
// min(cfl_dt, target - t), the output is recorded when the new time reaches
// target - 1e-7, the run stops when all outputs are written, the step cap is
// reached or the maximum is not finite.
struct StepPlan {
    StepScalars s;
    double dt;
    RainSeg rain;  // the segment of this step's rain rate
    int go;        // 1: the step runs
    int status;    // the run's status (SWE_ERR_NONFINITE when it stops on a non-finite maximum)
    int reach;     // output index the new time reaches, -1 if none
    int snap;      // output index written by the step (reach, when outputs are recorded), -1 if none
};

// Everything a warp reads to plan a step: the run position of the step's
// parity, this lane's CFL maximum word, and the run's constants.
struct PlanInputs {
    RunPos pos;
    unsigned long long w;   // maximum word `lane` of the parity (lanes < kMaxStripes)
    float gmax;             // the maximum across strips (row strips of a decomposed domain)
    int defer, n_out, max_steps;
    const float* out_h;
    double* dt_log;
    unsigned* done_counter;
};

// Issues the loads of a step's plan (every lane).  They are plain loads: the
// previous step's writes are visible to this grid (a kernel boundary, or
// griddepcontrol.wait, which the kernel has passed, under programmatic
// launch), and a load that every warp of an SM makes is then merged in the
// SM's L1 instead of reaching one L2 slice from every warp of the grid.
// The values are consumed later (plan_step), so the caller can start other
// loads while these are in flight.
__device__ __forceinline__ PlanInputs plan_fetch(const Control* c, int par) {
    const int lane = threadIdx.x & 31;
    PlanInputs in;
    in.pos = c->pos[par];
    in.w = lane < kMaxStripes ? c->maxk[par][lane * kStripeWords] : 0ull;
    in.gmax = c->maxinv;
    in.defer = c->defer_plan;
    in.n_out = c->n_out;
    in.max_steps = c->max_steps;
    in.out_h = c->out_h;
    in.dt_log = c->dt_log;
    in.done_counter = c->done_counter;
    return in;
}

// The CFL maximum of the state with `steps` steps taken, from the words of
// one parity (word `lane` in `w` on lanes < kMaxStripes) that carry that step
// count; NaN when none does, which stops the run as non-finite.  Every lane
// of the warp returns it.
__device__ __forceinline__ float words_maxinv(unsigned long long w, int steps) {
    const bool mine = (threadIdx.x & 31) < kMaxStripes && (int)(w >> 32) == steps;
    const unsigned m = __reduce_max_sync(0xffffffffu, mine ? (unsigned)w : 0u);
    const bool found = __any_sync(0xffffffffu, mine);
    return found ? __uint_as_float(m) : __int_as_float(0x7fffffff);
}

// The plan from the fetched inputs (every lane, the same values): the maximum
// from the words, or, for a strip of a decomposed domain, across strips.
__device__ inline StepPlan plan_step(const DomainDev& d, const PlanInputs& in) {
    const RunPos& pos = in.pos;
    const float wmax = words_maxinv(in.w, pos.steps);
    const float maxinv = in.defer ? in.gmax : wmax;
    StepPlan p;
    p.go = 0;
    p.status = pos.status;
    p.reach = p.snap = -1;
    p.dt = 0.0;
    p.s = StepScalars{0.f, 0.f, 0.f};
    p.rain = pos.rain;
    if (pos.done || pos.idx >= in.n_out || pos.steps >= in.max_steps) return p;
    if (!(maxinv == maxinv) || isinf(maxinv)) {
        p.status = 4;  // SWE_ERR_NONFINITE
        return p;
    }
    double dt = cfl_dt_from(d, maxinv);
    const double remain = __dsub_rn(pos.target, pos.t);
    if (remain < dt) dt = remain;
    p.dt = dt;
    p.s = step_scalars(d, dt, pos.t, p.rain);
    p.reach = (__dadd_rn(pos.t, dt) >= __dsub_rn(pos.target, 1.0e-7)) ? pos.idx : -1;
    // Without output buffers (advance, advance_to) nothing is recorded.
    p.snap = in.out_h ? p.reach : -1;
    p.go = 1;
    return p;
}

// Float64 output time i of a run.
__device__ __forceinline__ double output_time(const Control* c, int i) {
    return c->times64 ? c->times64[i] : (double)c->times[i];
}

// Programmatic dependent launch: a step kernel launched with the programmatic
// stream-serialisation attribute may be scheduled while the previous step is
// still running.  It lets its own successor launch at once and then waits,
// before it reads or writes anything, until the previous grid has completed
// and its memory is visible (a hardware wait, not a spin).  Launched without
// the attribute both instructions do nothing.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// NaN-propagating max (np.max semantics).
__device__ __forceinline__ float nan_max(float a, float b) { return (b > a || b != b) ? b : a; }

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = nan_max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

struct Accum {
    float maxinv;
    double vol, rain, outflow, clip, mask;
    __device__ void zero() { maxinv = 0.f; vol = rain = outflow = clip = mask = 0.0; }
};

// Per-thread accumulators of the step kernel.  Without a rain-multiplier plane
// every active cell receives the same float32 increment, so the rain term is
// kept as a cell count and multiplied out once per thread.
// Every ledger term is summed in float64 from the first cell on (a float32
// partial over a warp's rows already costs ~1e-6 of the ledger); without a
// rain-multiplier plane the rain term is an exact count of active cells.
struct StepAccum {
    float maxinv;
    unsigned rain_cells;
    double vol, rain, outflow, clip, mask;
    __device__ void zero() {
        maxinv = 0.f;
        rain_cells = 0u;
        vol = rain = outflow = clip = mask = 0.0;
    }
};

// CTA-wide reduction of a thread's accumulators (fixed order) into the CTA's
// totals, valid on thread 0.
template <int THREADS>
__device__ __forceinline__ Partial cta_reduce(Accum acc) {
    constexpr int W = THREADS / kWarp;
    __shared__ float s_max[W];
    __shared__ double s_sum[5][W];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    acc.maxinv = warp_max(acc.maxinv);
    acc.vol = warp_sum(acc.vol);
    acc.rain = warp_sum(acc.rain);
    acc.outflow = warp_sum(acc.outflow);
    acc.clip = warp_sum(acc.clip);
    acc.mask = warp_sum(acc.mask);
    if (lane == 0) {
        s_max[warp] = acc.maxinv;
        s_sum[0][warp] = acc.vol;
        s_sum[1][warp] = acc.rain;
        s_sum[2][warp] = acc.outflow;
        s_sum[3][warp] = acc.clip;
        s_sum[4][warp] = acc.mask;
    }
    __syncthreads();
    Partial p{};
    if (threadIdx.x == 0) {
        p.maxinv = s_max[0];
        p.vol = s_sum[0][0]; p.rain = s_sum[1][0]; p.outflow = s_sum[2][0];
        p.clip = s_sum[3][0]; p.mask = s_sum[4][0];
        for (int w = 1; w < W; ++w) {
            p.maxinv = nan_max(p.maxinv, s_max[w]);
            p.vol += s_sum[0][w]; p.rain += s_sum[1][w]; p.outflow += s_sum[2][w];
            p.clip += s_sum[3][w]; p.mask += s_sum[4][w];
        }
    }
    __syncthreads();  // s_max / s_sum are free again
    return p;
}

// End of the reduction that starts a run (reduce_kernel): the CTA partials are
// folded by the last CTA to arrive, in a fixed order, into the initial volume
// and CFL maximum, and the run's first position is set: clock at t_start,
// output 0 taken as the initial state, the first target loaded, the maximum
// stored for step 0 (step count 0 in the high word of stripe 0).
//
// PER: partials a thread of the last CTA loads before folding them.
template <int THREADS, int PER = 8>
__device__ void finish_start(const DomainDev& d, Control* ctl, Partial* parts, Accum acc) {
    const int nparts = (int)(gridDim.x * gridDim.y);
    __shared__ bool s_last;
    const Partial p = cta_reduce<THREADS>(acc);
    if (threadIdx.x == 0) {
        parts[blockIdx.y * gridDim.x + blockIdx.x] = p;
        __threadfence();
        const unsigned ticket = atomicAdd(&ctl->counter, 1u);
        s_last = (ticket == (unsigned)nparts - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // Fixed-order fold of all CTA partials: thread t folds partials t, t+T, ...,
    // a batch of them loaded from the L2 (.cg: the other CTAs' writes are
    // visible there after the fence) with every load in flight at once.
    Accum a;
    a.zero();
    constexpr int kPer = PER;
    for (int base = threadIdx.x; base < nparts; base += kPer * THREADS) {
        Partial buf[kPer];
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            const int b = base + j * THREADS;
            if (b < nparts) {
                buf[j].maxinv = __ldcg(&parts[b].maxinv);
                buf[j].vol = __ldcg(&parts[b].vol);
            }
        }
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            if (base + j * THREADS < nparts) {
                a.maxinv = nan_max(a.maxinv, buf[j].maxinv);
                a.vol += buf[j].vol;
            }
        }
    }
    const Partial t = cta_reduce<THREADS>(a);
    if (threadIdx.x != 0) return;
    float mx = t.maxinv;
    // A NaN volume means a non-finite state somewhere: report it as a NaN CFL
    // maximum, the form plan_step tests.
    if (!(t.vol == t.vol)) mx = __int_as_float(0x7fffffff);
    const double area = d.dx * d.dy;
    const int n_out = ctl->n_out;
    RunPos p0;
    p0.t = ctl->t_start;
    p0.target = n_out > 1 ? output_time(ctl, 1) : 0.0;
    p0.rain = RainSeg{0.0, 0.0, 0.0, 0.0, 0.0, -1};
    p0.steps = 0;
    p0.idx = 1;
    p0.done = (1 >= n_out || ctl->max_steps <= 0) ? 1 : 0;
    p0.status = 0;
    ctl->pos[0] = p0;
    ctl->t = p0.t;
    ctl->dt = 0.0;
    ctl->idx = 1;
    ctl->steps = 0;
    ctl->done = p0.done;
    ctl->status = 0;
    ctl->ledger[0] = t.vol * area;
    ctl->ledger[1] = t.vol * area;
    ctl->ledger[2] = ctl->ledger[3] = ctl->ledger[4] = ctl->ledger[5] = 0.0;
    // A row strip plans from the maximum across strips: NaN is kept as +inf
    // there, so that a maximum carries it.
    ctl->maxinv = (ctl->defer_plan && !(mx == mx)) ? INFINITY : mx;
    ctl->maxk[0][0] = (unsigned long long)(__float_as_uint(mx) & 0x7fffffffu);
    ctl->counter = 0;
    if (p0.done && ctl->done_counter) atomicAdd(ctl->done_counter, 1u);
    __threadfence();
}

// The CFL maximum of the state with `steps` steps taken, from the words of
// parity `par` (one load per lane).
__device__ __forceinline__ float stripes_maxinv(const Control* c, int par, int steps) {
    const int lane = threadIdx.x & 31;
    return words_maxinv(lane < kMaxStripes ? c->maxk[par][lane * kStripeWords] : 0ull, steps);
}

// Start of a step in a warp, with nothing to overlap: its run position
// (parity `par`) and its plan, the same on every lane.
__device__ __forceinline__ StepPlan warp_plan(const DomainDev& d, const Control* c, int par, PlanInputs& in) {
    in = plan_fetch(c, par);
    return plan_step(d, in);
}

// The lead warp of a run (one per run and step) advances the run position into
// the other parity's copy and publishes it: clock, step count, next output,
// completion (set as soon as the last output is written or the step cap is
// reached, so the host sees it after the step that ends the run), the dt log
// and an ensemble's completion counter.  A finished run's position is copied
// forward unchanged, so every later step of either parity sees it finished.
// Stores only, except the time of the next output when the step records one.
__device__ __forceinline__ void lead_advance(Control* c, int par, const PlanInputs& in, const StepPlan& p) {
    if ((threadIdx.x & 31) != 0) return;
    const RunPos& pos = in.pos;
    RunPos q = pos;
    int newly_done = 0;
    if (!pos.done) {
        if (!p.go) {
            q.done = 1;
            q.status = p.status;
            newly_done = 1;
        } else {
            q.t = __dadd_rn(pos.t, p.dt);
            q.steps = pos.steps + 1;
            q.rain = p.rain;
            if (p.reach >= 0) {
                q.idx = p.reach + 1;
                if (q.idx < in.n_out) q.target = output_time(c, q.idx);
            }
            q.done = (q.idx >= in.n_out || q.steps >= in.max_steps) ? 1 : 0;
            newly_done = q.done;
            if (in.dt_log) in.dt_log[pos.steps] = p.dt;  // steps < max_steps while not done
            c->dt = p.dt;
        }
    }
    c->pos[par ^ 1] = q;
    c->t = q.t;
    c->idx = q.idx;
    c->steps = q.steps;
    c->done = q.done;
    c->status = q.status;
    if (newly_done && in.done_counter) atomicAdd(in.done_counter, 1u);
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// 16-byte asynchronous copy global -> shared (both addresses 16-byte aligned).
__device__ __forceinline__ void cp_async_16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}

// Starts the copy of the warp's ledger slot (rain, outflow, clip, mask summed
// so far) into `old` (4 doubles of the warp's shared memory, 16-byte aligned):
// lanes 0 and 1 copy 16 bytes each.  The caller commits the group.
__device__ __forceinline__ void ledger_prefetch(const LedgerSlot* slot, double* old) {
    const int lane = threadIdx.x & 31;
    if (lane < 2) cp_async_16(old + 2 * lane, &slot->rain + 2 * lane);
}

// End of a step in a warp, once the prefetched slot has landed: the warp's
// ledger terms (fixed-order butterfly sums) go into its slot, the volume
// replaced and the other terms added to the run's sums, and its CFL maximum
// into stripe `stripe` of the next parity, tagged with the step count of the
// new state.  A NaN volume (a non-finite state in the warp's cells) counts as
// a NaN maximum, which beats every finite bit pattern.  Nothing here waits:
// the stores and the atomic maximum are complete when the grid is.
__device__ __forceinline__ void warp_end_step(Control* c, LedgerSlot* slot, const double* old, int par, int steps,
                                              int stripe, Accum a) {
    const double vol = warp_sum(a.vol);
    const double rain = warp_sum(a.rain);
    const double outflow = warp_sum(a.outflow);
    const double clip = warp_sum(a.clip);
    const double mask = warp_sum(a.mask);
    unsigned m = __reduce_max_sync(0xffffffffu, __float_as_uint(a.maxinv) & 0x7fffffffu);
    if (!(vol == vol)) m = 0x7fc00000u;
    if ((threadIdx.x & 31) != 0) return;
    slot->vol = vol;
    slot->rain = old[0] + rain;
    slot->outflow = old[1] + outflow;
    slot->clip = old[2] + clip;
    slot->mask = old[3] + mask;
    atomicMax(&c->maxk[par ^ 1][stripe * kStripeWords], ((unsigned long long)(steps + 1) << 32) | m);
}

// The run's ledger from the warps' slots (one CTA, fixed order): the stored
// volume of the last step and the rain, outflow, clip and mask terms summed over
// the run.  With no step taken the volume stays the initial one.
template <int THREADS>
__global__ void __launch_bounds__(THREADS) ledger_fold_kernel(const DomainDev d, Control* ctl, const LedgerSlot* slots,
                                                             int nslots) {
    Accum a;
    a.zero();
    for (int b = threadIdx.x; b < nslots; b += THREADS) {
        a.vol += slots[b].vol; a.rain += slots[b].rain; a.outflow += slots[b].outflow;
        a.clip += slots[b].clip; a.mask += slots[b].mask;
    }
    const Partial t = cta_reduce<THREADS>(a);
    if (threadIdx.x != 0) return;
    const double area = d.dx * d.dy;
    ctl->ledger[1] = ctl->steps > 0 ? t.vol * area : ctl->ledger[0];
    ctl->ledger[2] = t.rain * area;
    ctl->ledger[3] = t.outflow;
    ctl->ledger[4] = t.clip * area;
    ctl->ledger[5] = t.mask * area;
}

// A row strip's CFL maximum after its step, from the stripes of the step's
// parity, into ctl->maxinv (NaN as +inf), for the maximum across strips that
// the next step plans from.  One warp.
__global__ void stripe_fold_kernel(Control* ctl) {
    const int steps = __ldcg(&ctl->steps);
    const float m = stripes_maxinv(ctl, steps & 1, steps);
    if (threadIdx.x == 0) ctl->maxinv = (m == m) ? m : INFINITY;
}

// ---------------------------------------------------------------------------
// The step kernel
// ---------------------------------------------------------------------------
struct StepLaunch {
    DomainDev d;
    StateView in;
    StateOut out;
    StepScalars s;     // used when ctl == nullptr (plain step)
    Control* ctl;      // run mode when non-null
    LedgerSlot* slots; // run mode: one ledger slot per warp of the launch
    int par;           // run mode: parity of the step (k & 1 for the run's step k)
    int nstrips;       // ceil(cols / (32 V))
    int rows_per_warp;
};

// Resident CTAs per SM the register budget is capped for (V=2: 128 registers).
#ifndef SWE_MINBLOCKS_V2
#define SWE_MINBLOCKS_V2 4
#endif
template <int V>
struct MinBlocks {
    static constexpr int value = V == 1 ? 4 : (V == 2 ? SWE_MINBLOCKS_V2 : 2);
};

template <int V, class M, int THREADS, bool RUN, bool MASKED>
__global__ void __launch_bounds__(THREADS, MinBlocks<V>::value) step_kernel(const StepLaunch p) {
    constexpr int NW = THREADS / kWarp;
    constexpr int kBatch = kWarp;  // strip-edge work is done for 32 rows at a time
    // Warp-private staging of the strip edges for the current batch of rows:
    // hi side of the strip's left x-face, and the cell right of the strip.
    __shared__ float s_left[NW][3][kBatch];
    __shared__ float s_right[NW][7][kBatch];

    __shared__ alignas(16) double s_old[NW][4];  // the warp's ledger slot as the step found it

    pdl_enter();
    const DomainDev& d = p.d;
    const Consts& k = d.k;
    constexpr bool run = RUN;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int gw = blockIdx.x * NW + wib;
    StepScalars s = p.s;
    int snap = -1;
    double dtd = 0.0;
    int steps0 = 0;
    if constexpr (RUN) {
        ledger_prefetch(&p.slots[gw], s_old[wib]);
        cp_async_commit();
        PlanInputs in;
        const StepPlan pl = warp_plan(d, p.ctl, p.par, in);
        if (blockIdx.x == 0 && wib == 0) lead_advance(p.ctl, p.par, in, pl);
        if (!pl.go) {  // uniform over the grid: the run has ended
            cp_async_wait<0>();
            return;
        }
        s = pl.s;
        snap = pl.snap;
        dtd = pl.dt;
        steps0 = in.pos.steps;
    }
    const int strip = gw % p.nstrips;
    const int chunk = gw / p.nstrips;
    const int r0 = d.upd_lo + chunk * p.rows_per_warp;
    const int r1 = min(r0 + p.rows_per_warp, d.upd_hi);
    const int x0w = strip * kWarp * V;
    const int c0 = x0w + lane * V;
    StepAccum acc;
    acc.zero();

    if (r0 < d.upd_hi) {
        Cell A[V], B[V], C[V];
        float yT0[V], yT1[V], yT2[V];
        // Bottom face of the chunk: rows r0-1 (A) and r0 (B).
        load_cells<V>(d, p.in, r0 - 1, c0, A);
        load_cells<V>(d, p.in, r0, c0, B);
#pragma unroll
        for (int i = 0; i < V; ++i) {
            set_vel<M>(A[i], k.dry);
            set_vel<M>(B[i], k.dry);
            const FaceFlux f = face_flux<0, M, MASKED>(A[i], B[i], k);
            yT0[i] = f.f0;
            yT1[i] = f.f1;
            yT2[i] = M::add(f.f2, f.corr_hi);
            if (run && r0 == 0 && c0 + i < d.cols) acc.outflow -= dtd * (double)f.f0 * d.dx;
        }
        load_cells<V>(d, p.in, r0 + 1, c0, C);
#pragma unroll
        for (int i = 0; i < V; ++i) set_vel<M>(C[i], k.dry);

        // One row: `cur` is row r, `nxt` row r+1 (velocities set); `pre` receives row r+2.
        auto row = [&](const int r, Cell(&cur)[V], Cell(&nxt)[V], Cell(&pre)[V]) {
            const int j = (r - r0) & (kBatch - 1);
            if (j == 0) {
                // Strip edges for rows r .. r+31, one row per lane.
                __syncwarp();
                const int rr = min(r + lane, d.rows - 1);
                Cell L[1], E[1], R[1];
                load_cells<1>(d, p.in, rr, x0w - 1, L);
                load_cells<1>(d, p.in, rr, x0w, E);
                load_cells<1>(d, p.in, rr, x0w + kWarp * V, R);
                set_vel<M>(L[0], k.dry);
                set_vel<M>(E[0], k.dry);
                set_vel<M>(R[0], k.dry);
                const FaceFlux f = face_flux<1, M, MASKED>(L[0], E[0], k);
                s_left[wib][0][lane] = f.f0;
                s_left[wib][1][lane] = M::add(f.f1, f.corr_hi);
                s_left[wib][2][lane] = f.f2;
                if (run && x0w == 0 && r + lane < r1) acc.outflow -= dtd * (double)f.f0 * d.dy;
                s_right[wib][0][lane] = R[0].h;
                s_right[wib][1][lane] = R[0].hu;
                s_right[wib][2][lane] = R[0].hv;
                s_right[wib][3][lane] = R[0].z;
                s_right[wib][4][lane] = R[0].nm;
                s_right[wib][5][lane] = R[0].u;
                s_right[wib][6][lane] = R[0].v;
                __syncwarp();
            }
            // Prefetch the row after next.
            if (r + 1 < r1) load_cells<V>(d, p.in, r + 2, c0, pre);
            // y-faces above row r: lo side updates row r, hi side is carried to row r+1.
            float yB0[V], yB1[V], yB2[V], yN0[V], yN1[V], yN2[V];
#pragma unroll
            for (int i = 0; i < V; ++i) {
                const FaceFlux f = face_flux<0, M, MASKED>(cur[i], nxt[i], k);
                yB0[i] = f.f0;
                yB1[i] = f.f1;
                yB2[i] = M::add(f.f2, f.corr_lo);
                yN0[i] = f.f0;
                yN1[i] = f.f1;
                yN2[i] = M::add(f.f2, f.corr_hi);
                if (run && r == d.rows - 1 && c0 + i < d.cols) acc.outflow += dtd * (double)f.f0 * d.dx;
            }
            // x-faces of row r: right neighbour of each lane's last cell.
            Cell rn;
            rn.h = __shfl_down_sync(0xffffffffu, cur[0].h, 1);
            rn.hu = __shfl_down_sync(0xffffffffu, cur[0].hu, 1);
            rn.hv = __shfl_down_sync(0xffffffffu, cur[0].hv, 1);
            rn.z = __shfl_down_sync(0xffffffffu, cur[0].z, 1);
            rn.nm = __shfl_down_sync(0xffffffffu, cur[0].nm, 1);
            rn.u = __shfl_down_sync(0xffffffffu, cur[0].u, 1);
            rn.v = __shfl_down_sync(0xffffffffu, cur[0].v, 1);
            {
                const float e0 = s_right[wib][0][j], e1 = s_right[wib][1][j], e2 = s_right[wib][2][j];
                const float e3 = s_right[wib][3][j], e4 = s_right[wib][4][j], e5 = s_right[wib][5][j];
                const float e6 = s_right[wib][6][j];
                if (lane == 31) rn = Cell{e0, e1, e2, e3, e4, e5, e6};
            }
            float xl0[V], xl1[V], xl2[V];  // lo side of the right face of cell i
            float xr0[V], xr1[V], xr2[V];  // hi side of the left face of cell i
#pragma unroll
            for (int i = 0; i < V; ++i) {
                const Cell& right = (i + 1 < V) ? cur[(i + 1) % V] : rn;
                const FaceFlux f = face_flux<1, M, MASKED>(cur[i], right, k);
                xl0[i] = f.f0;
                xl1[i] = M::add(f.f1, f.corr_lo);
                xl2[i] = f.f2;
                if (i + 1 < V) {
                    xr0[(i + 1) % V] = f.f0;
                    xr1[(i + 1) % V] = M::add(f.f1, f.corr_hi);
                    xr2[(i + 1) % V] = f.f2;
                } else {
                    const float h0 = f.f0, h1 = M::add(f.f1, f.corr_hi), h2 = f.f2;
                    xr0[0] = __shfl_up_sync(0xffffffffu, h0, 1);
                    xr1[0] = __shfl_up_sync(0xffffffffu, h1, 1);
                    xr2[0] = __shfl_up_sync(0xffffffffu, h2, 1);
                }
                if (run && c0 + i == d.cols - 1) acc.outflow += dtd * (double)f.f0 * d.dy;
            }
            {
                const float l0 = s_left[wib][0][j], l1 = s_left[wib][1][j], l2 = s_left[wib][2][j];
                if (lane == 0) {
                    xr0[0] = l0;
                    xr1[0] = l1;
                    xr2[0] = l2;
                }
            }
            // Cell updates of row r.
            const int64_t so = (int64_t)r * p.out.pitch;
            float ho[V], huo[V], hvo[V];
#pragma unroll
            for (int i = 0; i < V; ++i) {
                const bool act = MASKED ? active(cur[i].nm) : true;
                const float n2 = MASKED ? fabsf(cur[i].nm) : cur[i].nm;
                float upd[3];
                const float U[3] = {cur[i].h, cur[i].hu, cur[i].hv};
                const float XL[3] = {xl0[i], xl1[i], xl2[i]};
                const float XR[3] = {xr0[i], xr1[i], xr2[i]};
                const float YB[3] = {yB0[i], yB1[i], yB2[i]};
                const float YT[3] = {yT0[i], yT1[i], yT2[i]};
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    const float divx = M::div(M::sub(XL[q], XR[q]), k.dx);
                    const float divy = M::div(M::sub(YB[q], YT[q]), k.dy);
                    upd[q] = M::sub(U[q], M::mul(s.dt, M::add(divx, divy)));
                }
                float rain;
                if (d.mult != nullptr) {
                    const int cc = min(max(c0 + i, 0), d.cols - 1);
                    rain = M::mul(s.dt_rain, __ldg(d.mult + (int64_t)r * d.spitch + cc));
                } else {
                    rain = act ? s.dt_rain : 0.0f;  // float(dt*rate) * 1.0 or * 0.0
                }
                upd[0] = M::add(upd[0], rain);
                const float h = fmaxf(upd[0], 0.0f);
                const float norm = M::hypot(upd[1], upd[2]);
                const float fr = M::div(M::mul(M::mul(s.dt_g, n2), norm), M::pow73(fmaxf(h, k.dry), k.expo));
                const float den = M::add(1.0f, fr);
                const float qx = M::div(upd[1], den);
                const float qy = M::div(upd[2], den);
                const bool wet = act & (h > k.dry);
                ho[i] = act ? h : 0.0f;
                huo[i] = wet ? qx : 0.0f;
                hvo[i] = wet ? qy : 0.0f;
                if (run && c0 + i < d.cols) {
                    float u, v;
                    M::vel2(huo[i], hvo[i], ho[i], k.dry, u, v);
                    const float w = M::sqrt(M::mul(k.g, ho[i]));
                    const float inv = M::add(M::div(M::add(fabsf(u), w), k.dx), M::div(M::add(fabsf(v), w), k.dy));
                    acc.maxinv = nan_max(acc.maxinv, act ? inv : 0.0f);
                    acc.vol += (double)ho[i];
                    if (d.mult != nullptr) acc.rain += (double)rain; else acc.rain_cells += act ? 1u : 0u;
                    if (upd[0] < 0.0f) acc.clip -= (double)upd[0];
                    if (MASKED && !act) acc.mask += (double)h;
                }
            }
            // Store row r.
            if (c0 + V <= d.cols) {
                if constexpr (V == 4) {
                    *reinterpret_cast<float4*>(p.out.h + so + c0) = make_float4(ho[0], ho[1], ho[2], ho[3]);
                    *reinterpret_cast<float4*>(p.out.hu + so + c0) = make_float4(huo[0], huo[1], huo[2], huo[3]);
                    *reinterpret_cast<float4*>(p.out.hv + so + c0) = make_float4(hvo[0], hvo[1], hvo[2], hvo[3]);
                } else if constexpr (V == 2) {
                    *reinterpret_cast<float2*>(p.out.h + so + c0) = make_float2(ho[0], ho[1]);
                    *reinterpret_cast<float2*>(p.out.hu + so + c0) = make_float2(huo[0], huo[1]);
                    *reinterpret_cast<float2*>(p.out.hv + so + c0) = make_float2(hvo[0], hvo[1]);
                } else {
#pragma unroll
                    for (int i = 0; i < V; ++i) {
                        p.out.h[so + c0 + i] = ho[i];
                        p.out.hu[so + c0 + i] = huo[i];
                        p.out.hv[so + c0 + i] = hvo[i];
                    }
                }
            } else {
#pragma unroll
                for (int i = 0; i < V; ++i) {
                    if (c0 + i < d.cols) {
                        p.out.h[so + c0 + i] = ho[i];
                        p.out.hu[so + c0 + i] = huo[i];
                        p.out.hv[so + c0 + i] = hvo[i];
                    }
                }
            }
            if (RUN && snap >= 0) {
                const Control* c = p.ctl;
                const int64_t base = (int64_t)snap * c->out_plane + (int64_t)r * d.cols;
#pragma unroll
                for (int i = 0; i < V; ++i) {
                    if (c0 + i < d.cols) {
                        c->out_h[base + c0 + i] = ho[i];
                        c->out_hu[base + c0 + i] = huo[i];
                        c->out_hv[base + c0 + i] = hvo[i];
                    }
                }
            }
            // Row r+1 inherits the carried face values; the prefetched row gets velocities.
#pragma unroll
            for (int i = 0; i < V; ++i) {
                yT0[i] = yN0[i];
                yT1[i] = yN1[i];
                yT2[i] = yN2[i];
                if (r + 1 < r1) set_vel<M>(pre[i], k.dry);
            }
        };

        // Three-way rotation of the row buffers avoids copying them every row.
        for (int r = r0; r < r1; r += 3) {
            row(r, B, C, A);
            if (r + 1 < r1) row(r + 1, C, A, B);
            if (r + 2 < r1) row(r + 2, A, B, C);
        }
    }
    if constexpr (RUN) {
        Accum a;
        a.maxinv = acc.maxinv;
        a.vol = acc.vol;
        a.rain = acc.rain + (double)acc.rain_cells * (double)s.dt_rain;
        a.outflow = acc.outflow;
        a.clip = acc.clip;
        a.mask = acc.mask;
        cp_async_wait<0>();
        __syncwarp();
        warp_end_step(p.ctl, &p.slots[gw], s_old[wib], p.par, steps0, gw % kMaxStripes, a);
    }
}

// Cells [r0, r1) x [0, cols) of a plane under a 2-D grid-stride launch (grid.x
// over columns, grid.y over rows, see cell_grid on the host): body(r, c) for
// each, with no division per cell.
template <class F>
__device__ __forceinline__ void for_cells(int r0, int r1, int cols, F&& body) {
    for (int r = r0 + (int)blockIdx.y; r < r1; r += (int)gridDim.y)
        for (int c = (int)(blockIdx.x * blockDim.x + threadIdx.x); c < cols; c += (int)(gridDim.x * blockDim.x))
            body(r, c);
}

// Max inverse CFL dt and stored volume of a state (the reduction of
// compute_cfl_dt, shallow_water_2d.py:269-273); initialises the run control.
// A 2-D launch: each CTA's partial is slot blockIdx.y * gridDim.x + blockIdx.x.
template <class M, int THREADS>
__global__ void __launch_bounds__(THREADS) reduce_kernel(const DomainDev d, const StateView s,
                                                         Control* ctl, Partial* parts) {
    const Consts& k = d.k;
    Accum acc;
    acc.zero();
    for_cells(d.upd_lo, d.upd_hi, d.cols, [&](int r, int c) {
        const float h = s.h[(int64_t)r * s.pitch + c];
        const float hu = s.hu[(int64_t)r * s.pitch + c];
        const float hv = s.hv[(int64_t)r * s.pitch + c];
        const bool act = active(d.nm[(int64_t)r * d.spitch + c]);
        float u, v;
        M::vel2(hu, hv, h, k.dry, u, v);
        const float w = M::sqrt(M::mul(k.g, fmaxf(h, 0.0f)));
        const float inv = M::add(M::div(M::add(fabsf(u), w), k.dx), M::div(M::add(fabsf(v), w), k.dy));
        acc.maxinv = nan_max(acc.maxinv, act ? inv : 0.0f);
        if (act) acc.vol += (double)h;
    });
    finish_start<THREADS>(d, ctl, parts, acc);
}

}  // namespace swe
