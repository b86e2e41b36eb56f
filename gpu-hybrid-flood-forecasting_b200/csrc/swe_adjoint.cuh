// Hand-written reverse mode (adjoint) of the shallow-water step (sm_100a).
//
// The reference has no adjoint: it never differentiates its solver (the only
// gradients in it are of the U-Net, src/hybrid_flood/ml/train.py:181).  This is
// the vector-Jacobian product of one step of
// src/hybrid_flood/numpy_solver/shallow_water_2d.py:277-327 with dt held fixed
// (a stop-gradient, as jax.grad of a fixed-dt scan would treat it):
//
//   given lambda' = dL/dU_{k+1}, returns lambda = dL/dU_k and accumulates
//   dL/d(n^2) per cell and dL/d(rain scale).
//
// Non-smooth points use these conventions (zero where the forward is flat or
// undefined): max(x, 0) passes the gradient only for x > 0; velocities m/h
// only for h > dry; sqrt(g H) only for H > 0; the friction term's max(h, dry)
// only for h > dry; hypot only for a non-zero norm; HLL speed min/max route to
// the selected argument; the flux select follows the taken branch.
//
// Two kernels per reverse step:
//   adj_cell_kernel  recomputes the cell's forward update (its four faces) and
//                    reverses the pointwise part (rain, clip, friction, masks):
//                    lambda_upd = dL/d(upd) per cell, plus the n^2 and rain
//                    scale gradients;
//   adj_face_tile_kernel  evaluates each face's flux VJP once per tile (each
//                    face's flux depends on the states of its two cells through
//                    reconstruction and HLL) and gathers, for each cell, its four
//                    faces' contributions into lambda = lambda_upd + their sum.
#pragma once

#include "swe_step.cuh"

namespace swe {

struct AdjConsts {
    float g, half_g, dry, eps, dx, dy;
};

// The reverse step needs derivative values to float accuracy, not the forward's
// rounding: approximate division, square root and power (a few ulp) keep it cheap.
__device__ __forceinline__ float adiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ float asqrt(float a) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
}
__device__ __forceinline__ float apow(float x, float e) {  // x > 0
    float l, r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(l) : "f"(x));
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(l * e));
    return r;
}

// One side of a face: the cell's state, its velocities (m/h where h > dry, else
// 0: computed once per cell and shared by the cell's four faces) and whether it
// is active.
struct FaceIn {
    float h, hu, hv, z, u, v;
    bool act;
};

__device__ __forceinline__ FaceIn face_in(float h, float hu, float hv, float z, bool act, float dry) {
    const bool wet = h > dry;
    return {h, hu, hv, z, wet ? adiv(hu, h) : 0.f, wet ? adiv(hv, h) : 0.f, act};
}

__device__ __forceinline__ FaceIn face_in(const Cell& c, float dry) {
    return face_in(c.h, c.hu, c.hv, c.z, active(c.nm), dry);
}

// The mirrored copy of a cell across a wall: the normal momentum and velocity change sign.
template <int AXIS>
__device__ __forceinline__ FaceIn mirror(FaceIn c) {
    if (AXIS == 1) {
        c.hu = -c.hu;
        c.u = -c.u;
    } else {
        c.hv = -c.hv;
        c.v = -c.v;
    }
    return c;
}

// Forward flux of one face (plain float32 arithmetic; the adjoint needs the
// values, not the reference's bit pattern).
template <int AXIS>
__device__ void adj_face_fwd(FaceIn lo, FaceIn hi, const AdjConsts& k, float F[3], float& clo, float& chi) {
    F[0] = F[1] = F[2] = 0.f;
    clo = chi = 0.f;
    if (!(lo.act || hi.act)) return;
    FaceIn L = lo, R = hi;
    if (lo.act && !hi.act) {
        R = mirror<AXIS>(lo);
    } else if (!lo.act && hi.act) {
        L = mirror<AXIS>(hi);
    }
    const float zf = fmaxf(L.z, R.z);
    const float HL = fmaxf(L.h + L.z - zf, 0.f), HR = fmaxf(R.h + R.z - zf, 0.f);
    const float uL = L.u, vL = L.v, uR = R.u, vR = R.v;
    const float XL = HL * uL, YL = HL * vL, XR = HR * uR, YR = HR * vR;
    const float nL = AXIS == 1 ? XL : YL, nR = AXIS == 1 ? XR : YR;
    const float unL = HL > k.dry ? adiv(nL, HL) : 0.f, unR = HR > k.dry ? adiv(nR, HR) : 0.f;
    const float tL = HL > k.dry ? adiv(YL, HL) : 0.f, tR = HR > k.dry ? adiv(YR, HR) : 0.f;
    const float cL = asqrt(k.g * HL), cR = asqrt(k.g * HR);
    const float sL = fminf(unL - cL, unR - cR), sR = fmaxf(unL + cL, unR + cR);
    const float pL = k.half_g * HL * HL, pR = k.half_g * HR * HR;
    float fL[3], fR[3];
    if (AXIS == 1) {
        fL[0] = XL; fL[1] = XL * unL + pL; fL[2] = XL * tL;
        fR[0] = XR; fR[1] = XR * unR + pR; fR[2] = XR * tR;
    } else {
        fL[0] = YL; fL[1] = XL * unL; fL[2] = YL * unL + pL;
        fR[0] = YR; fR[1] = XR * unR; fR[2] = YR * unR + pR;
    }
    const float UL[3] = {HL, XL, YL}, UR[3] = {HR, XR, YR};
    const float spread = sR - sL;
    const float den = spread > k.eps ? spread : 1.f;
    for (int q = 0; q < 3; ++q) {
        const float m = adiv(sR * fL[q] - sL * fR[q] + sL * sR * (UR[q] - UL[q]), den);
        F[q] = sL >= 0.f ? fL[q] : (sR <= 0.f ? fR[q] : m);
    }
    clo = k.half_g * (L.h * L.h - HL * HL);
    chi = k.half_g * (R.h * R.h - HR * HR);
}

// VJP of one face: given dL/dF (3), dL/dcorr_lo, dL/dcorr_hi, return dL/d(h, hu, hv)
// of the lo cell and of the hi cell (after undoing the wall mirroring).
template <int AXIS>
__device__ void adj_face_vjp(FaceIn lo, FaceIn hi, const AdjConsts& k, const float lF[3], float lclo,
                             float lchi, float dlo[3], float dhi[3]) {
    dlo[0] = dlo[1] = dlo[2] = 0.f;
    dhi[0] = dhi[1] = dhi[2] = 0.f;
    if (!(lo.act || hi.act)) return;
    const bool hi_wall = lo.act && !hi.act, lo_wall = !lo.act && hi.act;
    FaceIn L = lo, R = hi;
    if (hi_wall) {
        R = mirror<AXIS>(lo);
    } else if (lo_wall) {
        L = mirror<AXIS>(hi);
    }
    // ---- forward, keeping what the reverse needs ----
    const float zf = fmaxf(L.z, R.z);
    const float aL = L.h + L.z - zf, aR = R.h + R.z - zf;
    const float HL = fmaxf(aL, 0.f), HR = fmaxf(aR, 0.f);
    const bool dL = L.h > k.dry, dR = R.h > k.dry;
    const float uL = L.u, vL = L.v, uR = R.u, vR = R.v;
    const float XL = HL * uL, YL = HL * vL, XR = HR * uR, YR = HR * vR;
    const float nL = AXIS == 1 ? XL : YL, nR = AXIS == 1 ? XR : YR;
    const bool wL = HL > k.dry, wR = HR > k.dry;
    const float unL = wL ? adiv(nL, HL) : 0.f, unR = wR ? adiv(nR, HR) : 0.f;
    const float tL = wL ? adiv(YL, HL) : 0.f, tR = wR ? adiv(YR, HR) : 0.f;
    const float cL = asqrt(k.g * HL), cR = asqrt(k.g * HR);
    const float aminL = unL - cL, aminR = unR - cR, amaxL = unL + cL, amaxR = unR + cR;
    const float sL = fminf(aminL, aminR), sR = fmaxf(amaxL, amaxR);
    const float pL = k.half_g * HL * HL, pR = k.half_g * HR * HR;
    float fL[3], fR[3];
    if (AXIS == 1) {
        fL[0] = XL; fL[1] = XL * unL + pL; fL[2] = XL * tL;
        fR[0] = XR; fR[1] = XR * unR + pR; fR[2] = XR * tR;
    } else {
        fL[0] = YL; fL[1] = XL * unL; fL[2] = YL * unL + pL;
        fR[0] = YR; fR[1] = XR * unR; fR[2] = YR * unR + pR;
    }
    const float UL[3] = {HL, XL, YL}, UR[3] = {HR, XR, YR};
    const float spread = sR - sL;
    const bool use_spread = spread > k.eps;
    const float den = use_spread ? spread : 1.f;
    const bool take_l = sL >= 0.f, take_r = !take_l && sR <= 0.f;
    // ---- reverse ----
    float lfL[3] = {0.f, 0.f, 0.f}, lfR[3] = {0.f, 0.f, 0.f};
    float lUL[3] = {0.f, 0.f, 0.f}, lUR[3] = {0.f, 0.f, 0.f};
    float lsL = 0.f, lsR = 0.f;
    if (take_l) {
        for (int q = 0; q < 3; ++q) lfL[q] = lF[q];
    } else if (take_r) {
        for (int q = 0; q < 3; ++q) lfR[q] = lF[q];
    } else {
        float lden = 0.f;
        for (int q = 0; q < 3; ++q) {
            const float dU = UR[q] - UL[q];
            const float m = adiv(sR * fL[q] - sL * fR[q] + sL * sR * dU, den);
            const float lN = adiv(lF[q], den);
            lden -= m * lN;
            lsR += (fL[q] + sL * dU) * lN;
            lsL += (-fR[q] + sR * dU) * lN;
            lfL[q] += sR * lN;
            lfR[q] -= sL * lN;
            lUR[q] += sL * sR * lN;
            lUL[q] -= sL * sR * lN;
        }
        if (use_spread) {
            lsR += lden;
            lsL -= lden;
        }
    }
    // corrections: half_g (h^2 - H^2) on each side
    float lLh = k.g * L.h * lclo, lRh = k.g * R.h * lchi;
    float lHL = lUL[0] - k.g * HL * lclo, lHR = lUR[0] - k.g * HR * lchi;
    float lXL = lUL[1], lYL = lUL[2], lXR = lUR[1], lYR = lUR[2];
    float lunL = 0.f, lunR = 0.f, ltL = 0.f, ltR = 0.f, lpL = 0.f, lpR = 0.f;
    if (AXIS == 1) {
        lXL += lfL[0] + unL * lfL[1] + tL * lfL[2];
        lunL += XL * lfL[1];
        lpL += lfL[1];
        ltL += XL * lfL[2];
        lXR += lfR[0] + unR * lfR[1] + tR * lfR[2];
        lunR += XR * lfR[1];
        lpR += lfR[1];
        ltR += XR * lfR[2];
    } else {
        lYL += lfL[0] + unL * lfL[2];
        lXL += unL * lfL[1];
        lunL += XL * lfL[1] + YL * lfL[2];
        lpL += lfL[2];
        lYR += lfR[0] + unR * lfR[2];
        lXR += unR * lfR[1];
        lunR += XR * lfR[1] + YR * lfR[2];
        lpR += lfR[2];
    }
    lHL += k.g * HL * lpL;
    lHR += k.g * HR * lpR;
    // wave speeds: min/max route to the selected argument
    float lcL = 0.f, lcR = 0.f;
    if (aminL <= aminR) { lunL += lsL; lcL -= lsL; } else { lunR += lsL; lcR -= lsL; }
    if (amaxL >= amaxR) { lunL += lsR; lcL += lsR; } else { lunR += lsR; lcR += lsR; }
    if (cL > 0.f) lHL += adiv(0.5f * k.g, cL) * lcL;
    if (cR > 0.f) lHR += adiv(0.5f * k.g, cR) * lcR;
    // un = n / H, t = Y / H (for H > dry)
    float lnL = 0.f, lnR = 0.f;
    if (wL) {
        lnL += adiv(lunL, HL);
        lHL -= adiv(unL, HL) * lunL;
        if (AXIS == 1) {
            lYL += adiv(ltL, HL);
            lHL -= adiv(tL, HL) * ltL;
        }
    }
    if (wR) {
        lnR += adiv(lunR, HR);
        lHR -= adiv(unR, HR) * lunR;
        if (AXIS == 1) {
            lYR += adiv(ltR, HR);
            lHR -= adiv(tR, HR) * ltR;
        }
    }
    if (AXIS == 1) { lXL += lnL; lXR += lnR; } else { lYL += lnL; lYR += lnR; }
    // X = H u, Y = H v
    lHL += uL * lXL + vL * lYL;
    lHR += uR * lXR + vR * lYR;
    const float luL = HL * lXL, lvL = HL * lYL, luR = HR * lXR, lvR = HR * lYR;
    // H = max(h + z - zf, 0) with the bed held fixed
    if (aL > 0.f) lLh += lHL;
    if (aR > 0.f) lRh += lHR;
    // u = hu / h, v = hv / h (for h > dry)
    float gL[3] = {lLh, 0.f, 0.f}, gR[3] = {lRh, 0.f, 0.f};
    if (dL) {
        gL[1] = adiv(luL, L.h);
        gL[2] = adiv(lvL, L.h);
        gL[0] -= adiv(uL * luL + vL * lvL, L.h);
    }
    if (dR) {
        gR[1] = adiv(luR, R.h);
        gR[2] = adiv(lvR, R.h);
        gR[0] -= adiv(uR * luR + vR * lvR, R.h);
    }
    // undo the wall mirroring: the mirrored side's gradient belongs to the active cell
    const int nq = AXIS == 1 ? 1 : 2;
    if (hi_wall) {
        for (int q = 0; q < 3; ++q) dlo[q] = gL[q] + (q == nq ? -gR[q] : gR[q]);
    } else if (lo_wall) {
        for (int q = 0; q < 3; ++q) dhi[q] = gR[q] + (q == nq ? -gL[q] : gL[q]);
    } else {
        for (int q = 0; q < 3; ++q) {
            dlo[q] = gL[q];
            dhi[q] = gR[q];
        }
    }
}

struct AdjLaunch {
    DomainDev d;
    StateView in;        // U_k
    StateView next;      // U_{k+1} when known (h == nullptr otherwise)
    StateView lam;       // dL/dU_{k+1}
    StateOut lam_out;    // dL/dU_k
    float* lupd[3];      // scratch: dL/d(upd) planes, pitch lpitch
    int64_t lpitch;
    float* grad_n2;      // rows x cols, accumulated
    double* grad_rain;   // device scalar, accumulated
    StepScalars s;       // float32 dt, dt*rate (scaled), dt*g
    float dt_rate;       // float32 dt * rate(t) before the rain scale
    AdjConsts k;
    float rdx, rdy;      // 1/dx, 1/dy
};

__device__ __forceinline__ Cell adj_load(const DomainDev& d, const StateView& s, int r, int c) {
    Cell t[1];
    load_cells<1>(d, s, r, c, t);
    return t[0];
}

// The forward update of cell (r, c) from its four faces: upd (3) before the
// pointwise part.
__device__ void adj_cell_update(const AdjLaunch& p, int r, int c, float upd[3]) {
    const DomainDev& d = p.d;
    const float dry = p.k.dry;
    const FaceIn C = face_in(adj_load(d, p.in, r, c), dry);
    const FaceIn W = face_in(adj_load(d, p.in, r, c - 1), dry), E = face_in(adj_load(d, p.in, r, c + 1), dry);
    const FaceIn S = face_in(adj_load(d, p.in, r - 1, c), dry), N = face_in(adj_load(d, p.in, r + 1, c), dry);
    float Fl[3], Fr[3], Fb[3], Ft[3], cl_lo, cl_hi, cr_lo, cr_hi, cb_lo, cb_hi, ct_lo, ct_hi;
    adj_face_fwd<1>(W, C, p.k, Fl, cl_lo, cl_hi);
    adj_face_fwd<1>(C, E, p.k, Fr, cr_lo, cr_hi);
    adj_face_fwd<0>(S, C, p.k, Fb, cb_lo, cb_hi);
    adj_face_fwd<0>(C, N, p.k, Ft, ct_lo, ct_hi);
    const float U[3] = {C.h, C.hu, C.hv};
    for (int q = 0; q < 3; ++q) {
        const float xl = Fr[q] + (q == 1 ? cr_lo : 0.f);
        const float xr = Fl[q] + (q == 1 ? cl_hi : 0.f);
        const float yb = Ft[q] + (q == 2 ? ct_lo : 0.f);
        const float yt = Fb[q] + (q == 2 ? cb_hi : 0.f);
        upd[q] = U[q] - p.s.dt * ((xl - xr) * p.rdx + (yb - yt) * p.rdy);
    }
}

// The cell update before the pointwise part, rebuilt from the step's own output
// U_{k+1} = (h1, hu1, hv1) of an active cell instead of from its four faces.
// The momenta invert the semi-implicit friction: with a = dt g n^2 max(h,dry)^(-7/3),
// q = upd/(1 + a|upd|) gives upd = q/(1 - a|q|).  Returns false (rebuild from the
// faces instead) where that inversion loses precision (a|q| > 0.999, i.e. friction
// dividing the momentum by more than 1000).  For dry or clipped cells only the
// depth part is needed: the momentum outputs are zero and carry no gradient.
__device__ __forceinline__ bool adj_upd_from_next(const AdjLaunch& p, int r, int c, float n2, float upd[3]) {
    const int64_t o = (int64_t)r * p.next.pitch + c;
    const float h1 = p.next.h[o];
    upd[0] = h1;  // only the sign of upd0 + rain and h itself are used below
    upd[1] = upd[2] = 0.f;
    if (!(h1 > p.k.dry)) return true;
    const float q1 = p.next.hu[o], q2 = p.next.hv[o];
    const float aq = p.s.dt_g * n2 * apow(h1, -7.0f / 3.0f) * asqrt(q1 * q1 + q2 * q2);
    if (!(aq <= 0.999f)) return false;
    const float den = adiv(1.f, 1.f - aq);
    upd[1] = q1 * den;
    upd[2] = q2 * den;
    return true;
}

// Reverse of the pointwise part of cell (r, c) (rain, clip, friction, masks):
// returns lupd = dL/d(upd) (zero for an inactive cell); when `owned`, also adds
// the cell's dL/d(n^2) to grad_n2 and its rain-scale term to *rain_acc.
template <bool NEXT>
__device__ __forceinline__ void adj_cell_at(const AdjLaunch& p, int r, int c, bool owned, double* rain_acc,
                                            float lu[3]) {
    const DomainDev& d = p.d;
    const float nm = d.nm[(int64_t)r * d.spitch + c];
    lu[0] = lu[1] = lu[2] = 0.f;
    if (!active(nm)) return;
    const float mult = d.mult ? d.mult[(int64_t)r * d.spitch + c] : 1.f;
    float upd[3];
    // upd[0] below is the depth after the rain (before the clip).
    if (!(NEXT && adj_upd_from_next(p, r, c, fabsf(nm), upd))) {
        adj_cell_update(p, r, c, upd);
        upd[0] += p.s.dt_rain * mult;
    }
    const float h = fmaxf(upd[0], 0.f);
    const float norm = asqrt(upd[1] * upd[1] + upd[2] * upd[2]);
    const float m = fmaxf(h, p.k.dry);
    const float pw = apow(m, -7.0f / 3.0f);
    const float n2 = fabsf(nm);
    const float fr = p.s.dt_g * n2 * norm * pw;
    const float den = 1.f + fr;
    const float rden = adiv(1.f, den);
    const float qx = upd[1] * rden, qy = upd[2] * rden;
    const bool wet = h > p.k.dry;
    const int64_t li = (int64_t)r * p.lam.pitch + c;
    const float lqx = wet ? p.lam.hu[li] : 0.f, lqy = wet ? p.lam.hv[li] : 0.f;
    float lh = p.lam.h[li];
    const float lden = -(lqx * qx + lqy * qy) * rden;
    float lu1 = lqx * rden, lu2 = lqy * rden;
    if (norm > 0.f) {
        const float lnorm = lden * p.s.dt_g * n2 * pw;
        lu1 += adiv(lnorm * upd[1], norm);
        lu2 += adiv(lnorm * upd[2], norm);
    }
    if (h > p.k.dry) lh += adiv(lden * fr * (-7.0f / 3.0f), h);
    const float lu0 = upd[0] > 0.f ? lh : 0.f;
    if (owned) {
        p.grad_n2[(int64_t)r * d.cols + c] += lden * p.s.dt_g * norm * pw;
        *rain_acc += (double)lu0 * (double)p.dt_rate * (double)mult;
    }
    lu[0] = lu0;
    lu[1] = lu1;
    lu[2] = lu2;
}

// Adds a CTA's rain-scale gradient to the device scalar (one atomic per CTA).
template <int THREADS>
__device__ __forceinline__ void adj_flush_rain(const AdjLaunch& p, double rain_acc) {
    rain_acc = warp_sum(rain_acc);
    __shared__ double s_r[THREADS / kWarp];
    if ((threadIdx.x & 31) == 0) s_r[threadIdx.x >> 5] = rain_acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < THREADS / kWarp; ++w) t += s_r[w];
        if (t != 0.0) atomicAdd(p.grad_rain, t);
    }
}

template <int THREADS, bool NEXT>
__global__ void __launch_bounds__(THREADS) adj_cell_kernel(const AdjLaunch p) {
    const DomainDev& d = p.d;
    const int64_t n = (int64_t)d.rows * d.cols;
    double rain_acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * THREADS) {
        const int r = (int)(i / d.cols), c = (int)(i - (int64_t)r * d.cols);
        float lu[3];
        adj_cell_at<NEXT>(p, r, c, true, &rain_acc, lu);
        const int64_t lo = (int64_t)r * p.lpitch + c;
        p.lupd[0][lo] = lu[0];
        p.lupd[1][lo] = lu[1];
        p.lupd[2][lo] = lu[2];
    }
    adj_flush_rain<THREADS>(p, rain_acc);
}

// dL/d(upd) of cell (r, c); zero outside the grid (ghost cells are not updated).
__device__ __forceinline__ void lupd_at(const AdjLaunch& p, int r, int c, float l[3]) {
    if (r < 0 || r >= p.d.rows || c < 0 || c >= p.d.cols) {
        l[0] = l[1] = l[2] = 0.f;
        return;
    }
    const int64_t o = (int64_t)r * p.lpitch + c;
    l[0] = p.lupd[0][o];
    l[1] = p.lupd[1][o];
    l[2] = p.lupd[2][o];
}

// VJP of the face between the lo cell (rl, cl) and the hi cell (rh, ch) (ghost
// cells allowed: they carry no dL/d(upd)), given a = dt/dx or dt/dy; the
// normal-momentum component is hu for x-faces and hv for y-faces.
template <int AXIS>
__device__ __forceinline__ void adj_face_at(const AdjLaunch& p, int rl, int cl, int rh, int ch, float a,
                                            float* dlo, float* dhi) {
    const FaceIn L = face_in(adj_load(p.d, p.in, rl, cl), p.k.dry), H = face_in(adj_load(p.d, p.in, rh, ch), p.k.dry);
    float ll[3], lh[3], lF[3];
    lupd_at(p, rl, cl, ll);
    lupd_at(p, rh, ch, lh);
#pragma unroll
    for (int q = 0; q < 3; ++q) lF[q] = -a * ll[q] + a * lh[q];
    constexpr int nq = AXIS == 1 ? 1 : 2;
    float lo[3], hi[3];
    adj_face_vjp<AXIS>(L, H, p.k, lF, -a * ll[nq], a * lh[nq], lo, hi);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        dlo[q] = lo[q];
        dhi[q] = hi[q];
    }
}

// The face gather with every face evaluated once.  A CTA of 256 threads takes
// a tile of 32 x 8 cells: each thread evaluates the x-face left of its cell and
// the y-face below it (round 1), warp 0 the y-faces above the tile's top row
// and 8 lanes of warp 1 the x-faces right of its last column (round 2), all
// into shared memory; then each cell adds the four faces' VJPs for its side
// (round 3).  Tile-edge faces are evaluated by both neighbouring tiles, about
// 2.25 face VJPs per cell instead of the 4 of a per-cell gather.
constexpr int kAdjTW = 32, kAdjTH = 8;

__global__ void __launch_bounds__(kAdjTW * kAdjTH) adj_face_tile_kernel(const AdjLaunch p) {
    __shared__ float s_x[kAdjTH][kAdjTW + 1][6];  // face left of tile column c: dlo (0..2), dhi (3..5)
    __shared__ float s_y[kAdjTH + 1][kAdjTW][6];  // face below tile row r
    const DomainDev& d = p.d;
    const int tiles_x = (d.cols + kAdjTW - 1) / kAdjTW, tiles_y = (d.rows + kAdjTH - 1) / kAdjTH;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const float ax = p.s.dt * p.rdx, ay = p.s.dt * p.rdy;
    for (int tile = blockIdx.x; tile < tiles_x * tiles_y; tile += gridDim.x) {
        const int c0 = (tile % tiles_x) * kAdjTW, r0 = (tile / tiles_x) * kAdjTH;
        const int r = r0 + ty, c = c0 + tx;
        // x-faces exist for rows [0, rows) and columns [0, cols] (left of column c);
        // y-faces for columns [0, cols) and rows [0, rows] (below row r).
        if (r < d.rows && c <= d.cols) adj_face_at<1>(p, r, c - 1, r, c, ax, &s_x[ty][tx][0], &s_x[ty][tx][3]);
        if (c < d.cols && r <= d.rows) adj_face_at<0>(p, r - 1, c, r, c, ay, &s_y[ty][tx][0], &s_y[ty][tx][3]);
        if (ty == 0) {
            const int rt = r0 + kAdjTH;
            if (c < d.cols && rt <= d.rows) adj_face_at<0>(p, rt - 1, c, rt, c, ay, &s_y[kAdjTH][tx][0], &s_y[kAdjTH][tx][3]);
        } else if (ty == 1 && tx < kAdjTH) {
            const int rr = r0 + tx, cr = c0 + kAdjTW;
            if (rr < d.rows && cr <= d.cols) adj_face_at<1>(p, rr, cr - 1, rr, cr, ax, &s_x[tx][kAdjTW][0], &s_x[tx][kAdjTW][3]);
        }
        __syncthreads();
        if (r < d.rows && c < d.cols) {
            float g[3];
            lupd_at(p, r, c, g);  // upd_q = U_q - ... : direct term
            const float* fl = s_x[ty][tx];       // left face: this cell is its hi side
            const float* fr = s_x[ty][tx + 1];   // right face: lo side
            const float* fb = s_y[ty][tx];       // bottom face: hi side
            const float* ft = s_y[ty + 1][tx];   // top face: lo side
#pragma unroll
            for (int q = 0; q < 3; ++q) g[q] += fl[3 + q] + fr[q] + fb[3 + q] + ft[q];
            // Ghost cells are mirrored copies of their boundary cell: their side of a
            // boundary face belongs to that cell (normal momentum sign-flipped on reflective edges).
            if (c == 0) {
                const float s = d.bnd[0] == 0 ? -1.f : 1.f;
                g[0] += fl[0]; g[1] += s * fl[1]; g[2] += fl[2];
            }
            if (c == d.cols - 1) {
                const float s = d.bnd[1] == 0 ? -1.f : 1.f;
                g[0] += fr[3]; g[1] += s * fr[4]; g[2] += fr[5];
            }
            if (r == 0) {
                const float s = d.bnd[2] == 0 ? -1.f : 1.f;
                g[0] += fb[0]; g[1] += fb[1]; g[2] += s * fb[2];
            }
            if (r == d.rows - 1) {
                const float s = d.bnd[3] == 0 ? -1.f : 1.f;
                g[0] += ft[3]; g[1] += ft[4]; g[2] += s * ft[5];
            }
            const int64_t o = (int64_t)r * p.lam_out.pitch + c;
            p.lam_out.h[o] = g[0];
            p.lam_out.hu[o] = g[1];
            p.lam_out.hv[o] = g[2];
        }
        __syncthreads();  // the next tile reuses the shared faces
    }
}

// The whole reverse step in one kernel, for lam_out not aliasing lam.  A CTA
// of 256 threads takes a tile of 32 x 16 cells and stages, for the tile and its
// one-cell halo ring (34 x 18 cells), each cell's state, velocities and
// dL/d(upd) in shared memory (phase 0: the pointwise reverse of adj_cell_at;
// halo cells are recomputed, but only the tile's own cells add to the n^2 and
// rain-scale gradients).  Phase 1 evaluates every face of the tile once
// (16 x 33 x-faces and 17 x 32 y-faces over the 256 threads) from the staged
// cells; phase 2 gathers the four faces of each cell.  Reading the halo cells'
// lam while neighbouring tiles write lam_out is why the two must not alias.
constexpr int kFTW = 32, kFTH = 16, kFHW = kFTW + 2, kFHH = kFTH + 2, kFThreads = 256;

struct AdjTileSmem {
    float h[kFHH][kFHW], hu[kFHH][kFHW], hv[kFHH][kFHW], z[kFHH][kFHW], u[kFHH][kFHW], v[kFHH][kFHW];
    float l[3][kFHH][kFHW];
    float fx[kFTH][kFTW + 1][6];  // face left of tile column c: dlo (0..2), dhi (3..5)
    float fy[kFTH + 1][kFTW][6];  // face below tile row r
    unsigned char act[kFHH][kFHW];
};

__device__ __forceinline__ FaceIn staged(const AdjTileSmem& S, int hr, int hc) {
    return {S.h[hr][hc], S.hu[hr][hc], S.hv[hr][hc], S.z[hr][hc], S.u[hr][hc], S.v[hr][hc], S.act[hr][hc] != 0};
}

template <int AXIS>
__device__ __forceinline__ void staged_face(const AdjTileSmem& S, const AdjConsts& k, int lr, int lc, int hr, int hc,
                                            float a, float* out) {
    constexpr int nq = AXIS == 1 ? 1 : 2;
    float lF[3], lo[3], hi[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) lF[q] = -a * S.l[q][lr][lc] + a * S.l[q][hr][hc];
    adj_face_vjp<AXIS>(staged(S, lr, lc), staged(S, hr, hc), k, lF, -a * S.l[nq][lr][lc], a * S.l[nq][hr][hc], lo, hi);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        out[q] = lo[q];
        out[3 + q] = hi[q];
    }
}

template <bool NEXT>
__global__ void __launch_bounds__(kFThreads) adj_tile_kernel(const AdjLaunch p) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    AdjTileSmem& S = *reinterpret_cast<AdjTileSmem*>(s_raw);
    const DomainDev& d = p.d;
    const int tiles_x = (d.cols + kFTW - 1) / kFTW, tiles_y = (d.rows + kFTH - 1) / kFTH;
    const float ax = p.s.dt * p.rdx, ay = p.s.dt * p.rdy;
    double rain_acc = 0.0;
    for (int tile = blockIdx.x; tile < tiles_x * tiles_y; tile += gridDim.x) {
        const int c0 = (tile % tiles_x) * kFTW, r0 = (tile / tiles_x) * kFTH;
        // Phase 0: the tile and its halo ring (ghost cells outside the grid carry no dL/d(upd)).
        for (int i = threadIdx.x; i < kFHH * kFHW; i += kFThreads) {
            const int hr = i / kFHW, hc = i - hr * kFHW;
            const int r = r0 - 1 + hr, c = c0 - 1 + hc;
            const FaceIn f = face_in(adj_load(d, p.in, r, c), p.k.dry);
            S.h[hr][hc] = f.h;
            S.hu[hr][hc] = f.hu;
            S.hv[hr][hc] = f.hv;
            S.z[hr][hc] = f.z;
            S.u[hr][hc] = f.u;
            S.v[hr][hc] = f.v;
            S.act[hr][hc] = f.act ? 1 : 0;
            float lu[3] = {0.f, 0.f, 0.f};
            if (r >= 0 && r < d.rows && c >= 0 && c < d.cols) {
                const bool owned = hr >= 1 && hr <= kFTH && hc >= 1 && hc <= kFTW;
                adj_cell_at<NEXT>(p, r, c, owned, &rain_acc, lu);
            }
            S.l[0][hr][hc] = lu[0];
            S.l[1][hr][hc] = lu[1];
            S.l[2][hr][hc] = lu[2];
        }
        __syncthreads();
        // Phase 1: x-faces exist for rows [0, rows) and columns [0, cols] (left of
        // column c), y-faces for columns [0, cols) and rows [0, rows] (below row r).
        constexpr int NX = kFTH * (kFTW + 1), NY = (kFTH + 1) * kFTW;
        for (int f = threadIdx.x; f < NX + NY; f += kFThreads) {
            if (f < NX) {
                const int ty = f / (kFTW + 1), tx = f - ty * (kFTW + 1);
                if (r0 + ty < d.rows && c0 + tx <= d.cols)
                    staged_face<1>(S, p.k, ty + 1, tx, ty + 1, tx + 1, ax, S.fx[ty][tx]);
            } else {
                const int g = f - NX, ty = g / kFTW, tx = g - ty * kFTW;
                if (c0 + tx < d.cols && r0 + ty <= d.rows)
                    staged_face<0>(S, p.k, ty, tx + 1, ty + 1, tx + 1, ay, S.fy[ty][tx]);
            }
        }
        __syncthreads();
        // Phase 2: each cell of the tile adds its side of its four faces.
        for (int i = threadIdx.x; i < kFTH * kFTW; i += kFThreads) {
            const int ty = i / kFTW, tx = i - ty * kFTW;
            const int r = r0 + ty, c = c0 + tx;
            if (r >= d.rows || c >= d.cols) continue;
            const float* fl = S.fx[ty][tx];
            const float* fr = S.fx[ty][tx + 1];
            const float* fb = S.fy[ty][tx];
            const float* ft = S.fy[ty + 1][tx];
            float g[3];
#pragma unroll
            for (int q = 0; q < 3; ++q) g[q] = S.l[q][ty + 1][tx + 1] + fl[3 + q] + fr[q] + fb[3 + q] + ft[q];
            if (c == 0) {
                const float s = d.bnd[0] == 0 ? -1.f : 1.f;
                g[0] += fl[0]; g[1] += s * fl[1]; g[2] += fl[2];
            }
            if (c == d.cols - 1) {
                const float s = d.bnd[1] == 0 ? -1.f : 1.f;
                g[0] += fr[3]; g[1] += s * fr[4]; g[2] += fr[5];
            }
            if (r == 0) {
                const float s = d.bnd[2] == 0 ? -1.f : 1.f;
                g[0] += fb[0]; g[1] += fb[1]; g[2] += s * fb[2];
            }
            if (r == d.rows - 1) {
                const float s = d.bnd[3] == 0 ? -1.f : 1.f;
                g[0] += ft[3]; g[1] += ft[4]; g[2] += s * ft[5];
            }
            const int64_t o = (int64_t)r * p.lam_out.pitch + c;
            p.lam_out.h[o] = g[0];
            p.lam_out.hu[o] = g[1];
            p.lam_out.hv[o] = g[2];
        }
        __syncthreads();  // the next tile reuses the shared planes
    }
    adj_flush_rain<kFThreads>(p, rain_acc);
}

}  // namespace swe
