// Paired-lane step kernel: the production kernel for 2-column lanes (sm_100a).
//
// Same work decomposition as step_kernel (swe_step.cuh) -- a warp marches up
// a chunk of rows of a 64-column strip, each face evaluated once, strip edges
// staged 32 rows at a time in warp-private shared memory -- but each lane's
// two cells are carried as one float2 pair, so the y-faces of both columns,
// the lane's internal and right x-faces, and both cell updates are each one
// paired evaluation (packed f32x2 add/mul/fma, see swe_pair.cuh).
//
// Rows arrive through a warp-private ring of kRing rows in shared memory: each
// lane copies its own two cells of the five input fields with cp.async (no
// register is held while the copy is in flight) and waits with
// cp.async.wait_group, a hardware wait with no polling.  Lanes past the right
// edge copy nothing; their cells are filled from the last column (ghost ring).
#pragma once

#include "swe_pair.cuh"
#include "swe_step.cuh"

namespace swe {

struct KScalar {
    float g, half_g, dry, eps, zero, one, tiny;
};

__device__ __forceinline__ KScalar make_kscalar(const Consts& k) {
    return {k.g, k.half_g, k.dry, k.eps, 0.f, 1.f, 1.0e-30f};
}

// Raw fields of the lane's two cells of row r (ghost ring applied), no velocities.
__device__ __forceinline__ void load_pair_raw(const DomainDev& d, const StateView& s, int r, int c0,
                                              CellT<float2>& c) {
    Cell t[2];
    load_cells<2>(d, s, r, c0, t);
    c.h = f2(t[0].h, t[1].h);
    c.hu = f2(t[0].hu, t[1].hu);
    c.hv = f2(t[0].hv, t[1].hv);
    c.z = f2(t[0].z, t[1].z);
    c.nm = f2(t[0].nm, t[1].nm);
}

constexpr int kRing = 4;  // rows in flight per warp

__device__ __forceinline__ void cp_async_8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

#ifndef SWE_PAIR_MINBLOCKS
#define SWE_PAIR_MINBLOCKS 4
#endif

// Warp-private shared memory of the march: strip edges of the current 32-row
// batch and the cp.async row ring.
struct WarpSmem {
    float left[3][kWarp];      // hi side of the strip's left x-face, per batch row
    float right[7][kWarp];     // the cell right of the strip, per batch row
    float2 ring[kRing][5][kWarp];  // [slot][field][lane]
};

// One warp marches rows [r0, r1) of the 64-column strip starting at x0w: every
// face once, cells updated, row r written to `out` (and to snapshot `snap` of
// `ctl` in run mode); CFL maximum and ledger terms accumulate into `acc`.
template <class M, bool RUN, bool MASKED>
__device__ __forceinline__ void march_pair(const DomainDev& d, const StateView& in,
                                           const StateOut& out, const StepScalars& s, int snap,
                                           double dtd, const Control* ctl, int r0, int r1,
                                           int x0w, WarpSmem& sm, StepAccum& acc) {
    constexpr int kBatch = kWarp;
    constexpr int V = 2;
    using A = P<M>;
    const Consts& k = d.k;
    const KPair kp = make_kpair(k);
    const KScalar ks = make_kscalar(k);
    const int lane = threadIdx.x & 31;
    const int c0 = x0w + lane * V;
    const B2 valid{c0 < d.cols, c0 + 1 < d.cols};
    const int right_edge = d.cols - 1 - c0;  // 0 or 1 when this lane holds the last column
    const float2 dt2 = splat(s.dt), dtr2 = splat(s.dt_rain), dtg2 = splat(s.dt_g);
    const float2 dx2 = splat(k.dx), dy2 = splat(k.dy);
    const float rdx = 1.0f / k.dx, rdy = 1.0f / k.dy;
    const float2 ndtdx2 = splat(-s.dt * rdx), ndtdy2 = splat(-s.dt * rdy);
    const float2 rdx2 = splat(rdx), rdy2 = splat(rdy);
    const float2 nexpo2 = splat(-k.expo);
    {
        const int nq = r1 - r0 + 2;  // rows r0-1 .. r1 pass through the ring
        const float* planes[5] = {in.h, in.hu, in.hv, d.bed, d.nm};
        const int64_t pitches[5] = {in.pitch, in.pitch, in.pitch, d.spitch, d.spitch};
        const bool edge_strip = x0w + kWarp * V > d.cols;
        // Start the copies of ring row qi (row r0-1+qi, clamped to the grid); one group per row.
        auto issue = [&](int qi) {
            if (qi < nq) {
                const int q = r0 - 1 + qi;
                const int rr = q < 0 ? 0 : (q >= d.rows ? d.rows - 1 : q);
                const int st = qi % kRing;
#pragma unroll
                for (int f = 0; f < 5; ++f) {
                    const float* src = planes[f] + (int64_t)rr * pitches[f] + c0;
                    if (c0 + 1 < d.cols) cp_async_8(&sm.ring[st][f][lane], src);
                    else if (c0 < d.cols) cp_async_4(&sm.ring[st][f][lane], src);
                }
            }
            cp_async_commit();
        };
        // Ring row qi into registers with the ghost ring applied; refill its slot.
        auto consume = [&](int qi, CellT<float2>& out) {
            cp_async_wait<kRing - 1>();
            const int st = qi % kRing;
            const int q = r0 - 1 + qi;
            float2 fv[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) fv[f] = sm.ring[st][f][lane];
            if (edge_strip) {
                __syncwarp();  // the last column may sit in another lane's slot
                const int last = d.cols - 1 - x0w;
                const float* lastp = reinterpret_cast<const float*>(&sm.ring[st][0][0]);
                float g[5];
#pragma unroll
                for (int f = 0; f < 5; ++f) g[f] = lastp[f * 2 * kWarp + last];
                if (d.bnd[1] == 0) g[1] = -g[1];
                if (c0 >= d.cols) {
#pragma unroll
                    for (int f = 0; f < 5; ++f) fv[f].x = g[f];
                }
                if (c0 + 1 >= d.cols) {
#pragma unroll
                    for (int f = 0; f < 5; ++f) fv[f].y = g[f];
                }
                __syncwarp();  // every lane has read before any slot is refilled
            }
            if ((q < 0 && d.bnd[2] == 0) || (q >= d.rows && d.bnd[3] == 0)) fv[2] = neg(fv[2]);
            out.h = fv[0];
            out.hu = fv[1];
            out.hv = fv[2];
            out.z = fv[3];
            out.nm = fv[4];
            set_vel_t<M>(out, kp);
            issue(qi + kRing);
        };
#pragma unroll
        for (int qi = 0; qi < kRing; ++qi) issue(qi);

        CellT<float2> Ab, Bb;
        float2 yT0, yT1, yT2;
        consume(0, Ab);  // row r0-1
        consume(1, Bb);  // row r0
        {
            const FaceT<float2> f = face_t<0, M, MASKED>(Ab, Bb, kp);
            yT0 = f.f0;
            yT1 = f.f1;
            yT2 = A::add(f.f2, f.corr_hi);
            if (RUN && r0 == 0) {
                if (valid.x) acc.outflow -= dtd * (double)f.f0.x * d.dx;
                if (valid.y) acc.outflow -= dtd * (double)f.f0.y * d.dx;
            }
        }
        consume(2, Ab);  // row r0+1

        auto row = [&](const int r, CellT<float2>& cur, CellT<float2>& nxt) {
            const int j = (r - r0) & (kBatch - 1);
            if (j == 0) {
                // Strip edges for rows r .. r+31, one row per lane.
                __syncwarp();
                const int rr = min(r + lane, d.rows - 1);
                Cell L[1], E[1], R[1];
                load_cells<1>(d, in, rr, x0w - 1, L);
                load_cells<1>(d, in, rr, x0w, E);
                load_cells<1>(d, in, rr, x0w + kWarp * V, R);
                CellT<float> l{L[0].h, L[0].hu, L[0].hv, L[0].z, L[0].nm, 0.f, 0.f};
                CellT<float> e{E[0].h, E[0].hu, E[0].hv, E[0].z, E[0].nm, 0.f, 0.f};
                CellT<float> q{R[0].h, R[0].hu, R[0].hv, R[0].z, R[0].nm, 0.f, 0.f};
                set_vel_t<M>(l, ks);
                set_vel_t<M>(e, ks);
                set_vel_t<M>(q, ks);
                const FaceT<float> f = face_t<1, M, MASKED>(l, e, ks);
                sm.left[0][lane] = f.f0;
                sm.left[1][lane] = A::add(f.f1, f.corr_hi);
                sm.left[2][lane] = f.f2;
                if (RUN && x0w == 0 && r + lane < r1) acc.outflow -= dtd * (double)f.f0 * d.dy;
                sm.right[0][lane] = q.h;
                sm.right[1][lane] = q.hu;
                sm.right[2][lane] = q.hv;
                sm.right[3][lane] = q.z;
                sm.right[4][lane] = q.nm;
                sm.right[5][lane] = q.u;
                sm.right[6][lane] = q.v;
                __syncwarp();
            }

            // y-faces above both columns: lo side for row r, hi side carried to row r+1.
            const FaceT<float2> fy = face_t<0, M, MASKED>(cur, nxt, kp);
            const float2 yB0 = fy.f0, yB1 = fy.f1, yB2 = A::add(fy.f2, fy.corr_lo);
            const float2 yN2 = A::add(fy.f2, fy.corr_hi);
            if (RUN && r == d.rows - 1) {
                if (valid.x) acc.outflow += dtd * (double)fy.f0.x * d.dx;
                if (valid.y) acc.outflow += dtd * (double)fy.f0.y * d.dx;
            }

            // x-faces: (cell 0 | cell 1) and (cell 1 | first cell of the next lane).
            float rh = __shfl_down_sync(0xffffffffu, cur.h.x, 1);
            float rhu = __shfl_down_sync(0xffffffffu, cur.hu.x, 1);
            float rhv = __shfl_down_sync(0xffffffffu, cur.hv.x, 1);
            float rz = __shfl_down_sync(0xffffffffu, cur.z.x, 1);
            float rnm = __shfl_down_sync(0xffffffffu, cur.nm.x, 1);
            float ru = __shfl_down_sync(0xffffffffu, cur.u.x, 1);
            float rv = __shfl_down_sync(0xffffffffu, cur.v.x, 1);
            {
                const float e0 = sm.right[0][j], e1 = sm.right[1][j], e2 = sm.right[2][j];
                const float e3 = sm.right[3][j], e4 = sm.right[4][j], e5 = sm.right[5][j];
                const float e6 = sm.right[6][j];
                if (lane == 31) {
                    rh = e0; rhu = e1; rhv = e2; rz = e3; rnm = e4; ru = e5; rv = e6;
                }
            }
            CellT<float2> xhi;
            xhi.h = f2(cur.h.y, rh);
            xhi.hu = f2(cur.hu.y, rhu);
            xhi.hv = f2(cur.hv.y, rhv);
            xhi.z = f2(cur.z.y, rz);
            xhi.nm = f2(cur.nm.y, rnm);
            xhi.u = f2(cur.u.y, ru);
            xhi.v = f2(cur.v.y, rv);
            const FaceT<float2> fx = face_t<1, M, MASKED>(cur, xhi, kp);
            const float2 xl0 = fx.f0, xl1 = A::add(fx.f1, fx.corr_lo), xl2 = fx.f2;
            const float2 xh1 = A::add(fx.f1, fx.corr_hi);
            float up0 = __shfl_up_sync(0xffffffffu, fx.f0.y, 1);
            float up1 = __shfl_up_sync(0xffffffffu, xh1.y, 1);
            float up2 = __shfl_up_sync(0xffffffffu, fx.f2.y, 1);
            {
                const float l0 = sm.left[0][j], l1 = sm.left[1][j], l2 = sm.left[2][j];
                if (lane == 0) {
                    up0 = l0; up1 = l1; up2 = l2;
                }
            }
            const float2 xr0 = f2(up0, fx.f0.x), xr1 = f2(up1, xh1.x), xr2 = f2(up2, fx.f2.x);
            if (RUN && (right_edge == 0 || right_edge == 1))
                acc.outflow += dtd * (double)(right_edge == 0 ? fx.f0.x : fx.f0.y) * d.dy;

            // Cell updates of both columns.
            const auto act = MASKED ? act_of(cur.nm) : all_true<float2>();
            const float2 n2 = MASKED ? vabs(cur.nm) : cur.nm;
            float2 u0, u1, u2;
            if constexpr (A::kExact) {
                u0 = A::sub(cur.h, A::mul(dt2, A::add(A::div(A::sub(xl0, xr0), dx2), A::div(A::sub(yB0, yT0), dy2))));
                u1 = A::sub(cur.hu, A::mul(dt2, A::add(A::div(A::sub(xl1, xr1), dx2), A::div(A::sub(yB1, yT1), dy2))));
                u2 = A::sub(cur.hv, A::mul(dt2, A::add(A::div(A::sub(xl2, xr2), dx2), A::div(A::sub(yB2, yT2), dy2))));
            } else {
                u0 = A::fma(ndtdx2, A::sub(xl0, xr0), A::fma(ndtdy2, A::sub(yB0, yT0), cur.h));
                u1 = A::fma(ndtdx2, A::sub(xl1, xr1), A::fma(ndtdy2, A::sub(yB1, yT1), cur.hu));
                u2 = A::fma(ndtdx2, A::sub(xl2, xr2), A::fma(ndtdy2, A::sub(yB2, yT2), cur.hv));
            }
            float2 rain;
            if (d.mult != nullptr) {
                const int64_t mo = (int64_t)r * d.spitch;
                const float m0 = __ldg(d.mult + mo + min(c0, d.cols - 1));
                const float m1 = __ldg(d.mult + mo + min(c0 + 1, d.cols - 1));
                rain = A::mul(dtr2, f2(m0, m1));
            } else {
                rain = sel(act, dtr2, kp.zero);
            }
            u0 = A::add(u0, rain);
            const float2 h = vmax(u0, kp.zero);
            float2 qx, qy;
            if constexpr (A::kExact) {
                const float2 norm = A::hypot(u1, u2);
                const float2 fr = A::div(A::mul(A::mul(dtg2, n2), norm), A::pow73(vmax(h, kp.dry), k.expo));
                const float2 den = A::add(kp.one, fr);
                qx = A::div(u1, den);
                qy = A::div(u2, den);
            } else {
                const float2 norm = A::sqrt(A::fma(u1, u1, A::mul(u2, u2)));
                const float2 hm = A::ex2(A::mul(A::lg2(vmax(h, kp.dry)), nexpo2));  // max(h,dry)^(-7/3)
                const float2 fr = A::mul(A::mul(A::mul(dtg2, n2), norm), hm);
                const float2 rd = A::rcp(A::add(kp.one, fr));
                qx = A::mul(u1, rd);
                qy = A::mul(u2, rd);
            }
            const auto wet = act & gt(h, kp.dry);
            const float2 ho = sel(act, h, kp.zero);
            const float2 huo = sel(wet, qx, kp.zero);
            const float2 hvo = sel(wet, qy, kp.zero);
            if constexpr (RUN) {
                CellT<float2> nc;
                nc.h = ho;
                nc.hu = huo;
                nc.hv = hvo;
                set_vel_t<M>(nc, kp);
                const float2 w = A::sqrt(A::mul(kp.g, ho));
                float2 inv;
                if constexpr (A::kExact) {
                    inv = A::add(A::div(A::add(vabs(nc.u), w), dx2), A::div(A::add(vabs(nc.v), w), dy2));
                } else {
                    inv = A::fma(A::add(vabs(nc.u), w), rdx2, A::mul(A::add(vabs(nc.v), w), rdy2));
                }
                const auto use = act & valid;
                acc.maxinv = nan_max(acc.maxinv, use.x ? inv.x : 0.0f);
                acc.maxinv = nan_max(acc.maxinv, use.y ? inv.y : 0.0f);
                acc.vol += (double)(valid.x ? ho.x : 0.0f) + (double)(valid.y ? ho.y : 0.0f);
                if (d.mult != nullptr) {
                    acc.rain += (double)(valid.x ? rain.x : 0.0f) + (double)(valid.y ? rain.y : 0.0f);
                } else {
                    acc.rain_cells += (use.x ? 1u : 0u) + (use.y ? 1u : 0u);
                }
                if (valid.x && u0.x < 0.0f) acc.clip -= (double)u0.x;
                if (valid.y && u0.y < 0.0f) acc.clip -= (double)u0.y;
                if (MASKED) {
                    if (valid.x && !act.x) acc.mask += (double)h.x;
                    if (valid.y && !act.y) acc.mask += (double)h.y;
                }
            }
            const int64_t so = (int64_t)r * out.pitch;
            if (c0 + 2 <= d.cols) {
                *reinterpret_cast<float2*>(out.h + so + c0) = ho;
                *reinterpret_cast<float2*>(out.hu + so + c0) = huo;
                *reinterpret_cast<float2*>(out.hv + so + c0) = hvo;
            } else if (valid.x) {
                out.h[so + c0] = ho.x;
                out.hu[so + c0] = huo.x;
                out.hv[so + c0] = hvo.x;
            }
            if (RUN && snap >= 0) {
                const Control* c = ctl;
                const int64_t base = (int64_t)snap * c->out_plane + (int64_t)r * d.cols + c0;
                if (valid.x) {
                    c->out_h[base] = ho.x;
                    c->out_hu[base] = huo.x;
                    c->out_hv[base] = hvo.x;
                }
                if (valid.y) {
                    c->out_h[base + 1] = ho.y;
                    c->out_hu[base + 1] = huo.y;
                    c->out_hv[base + 1] = hvo.y;
                }
            }
            yT0 = fy.f0;
            yT1 = fy.f1;
            yT2 = yN2;
            // Row r+2 takes over the registers row r leaves free.
            if (r + 1 < r1) consume(r + 3 - r0, cur);
        };

        for (int r = r0; r < r1; r += 2) {
            row(r, Bb, Ab);
            if (r + 1 < r1) row(r + 1, Ab, Bb);
        }
        cp_async_wait<0>();  // nothing may land after the warp is done
    }
}

template <class M, int THREADS, bool RUN, bool MASKED>
__global__ void __launch_bounds__(THREADS, SWE_PAIR_MINBLOCKS) step_kernel_pair(const StepLaunch p) {
    constexpr int NW = THREADS / kWarp;
    __shared__ WarpSmem s_warp[NW];
    const DomainDev& d = p.d;
    StepScalars s = p.s;
    int snap = -1;
    double dtd = 0.0;
    if constexpr (RUN) {
        const Control* c = p.ctl;
        if (*((volatile const int*)&c->done)) return;  // uniform early exit of the whole grid
        s = c->s;
        snap = c->snap;
        dtd = c->dt;
    }
    const int wib = threadIdx.x >> 5;
    const int gw = blockIdx.x * NW + wib;
    const int strip = gw % p.nstrips;
    const int chunk = gw / p.nstrips;
    const int r0 = chunk * p.rows_per_warp;
    const int r1 = min(r0 + p.rows_per_warp, d.rows);
    StepAccum acc;
    acc.zero();
    if (r0 < d.rows)
        march_pair<M, RUN, MASKED>(d, p.in, p.out, s, snap, dtd, p.ctl, r0, r1, strip * kWarp * 2,
                                   s_warp[wib], acc);
    if constexpr (RUN) {
        Accum a;
        a.maxinv = acc.maxinv;
        a.vol = acc.vol;
        a.rain = acc.rain + (double)acc.rain_cells * (double)s.dt_rain;
        a.outflow = acc.outflow;
        a.clip = acc.clip;
        a.mask = acc.mask;
        finish_run_step<THREADS>(d, p.ctl, p.parts, a, false);
    }
}


// ---------------------------------------------------------------------------
// Batched ensemble: many domains of uneven size, one launch per step
// ---------------------------------------------------------------------------
// Each member is a complete domain (its own static planes, ping-pong state,
// run control with float64 clock, CFL dt and mass ledger).  The launch's CTAs
// are persistent: CTA b takes work items b, b + gridDim.x, ...; an item is one
// CTA's worth of warps of one member (item.y = its slot among the member's
// `ncta` slots).  After its march the CTA folds into that member's partials and
// the member's last slot advances the member's clock and plans its next dt, so
// members step with their own CFL dt and finish independently (a finished
// member's items return at once).
struct MemberDev {
    DomainDev d;
    float* buf[2][3];  // ping-pong h, hu, hv planes
    int64_t pitch;
    Control* ctl;
    Partial* parts;
    int nstrips, rows_per_warp, ncta;
};

template <class M, int THREADS, bool MASKED>
__global__ void __launch_bounds__(THREADS, SWE_PAIR_MINBLOCKS)
ensemble_step_kernel(const MemberDev* __restrict__ members, const int2* __restrict__ items,
                     int n_items, int parity) {
    constexpr int NW = THREADS / kWarp;
    __shared__ WarpSmem s_warp[NW];
    __shared__ MemberDev s_md;
    const int wib = threadIdx.x >> 5;
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const int2 item = items[it];
        const Control* c = members[item.x].ctl;
        if (*((volatile const int*)&c->done)) continue;  // uniform for the CTA
        __syncthreads();  // the previous item is done with s_md
        if (threadIdx.x == 0) s_md = members[item.x];
        __syncthreads();
        const MemberDev& md = s_md;
        const StepScalars s = c->s;
        const int snap = c->snap;
        const double dtd = c->dt;
        const int gw = item.y * NW + wib;
        const int strip = gw % md.nstrips;
        const int chunk = gw / md.nstrips;
        const int r0 = chunk * md.rows_per_warp;
        const int r1 = min(r0 + md.rows_per_warp, md.d.rows);
        const StateView in{md.buf[parity][0], md.buf[parity][1], md.buf[parity][2], md.pitch};
        const StateOut out{md.buf[parity ^ 1][0], md.buf[parity ^ 1][1], md.buf[parity ^ 1][2], md.pitch};
        StepAccum acc;
        acc.zero();
        if (r0 < md.d.rows)
            march_pair<M, true, MASKED>(md.d, in, out, s, snap, dtd, md.ctl, r0, r1, strip * kWarp * 2,
                                        s_warp[wib], acc);
        Accum a;
        a.maxinv = acc.maxinv;
        a.vol = acc.vol;
        a.rain = acc.rain + (double)acc.rain_cells * (double)s.dt_rain;
        a.outflow = acc.outflow;
        a.clip = acc.clip;
        a.mask = acc.mask;
        finish_run_step<THREADS>(md.d, md.ctl, md.parts, a, false, false, item.y, md.ncta);
    }
}

}  // namespace swe
