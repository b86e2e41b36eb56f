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
// edge copy zero bytes; their cells are filled from the last column (ghost
// ring).
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

constexpr int kRing = 4;  // rows in flight per warp (a power of two)


#ifndef SWE_PAIR_MINBLOCKS
#define SWE_PAIR_MINBLOCKS 4
#endif

// Warp-private shared memory of the march: strip edges of the current 32-row
// batch and the cp.async row ring.
struct WarpSmem {
    float left[3][kWarp];      // hi side of the strip's left x-face, per batch row
    float right[5][kWarp];     // the cell right of the strip per batch row: h, z, n^2, u, v
    float2 ring[kRing][5][kWarp];  // [slot][field][lane]
    double led[5][kWarp];      // float64 ledger sums per lane (vol, rain, clip, mask, outflow)
    alignas(16) double old[4]; // the warp's ledger slot as the step found it (run mode)
};

__device__ __forceinline__ void cp_async_8z(void* dst, const void* src, int src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src), "r"(src_bytes)
                 : "memory");
}

// What a march needs from its step's plan: the float32 scalars, the snapshot
// index, the float64 dt and whether the step runs at all.
struct MarchPlan {
    StepScalars s;
    int snap;
    double dtd;
    int go;
};

// Ledger accumulation (float partials of diagnostics, not step arithmetic): packed FMA in both policies.
__device__ __forceinline__ float2 lfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// One warp marches rows [r0, r1) of the 64-column strip starting at x0w: every
// face once, cells updated, row r written to `out` (and to snapshot `snap` of
// `ctl` in run mode); CFL maximum and ledger terms accumulate into `acc`.
//
// The row body has no data-dependent branch: partial lanes and boundary fluxes
// are handled by per-lane float masks, ghost rows by a sign factor, and the
// ring copies by their source size (zero bytes past the chunk or the right
// edge).  The ledger terms accumulate as float partials over at most one
// 32-row batch and are folded into the float64 accumulators per batch.
//
// LAST_CONSUME: the last row also consumes (zero-byte copies past the chunk,
// values unused), which keeps the row body free of that branch; the plain step
// measured 0.6 % faster with it, the ensemble kernel spills with it.
//
// EDGES (the plain run-mode step): with epar >= 0, the domain keeps its
// strip-boundary columns (DomainDev::edge) and `in` is ping-pong buffer epar.
// The strip edges are then read from edge[epar] where the neighbouring cells
// lie inside the grid (one coalesced access per quantity for 32 rows, where
// the state would need one cache line per row), and lanes 0 and 31 write the
// strip's first and last columns of `out` into edge[epar ^ 1] for the next
// step.  In fast arithmetic the 2048^2 step measured 7 % faster with it and
// the ensemble of 16 x 1024^2 members (114-row marches) 6 % (the 64-member mix,
// 256-row marches, the same); in exact arithmetic (more registers) it spilled
// and measured 1.5 % slower, so exact marches load their edges from the state.
static_assert(kEdgeStrip == 2 * kWarp, "a paired-march strip is 2 x 32 columns");

template <class M, bool RUN, bool MASKED, bool LAST_CONSUME, bool EDGES, class PlanFn>
__device__ __forceinline__ bool march_pair(const DomainDev& d, const StateView& in,
                                            const StateOut& out, PlanFn&& plan_fn, const Control* ctl,
                                            int r0, int r1, int x0w, WarpSmem& sm, StepAccum& acc, int epar = -1) {
    constexpr int kBatch = kWarp;
    using A = P<M>;
    const Consts& k = d.k;
    const KPair kp = make_kpair(k);
    const KScalar ks = make_kscalar(k);
    const int lane = threadIdx.x & 31;
    const int c0 = x0w + lane * 2;
    const B2 valid{c0 < d.cols, c0 + 1 < d.cols};
    const float2 vmask = f2(valid.x ? 1.f : 0.f, valid.y ? 1.f : 0.f);
    // The component holding the last column: its right x-face is the east boundary.
    const float2 emask = f2(c0 == d.cols - 1 ? 1.f : 0.f, c0 + 1 == d.cols - 1 ? 1.f : 0.f);
    // The step's dt and everything made from it are known once the plan is
    // (after the march's first loads are in flight).
    float2 dt2, dtr2, dtg2, ndtdx2, ndtdy2;
    int snap = -1;
    double dtd = 0.0;
    const float2 dx2 = splat(k.dx), dy2 = splat(k.dy);
    const float rdx = 1.0f / k.dx, rdy = 1.0f / k.dy;
    const float2 rdx2 = splat(rdx), rdy2 = splat(rdy);
    const float2 nexpo2 = splat(-k.expo);
    // Exact arithmetic divides by dx and dy as the reference does; when both are
    // powers of two that is the multiplication by their (exact) reciprocals, the
    // same correctly rounded result (a warp-uniform branch).
    const bool pow2 = k.pow2 != 0;
    const float2 rdxe = splat(__frcp_rn(k.dx)), rdye = splat(__frcp_rn(k.dy));
    auto over_dx = [&](float2 a) {
        if constexpr (A::kExact) return pow2 ? A::mul(a, rdxe) : A::div(a, dx2);
        else return A::mul(a, rdxe);  // not used by the fast policy
    };
    auto over_dy = [&](float2 a) {
        if constexpr (A::kExact) return pow2 ? A::mul(a, rdye) : A::div(a, dy2);
        else return A::mul(a, rdye);
    };
    // This lane's column run of the next step's edges (lanes 0 and 31), or null.
    float* ep = nullptr;
    if (EDGES && epar >= 0) {
        const int eb = x0w / kEdgeStrip;
        if (lane == 0) ep = d.edge[epar ^ 1] + edge_index(d, eb, 3, 0);
        else if (lane == kWarp - 1 && valid.y) ep = d.edge[epar ^ 1] + edge_index(d, eb + 1, 0, 0);
    }
    const int nq = r1 - r0 + 2;  // rows r0-1 .. r1 pass through the ring
    const bool edge_strip = x0w + kWarp * 2 > d.cols;
    const int csize = valid.y ? 8 : (valid.x ? 4 : 0);
    const int ccol = csize ? c0 : 0;  // copy source column (any aligned in-grid column when nothing is read)

    // Start the copies of ring row qi (row r0-1+qi, clamped to the grid): one group per row,
    // zero bytes past the chunk or the right edge, so the issue path has no branch.
    auto issue = [&](int qi) {
        const int q = r0 - 1 + qi;
        const int rr = min(max(q, 0), d.rows - 1);
        const int sz = qi < nq ? csize : 0;
        const int slot = qi & (kRing - 1);
        // 32-bit element offsets: planes hold fewer than 2^31 elements (checked on the host).
        const uint32_t so = (uint32_t)rr * (uint32_t)in.pitch + (uint32_t)ccol;
        const uint32_t zo = (uint32_t)rr * (uint32_t)d.spitch + (uint32_t)ccol;
        cp_async_8z(&sm.ring[slot][0][lane], in.h + so, sz);
        cp_async_8z(&sm.ring[slot][1][lane], in.hu + so, sz);
        cp_async_8z(&sm.ring[slot][2][lane], in.hv + so, sz);
        cp_async_8z(&sm.ring[slot][3][lane], d.bed + zo, sz);
        cp_async_8z(&sm.ring[slot][4][lane], d.nm + zo, sz);
        cp_async_commit();
    };
    // Ring row qi into registers, ghost ring applied; its slot is refilled with row qi+kRing.
    auto consume = [&](int qi, CellT<float2>& c) {
        cp_async_wait<kRing - 1>();
        const int slot = qi & (kRing - 1);
        const int q = r0 - 1 + qi;
        float2 fv[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) fv[f] = sm.ring[slot][f][lane];
        if (edge_strip) {
            __syncwarp();  // the last column may sit in another lane's slot
            const int last = d.cols - 1 - x0w;
            const float* lastp = reinterpret_cast<const float*>(&sm.ring[slot][0][0]);
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
        c.h = fv[0];
        c.hu = fv[1];
        c.hv = fv[2];
        // Ghost rows (q is the same on every lane): a reflective edge mirrors hv.
        if (q < 0 || q >= d.rows) {
            if ((q < 0 ? d.bnd[2] : d.bnd[3]) == 0) c.hv = neg(c.hv);
        }
        c.z = fv[3];
        c.nm = fv[4];
        set_vel_t<M>(c, kp);
        issue(qi + kRing);
    };

    struct {
        float2 vol, rain, clip, mask, out_x, out_y;
    } lg;
    auto zero_ledger = [&]() { lg.vol = lg.rain = lg.clip = lg.mask = lg.out_x = lg.out_y = kp.zero; };
    zero_ledger();
    float maxinv = 0.f;
    // Float ledger partials cover at most one 32-row batch (64 cells per term), then go to float64.
    // The float64 sums live in the warp's shared memory during the march, so
    // that they hold no registers; they return to `acc` at the end.
    if constexpr (RUN) {
#pragma unroll
        for (int q = 0; q < 5; ++q) sm.led[q][lane] = 0.0;
    }
    auto flush_ledger = [&]() {
        if constexpr (RUN) {
            sm.led[0][lane] += (double)lg.vol.x + (double)lg.vol.y;
            sm.led[1][lane] += (double)lg.rain.x + (double)lg.rain.y;
            sm.led[2][lane] += (double)lg.clip.x + (double)lg.clip.y;
            sm.led[3][lane] += (double)lg.mask.x + (double)lg.mask.y;
            sm.led[4][lane] += dtd * ((double)(lg.out_x.x + lg.out_x.y) * d.dy + (double)(lg.out_y.x + lg.out_y.y) * d.dx);
            zero_ledger();
        }
    };

#pragma unroll
    for (int qi = 0; qi < kRing; ++qi) issue(qi);

    CellT<float2> R0, R1;
    float2 yT0, yT1, yT2;

    // The x-faces of a row: (cell 0 | cell 1) and (cell 1 | first cell of the next lane).
    // Returns the lo-side fluxes of both cells' left faces and the hi-side of their right faces.
    struct XF {
        float2 l0, l1, l2;  // flux entering through each cell's left face (hi side of that face)
        float2 r0, r1, r2;  // flux leaving through each cell's right face (lo side)
        float2 e0;          // mass flux through each cell's right face (east outflow)
    };
    auto xfaces = [&](const CellT<float2>& cur, int j) -> XF {
        // The face reads depth, bed and velocities of its two cells (and n^2 for
        // the mask): the neighbour's momenta are not moved.
        float rh = __shfl_down_sync(0xffffffffu, cur.h.x, 1);
        float rz = __shfl_down_sync(0xffffffffu, cur.z.x, 1);
        float rnm = MASKED ? __shfl_down_sync(0xffffffffu, cur.nm.x, 1) : 0.f;
        float ru = __shfl_down_sync(0xffffffffu, cur.u.x, 1);
        float rv = __shfl_down_sync(0xffffffffu, cur.v.x, 1);
        if (lane == 31) {
            rh = sm.right[0][j]; rz = sm.right[1][j]; ru = sm.right[3][j]; rv = sm.right[4][j];
            if (MASKED) rnm = sm.right[2][j];
        }
        CellT<float2> xhi;
        xhi.h = f2(cur.h.y, rh);
        xhi.hu = kp.zero;
        xhi.hv = kp.zero;
        xhi.z = f2(cur.z.y, rz);
        xhi.nm = f2(cur.nm.y, rnm);
        xhi.u = f2(cur.u.y, ru);
        xhi.v = f2(cur.v.y, rv);
        const FaceT<float2> fx = face_t<1, M, MASKED>(cur, xhi, kp);
        const float2 xh1 = A::add(fx.f1, fx.corr_hi);
        float up0 = __shfl_up_sync(0xffffffffu, fx.f0.y, 1);
        float up1 = __shfl_up_sync(0xffffffffu, xh1.y, 1);
        float up2 = __shfl_up_sync(0xffffffffu, fx.f2.y, 1);
        if (lane == 0) {
            up0 = sm.left[0][j]; up1 = sm.left[1][j]; up2 = sm.left[2][j];
        }
        XF x;
        x.r0 = fx.f0;
        x.r1 = A::add(fx.f1, fx.corr_lo);
        x.r2 = fx.f2;
        x.l0 = f2(up0, fx.f0.x);
        x.l1 = f2(up1, xh1.x);
        x.l2 = f2(up2, fx.f2.x);
        x.e0 = fx.f0;
        return x;
    };

    struct Row {
        float2 h, hu, hv;
    };
    // Cell update of one row from its faces: bottom (b*), top (t*, lo side), x-faces.
    auto update = [&](int r, const CellT<float2>& cur, float2 b0, float2 b1, float2 b2, float2 t0, float2 t1,
                      float2 t2, const XF& x) -> Row {
        const auto act = MASKED ? act_of(cur.nm) : all_true<float2>();
        const float2 n2 = MASKED ? vabs(cur.nm) : cur.nm;
        float2 u0, u1, u2;
        if constexpr (A::kExact) {
            u0 = A::sub(cur.h, A::mul(dt2, A::add(over_dx(A::sub(x.r0, x.l0)), over_dy(A::sub(t0, b0)))));
            u1 = A::sub(cur.hu, A::mul(dt2, A::add(over_dx(A::sub(x.r1, x.l1)), over_dy(A::sub(t1, b1)))));
            u2 = A::sub(cur.hv, A::mul(dt2, A::add(over_dx(A::sub(x.r2, x.l2)), over_dy(A::sub(t2, b2)))));
        } else {
            u0 = A::fma(ndtdx2, A::sub(x.r0, x.l0), A::fma(ndtdy2, A::sub(t0, b0), cur.h));
            u1 = A::fma(ndtdx2, A::sub(x.r1, x.l1), A::fma(ndtdy2, A::sub(t1, b1), cur.hu));
            u2 = A::fma(ndtdx2, A::sub(x.r2, x.l2), A::fma(ndtdy2, A::sub(t2, b2), cur.hv));
        }
        float2 rain = sel(act, dtr2, kp.zero);
        if (d.mult != nullptr) {
            const int64_t mo = (int64_t)r * d.spitch;
            rain = A::mul(dtr2, f2(__ldg(d.mult + mo + min(c0, d.cols - 1)), __ldg(d.mult + mo + min(c0 + 1, d.cols - 1))));
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
        Row o;
        o.h = sel(act, h, kp.zero);
        o.hu = sel(wet, qx, kp.zero);
        o.hv = sel(wet, qy, kp.zero);
        if constexpr (RUN) {
            const float2 w = A::sqrt(A::mul(kp.g, o.h));
            float2 inv;
            if constexpr (A::kExact) {
                CellT<float2> nc;
                nc.h = o.h;
                nc.hu = o.hu;
                nc.hv = o.hv;
                set_vel_t<M>(nc, kp);
                inv = A::add(over_dx(A::add(vabs(nc.u), w)), over_dy(A::add(vabs(nc.v), w)));
            } else {
                // The new momenta are zero wherever h <= dry, so 1/max(h, dry) gives the
                // same velocities as the dry-cell rule of the reference.
                const float2 rh = A::rcp(vmax(o.h, kp.dry));
                inv = A::fma(A::add(vabs(A::mul(o.hu, rh)), w), rdx2, A::mul(A::add(vabs(A::mul(o.hv, rh)), w), rdy2));
            }
            // Inactive cells have h = hu = hv = 0 and so inv = 0; lanes past the edge are masked.
            inv = A::mul(inv, vmask);
            // Maximum without the NaN test per cell: a NaN or infinite inverse dt
            // turns the float volume partial into NaN (0 * NaN, 0 * inf), and the
            // fold reports the step as non-finite.
            maxinv = fmaxf(maxinv, fmaxf(inv.x, inv.y));
            lg.vol = lfma(inv, kp.zero, lfma(o.h, vmask, lg.vol));
            if (d.mult != nullptr) lg.rain = lfma(rain, vmask, lg.rain);
            lg.clip = lfma(neg(vmin(u0, kp.zero)), vmask, lg.clip);
            if constexpr (MASKED) {
                lg.mask = lfma(sel(act, kp.zero, h), vmask, lg.mask);
                if (d.mult == nullptr) acc.rain_cells += (act.x && valid.x ? 1u : 0u) + (act.y && valid.y ? 1u : 0u);
            }
            lg.out_x = lfma(x.e0, emask, lg.out_x);
        }
        return o;
    };
    auto store = [&](int r, const Row& o) {
        const uint32_t so = (uint32_t)r * (uint32_t)out.pitch + (uint32_t)c0;
        if (valid.y) {
            *reinterpret_cast<float2*>(out.h + so) = o.h;
            *reinterpret_cast<float2*>(out.hu + so) = o.hu;
            *reinterpret_cast<float2*>(out.hv + so) = o.hv;
        } else if (valid.x) {
            out.h[so] = o.h.x;
            out.hu[so] = o.hu.x;
            out.hv[so] = o.hv.x;
        }
        if (EDGES && ep != nullptr) {
            const bool first = lane == 0;
            ep[r] = first ? o.h.x : o.h.y;
            ep[r + d.edge_rows] = first ? o.hu.x : o.hu.y;
            ep[r + 2 * d.edge_rows] = first ? o.hv.x : o.hv.y;
        }
        if (RUN && snap >= 0) {
            const Control* c = ctl;
            const int64_t base = (int64_t)snap * c->out_plane + (int64_t)r * d.cols + c0;
            if (valid.x) {
                c->out_h[base] = o.h.x;
                c->out_hu[base] = o.hu.x;
                c->out_hv[base] = o.hv.x;
            }
            if (valid.y) {
                c->out_h[base + 1] = o.h.y;
                c->out_hu[base + 1] = o.hu.y;
                c->out_hv[base + 1] = o.hv.y;
            }
        }
    };
    // Strip edges for rows rb .. rb+31, one row per lane (the left x-face and the right halo cell).
    auto batch = [&](int rb) {
        __syncwarp();
        const int rr = min(rb + lane, d.rows - 1);
        Cell L[1], E[1], Q[1];
        const int b = x0w / kEdgeStrip;
        const float* ein = EDGES && epar >= 0 ? d.edge[epar] : nullptr;
        if (EDGES && ein != nullptr && x0w > 0) {
            L[0] = {__ldg(ein + edge_index(d, b, 0, rr)), __ldg(ein + edge_index(d, b, 1, rr)),
                    __ldg(ein + edge_index(d, b, 2, rr)), __ldg(d.edge_static + edge_static_index(d, b, 0, rr)),
                    __ldg(d.edge_static + edge_static_index(d, b, 1, rr)), 0.f, 0.f};
            E[0] = {__ldg(ein + edge_index(d, b, 3, rr)), __ldg(ein + edge_index(d, b, 4, rr)),
                    __ldg(ein + edge_index(d, b, 5, rr)), __ldg(d.edge_static + edge_static_index(d, b, 2, rr)),
                    __ldg(d.edge_static + edge_static_index(d, b, 3, rr)), 0.f, 0.f};
        } else {
            load_cells<1>(d, in, rr, x0w - 1, L);
            load_cells<1>(d, in, rr, x0w, E);
        }
        if (EDGES && ein != nullptr && x0w + kEdgeStrip < d.cols) {
            Q[0] = {__ldg(ein + edge_index(d, b + 1, 3, rr)), __ldg(ein + edge_index(d, b + 1, 4, rr)),
                    __ldg(ein + edge_index(d, b + 1, 5, rr)), __ldg(d.edge_static + edge_static_index(d, b + 1, 2, rr)),
                    __ldg(d.edge_static + edge_static_index(d, b + 1, 3, rr)), 0.f, 0.f};
        } else {
            load_cells<1>(d, in, rr, x0w + kWarp * 2, Q);
        }
        CellT<float> l{L[0].h, L[0].hu, L[0].hv, L[0].z, L[0].nm, 0.f, 0.f};
        CellT<float> e{E[0].h, E[0].hu, E[0].hv, E[0].z, E[0].nm, 0.f, 0.f};
        CellT<float> q{Q[0].h, Q[0].hu, Q[0].hv, Q[0].z, Q[0].nm, 0.f, 0.f};
        set_vel_t<M>(l, ks);
        set_vel_t<M>(e, ks);
        set_vel_t<M>(q, ks);
        const FaceT<float> f = face_t<1, M, MASKED>(l, e, ks);
        sm.left[0][lane] = f.f0;
        sm.left[1][lane] = A::add(f.f1, f.corr_hi);
        sm.left[2][lane] = f.f2;
        if (RUN && x0w == 0 && rb + lane < r1) lg.out_x.x -= f.f0;
        sm.right[0][lane] = q.h;
        sm.right[1][lane] = q.z;
        sm.right[2][lane] = q.nm;
        sm.right[3][lane] = q.u;
        sm.right[4][lane] = q.v;
        __syncwarp();
    };

    // One row: `cur` is row r, `nxt` row r+1; afterwards `cur` receives row r+2.
    auto row = [&](const int r, const int j, CellT<float2>& cur, const CellT<float2>& nxt) {
        const FaceT<float2> fy = face_t<0, M, MASKED>(cur, nxt, kp);
        const XF x = xfaces(cur, j);
        const Row o = update(r, cur, yT0, yT1, yT2, fy.f0, fy.f1, A::add(fy.f2, fy.corr_lo), x);
        if constexpr (RUN) {
            if (r == d.rows - 1) lg.out_y = lfma(fy.f0, vmask, lg.out_y);
        }
        yT0 = fy.f0;
        yT1 = fy.f1;
        yT2 = A::add(fy.f2, fy.corr_hi);
        store(r, o);
        if (LAST_CONSUME || r + 1 < r1) consume(r + 3 - r0, cur);
    };
    // The first batch's strip edges are loaded before the ring's first rows are
    // waited for, and the step is planned while the ring's rows are in flight,
    // so that the latencies of the march's start overlap.
    batch(r0);
    {
        const MarchPlan mp = plan_fn();
        if (!mp.go) {
            cp_async_wait<0>();
            return false;
        }
        dt2 = splat(mp.s.dt);
        dtr2 = splat(mp.s.dt_rain);
        dtg2 = splat(mp.s.dt_g);
        ndtdx2 = splat(-mp.s.dt * rdx);
        ndtdy2 = splat(-mp.s.dt * rdy);
        snap = mp.snap;
        dtd = mp.dtd;
    }
    consume(0, R1);  // row r0-1
    consume(1, R0);  // row r0
    {
        const FaceT<float2> f = face_t<0, M, MASKED>(R1, R0, kp);
        yT0 = f.f0;
        yT1 = f.f1;
        yT2 = A::add(f.f2, f.corr_hi);
        if constexpr (RUN) {
            if (r0 == 0) lg.out_y = lfma(neg(f.f0), vmask, lg.out_y);
        }
    }
    consume(2, R1);  // row r0+1
    for (int rb = r0; rb < r1; rb += kBatch) {
        flush_ledger();
        if (rb != r0) batch(rb);
        const int re = min(rb + kBatch, r1);
        for (int r = rb; r < re; r += 2) {
            row(r, r - rb, R0, R1);
            if (r + 1 < re) row(r + 1, r + 1 - rb, R1, R0);
        }
    }
    flush_ledger();
    if constexpr (RUN) {
        acc.vol += sm.led[0][lane];
        acc.rain += sm.led[1][lane];
        acc.clip += sm.led[2][lane];
        acc.mask += sm.led[3][lane];
        acc.outflow += sm.led[4][lane];
        acc.maxinv = nan_max(acc.maxinv, maxinv);
        // Without a mask every in-grid cell of every row received dt*rate.
        if (!MASKED && d.mult == nullptr) acc.rain_cells += (unsigned)((valid.x ? 1 : 0) + (valid.y ? 1 : 0)) * (unsigned)(r1 - r0);
    }
    cp_async_wait<0>();  // nothing may land after the warp is done
    return true;
}

template <class M, int THREADS, bool RUN, bool MASKED>
__global__ void __launch_bounds__(THREADS, SWE_PAIR_MINBLOCKS) step_kernel_pair(const StepLaunch p) {
    constexpr int NW = THREADS / kWarp;
    __shared__ WarpSmem s_warp[NW];
    pdl_enter();
    const DomainDev& d = p.d;
    const int wib = threadIdx.x >> 5;
    const int gw = blockIdx.x * NW + wib;
    const int strip = gw % p.nstrips;
    const int chunk = gw / p.nstrips;
    const int r0 = d.upd_lo + chunk * p.rows_per_warp;
    const int r1 = min(r0 + p.rows_per_warp, d.upd_hi);
    StepAccum acc;
    acc.zero();
    if constexpr (RUN) {
        // The slot copy and the plan's loads are in flight while the march
        // starts its own; the plan is made once those are issued.
        ledger_prefetch(&p.slots[gw], s_warp[wib].old);
        cp_async_commit();
        const PlanInputs in = plan_fetch(p.ctl, p.par);
        StepPlan pl;
        auto plan_fn = [&]() -> MarchPlan {
            pl = plan_step(d, in);
            if (blockIdx.x == 0 && wib == 0) lead_advance(p.ctl, p.par, in, pl);
            return MarchPlan{pl.s, pl.snap, pl.dt, pl.go};
        };
        const bool went = r0 < d.upd_hi
                              ? march_pair<M, true, MASKED, true, !P<M>::kExact>(d, p.in, p.out, plan_fn, p.ctl, r0, r1,
                                                                  strip * kWarp * 2, s_warp[wib], acc,
                                                                  d.edge[0] ? p.par : -1)
                              : plan_fn().go != 0;
        if (!went) {  // uniform over the grid: the run has ended
            cp_async_wait<0>();
            return;
        }
        Accum a;
        a.maxinv = acc.maxinv;
        a.vol = acc.vol;
        a.rain = acc.rain + (double)acc.rain_cells * (double)pl.s.dt_rain;
        a.outflow = acc.outflow;
        a.clip = acc.clip;
        a.mask = acc.mask;
        cp_async_wait<0>();
        __syncwarp();
        warp_end_step(p.ctl, &p.slots[gw], s_warp[wib].old, p.par, in.pos.steps, gw % kMaxStripes, a);
    } else {
        if (r0 < d.upd_hi)
            march_pair<M, false, MASKED, true, false>(d, p.in, p.out, [&]() { return MarchPlan{p.s, -1, 0.0, 1}; }, nullptr, r0,
                                         r1, strip * kWarp * 2, s_warp[wib], acc);
    }
}


// ---------------------------------------------------------------------------
// Batched ensemble: many domains of uneven size, one launch per step
// ---------------------------------------------------------------------------
// Each member is a complete domain (its own static planes, ping-pong state,
// run control with float64 clock, CFL dt and mass ledger).  The launch's CTAs
// are persistent: CTA b takes work items b, b + gridDim.x, ...; an item is one
// CTA's worth of warps of one member (its slot among the member's `ncta`
// slots).  Every warp plans its member's step from the member's run position
// and CFL maximum, so members step with their own CFL dt and finish
// independently (a finished member's items return at once); the warps of
// slot 0 lead the member's run position.
struct MemberDev {
    DomainDev d;
    float* buf[2][3];  // ping-pong h, hu, hv planes
    int64_t pitch;
    Control* ctl;
    LedgerSlot* slots;  // ncta * warps per CTA
    int nstrips, rows_per_warp, ncta;
};

// One item of a batched step: warp `wib` of slot `slot` of member `md`.
template <class M, int THREADS, bool MASKED>
__device__ __forceinline__ void ensemble_item(const MemberDev& md, int slot, int par, WarpSmem& sm) {
    constexpr int NW = THREADS / kWarp;
    const int wib = threadIdx.x >> 5;
    const int gw = slot * NW + wib;
    __syncwarp();  // the previous item's slot copy has been read
    ledger_prefetch(&md.slots[gw], sm.old);
    cp_async_commit();
    const PlanInputs pin = plan_fetch(md.ctl, par);
    StepPlan pl;
    auto plan_fn = [&]() -> MarchPlan {
        pl = plan_step(md.d, pin);
        if (slot == 0 && wib == 0) lead_advance(md.ctl, par, pin, pl);
        return MarchPlan{pl.s, pl.snap, pl.dt, pl.go};
    };
    const int strip = gw % md.nstrips;
    const int chunk = gw / md.nstrips;
    const int r0 = chunk * md.rows_per_warp;
    const int r1 = min(r0 + md.rows_per_warp, md.d.rows);
    const StateView in{md.buf[par][0], md.buf[par][1], md.buf[par][2], md.pitch};
    const StateOut out{md.buf[par ^ 1][0], md.buf[par ^ 1][1], md.buf[par ^ 1][2], md.pitch};
    StepAccum acc;
    acc.zero();
    const bool went = r0 < md.d.rows ? march_pair<M, true, MASKED, false, !P<M>::kExact>(md.d, in, out, plan_fn, md.ctl,
                                                                   r0, r1, strip * kWarp * 2, sm, acc,
                                                                   md.d.edge[0] ? par : -1)
                                     : plan_fn().go != 0;
    if (!went) {
        cp_async_wait<0>();
        return;
    }
    Accum a;
    a.maxinv = acc.maxinv;
    a.vol = acc.vol;
    a.rain = acc.rain + (double)acc.rain_cells * (double)pl.s.dt_rain;
    a.outflow = acc.outflow;
    a.clip = acc.clip;
    a.mask = acc.mask;
    cp_async_wait<0>();
    __syncwarp();
    warp_end_step(md.ctl, &md.slots[gw], sm.old, par, pin.pos.steps, gw % kMaxStripes, a);
}

// The ensemble kernel keeps member fields in registers on top of the march.
// At 4 CTAs/SM (128 registers) it spills a few words but, with marches of
// 128-256 rows, is faster than at 3 CTAs/SM without spills (measured on the
// 64-member mix: 97.4 vs 90.0 G cell-updates/s at their best rows per warp).
#ifndef SWE_ENS_MINBLOCKS
#define SWE_ENS_MINBLOCKS 4
#endif
template <class M, int THREADS, bool MASKED>
__global__ void __launch_bounds__(THREADS, SWE_ENS_MINBLOCKS)
ensemble_step_kernel(const MemberDev* __restrict__ members, const int2* __restrict__ items,
                     int n_items, int parity) {
    constexpr int NW = THREADS / kWarp;
    __shared__ WarpSmem s_warp[NW];
    __shared__ MemberDev s_md;
    pdl_enter();
    const int wib = threadIdx.x >> 5;
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const int2 item = items[it];
        __syncthreads();  // the previous item is done with s_md
        if (threadIdx.x == 0) s_md = members[item.x];
        __syncthreads();
        ensemble_item<M, THREADS, MASKED>(s_md, item.y, parity, s_warp[wib]);
    }
}

// The same persistent step with the member table in the kernel's parameter
// space (ensembles of up to kEnsParamMembers members).  A CTA's member index
// and every member field it reads are then uniform values of constant memory,
// which the march reads as operands instead of holding them in registers.
// Work items are numbered member after member; cta_begin[m] is member m's
// first item, so a CTA finds its item's member by walking forward (its items
// ascend).  The warps of a CTA never wait for one another.
constexpr int kEnsParamMembers = 96;
struct EnsParams {
    MemberDev m[kEnsParamMembers];
    int cta_begin[kEnsParamMembers + 1];
    int n_members, n_items, parity;
};

template <class M, int THREADS, bool MASKED>
__global__ void __launch_bounds__(THREADS, SWE_ENS_MINBLOCKS)
ensemble_step_kernel_p(const __grid_constant__ EnsParams p) {
    constexpr int NW = THREADS / kWarp;
    __shared__ WarpSmem s_warp[NW];
    pdl_enter();
    const int wib = threadIdx.x >> 5;
    int member = 0;
    for (int it = blockIdx.x; it < p.n_items; it += gridDim.x) {
        while (it >= p.cta_begin[member + 1]) ++member;
        ensemble_item<M, THREADS, MASKED>(p.m[member], it - p.cta_begin[member], p.parity, s_warp[wib]);
    }
}

}  // namespace swe
