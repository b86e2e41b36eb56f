// C-ABI of the B200 shallow-water step (declared in include/swe_b200.h).
//
// Host side: argument validation with the reference's error conventions,
// packing of the static fields, launch planning, and the run driver.  The run
// driver keeps the float64 clock, dt, output bookkeeping and mass ledger on
// the device (swe::Control); the host enqueues step kernels in chunks and only
// polls a pinned copy of the control block to learn when the run is done.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <time.h>
#include <unistd.h>
#include <nccl.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "swe_b200.h"
#include "swe_step.cuh"
#include "swe_step_pair.cuh"
#include "swe_adjoint.cuh"
#include "swe_hybrid.cuh"
#include "swe_nn.cuh"
#include "swe_gen.cuh"

using namespace swe;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define SWE_CK(expr)                                                                        \
    do {                                                                                    \
        cudaError_t e_ = (expr);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail(SWE_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

constexpr int kThreads = 128;
constexpr int kWarpsPerCta = kThreads / kWarp;

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

// Host restatement of np.interp for the plain-step entry point (float64, the
// same expression order as the device version).
double host_rain_rate(const std::vector<double>& t, const std::vector<double>& r, double dflt,
                      double x) {
    const int n = (int)t.size();
    if (n <= 0) return dflt;
    if (x != x) return x;
    if (x < t[0] || x > t[n - 1]) return dflt;
    if (n == 1 || x == t[n - 1]) return r[n - 1];
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (t[mid] <= x) lo = mid; else hi = mid;
    }
    if (x == t[lo]) return r[lo];
    const volatile double slope = (r[lo + 1] - r[lo]) / (t[lo + 1] - t[lo]);
    const volatile double prod = slope * (x - t[lo]);
    double v = prod + r[lo];
    if (v != v) {
        const volatile double prod2 = slope * (x - t[lo + 1]);
        v = prod2 + r[lo + 1];
        if (v != v && r[lo] == r[lo + 1]) v = r[lo];
    }
    return v;
}

struct Plan {
    int V;
    int nstrips;
    int rows_per_warp;
    int blocks;
};

}  // namespace

struct swe_domain {
    DomainDev dd{};
    int arith = SWE_ARITH_EXACT;
    int device = 0;
    int sms = 148;
    float* bed = nullptr;
    float* nm = nullptr;
    float* mult = nullptr;
    double* rain = nullptr;
    std::vector<double> rain_t, rain_r;
    Control* ctl = nullptr;          // run control (device)
    Control* ctl_scratch = nullptr;  // standalone reductions (device)
    Control* ctl_host = nullptr;     // pinned poll slots [2]
    LedgerSlot* slots = nullptr;  // step warps' ledger slots (kept over a run)
    int slots_cap = 0;            // in CTAs (kWarpsPerCta slots each)
    Partial* rparts = nullptr;     // partials of the standalone CFL/volume reductions
    int rparts_cap = 0;
    float* ping[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
    int64_t ppitch = 0;
    float* edge_buf[2] = {nullptr, nullptr};  // strip-boundary columns per ping buffer (dd.edge)
    float* edge_stat = nullptr;               // their bed and n^2 (dd.edge_static)
    float* times_dev = nullptr;
    int times_cap = 0;
    cudaEvent_t poll_ev[2] = {nullptr, nullptr};
    cudaEvent_t time_ev[2] = {nullptr, nullptr};
    bool timing = false;
    bool timed_valid = false;
    int64_t timed_steps = 0;
    int64_t launches = 0;
    int rows_per_warp_override = 0;
    int run_vec = 2;     // lane width of the run-mode kernel (SWE_RUN_VEC=1|2)
    bool masked = true;  // false when every cell is active (mask-free kernels)
    int occ_cache[2][2] = {{0, 0}, {0, 0}};  // [V-1][run]: CTAs per SM of the step kernels
    float* lupd[3] = {nullptr, nullptr, nullptr};  // adjoint scratch
    int64_t lpitch = 0;
    double* times64_dev = nullptr;  // float64 targets of advance_to
    float* next_scratch = nullptr;  // rollout backward: the output of a segment's last step
    // Rollout backward's second segment buffer, its last-step output, and the
    // stream that recomputes the next segment while the current one is reversed.
    float* seg2 = nullptr;
    int64_t seg2_cap = 0;  // floats
    float* next_scratch2 = nullptr;
    cudaStream_t aux_stream = nullptr;
    cudaEvent_t seg_ev[6] = {};  // start, recomputed[2], reversed[2], end
    double* corr_sums = nullptr;    // volume sums of the residual correction
    float* corr_prov = nullptr;     // provisional-depth plane of the correction
    unsigned* done_counter = nullptr;  // set by an ensemble: shared completion counter
    // swe_run_host: device staging of the recorded outputs and the copy stream.
    float* snap_dev = nullptr;
    int64_t snap_cap = 0;  // floats
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t snap_ev = nullptr;
    // CUDA graphs of 1..kChunk run-mode steps from either ping buffer, and the
    // inputs they were captured with (a change of any of them re-captures them).
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t chunk_graph[2][33] = {};  // [start buffer parity][steps 1..32]
    const LedgerSlot* chunk_graph_slots = nullptr;
    double chunk_graph_rain_scale = 0.0;
    int chunk_graph_rows = 0;
    // Resident run (swe_resident_*): state kept in the ping buffers between calls.
    bool resident = false;
    int64_t resident_steps = 0;  // steps enqueued since swe_resident_load (buffer parity)
    // Row strip of a decomposed domain: its owned global rows and the domain's rows.
    int strip_row_begin = -1, strip_row_end = -1, strip_total_rows = -1;
};

namespace {

// SWE_PDL=1 launches the step kernels with programmatic stream serialisation,
// so that a step's CTAs are placed while the previous step ends (the kernels
// wait for their predecessor with griddepcontrol.wait before touching memory;
// without the attribute that instruction does nothing).  Off by default: the
// one-wave step grid measured 1.3 % faster with ordinary launches inside the
// captured graphs.
bool pdl_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("SWE_PDL");
        return e && e[0] == '1';
    }();
    return on;
}

cudaLaunchConfig_t pdl_config(int blocks, cudaStream_t st) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3((unsigned)kThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    return cfg;
}

void attach_pdl(cudaLaunchConfig_t& cfg, cudaLaunchAttribute* attr) {
    if (!pdl_enabled()) return;
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
}

// Kernel instance for (vector width, arithmetic, run mode, masked) chosen at run time.
// V = 2 runs the paired-lane kernel; V = 1 (pitches or pointers that are not
// 8-byte aligned) the scalar one.
template <int V, class M, bool RUN, bool MASKED>
struct StepK {
    static const void* fn() {
        if constexpr (V == 2)
            return reinterpret_cast<const void*>(&step_kernel_pair<M, kThreads, RUN, MASKED>);
        else
            return reinterpret_cast<const void*>(&step_kernel<V, M, kThreads, RUN, MASKED>);
    }
    static void launch(int blocks, const StepLaunch& sl, cudaStream_t st) {
        cudaLaunchConfig_t cfg = pdl_config(blocks, st);
        cudaLaunchAttribute attr[1];
        attach_pdl(cfg, attr);
        if constexpr (V == 2)
            cudaLaunchKernelEx(&cfg, step_kernel_pair<M, kThreads, RUN, MASKED>, sl);
        else
            cudaLaunchKernelEx(&cfg, step_kernel<V, M, kThreads, RUN, MASKED>, sl);
    }
};

template <class M, bool RUN, bool MASKED, class F>
void dispatch_v(int V, F&& f) {
    if (V == 2) f(StepK<2, M, RUN, MASKED>{}); else f(StepK<1, M, RUN, MASKED>{});
}

template <class F>
void dispatch(int V, int arith, bool run, bool masked, F&& f) {
    if (arith == SWE_ARITH_FAST) {
        if (run) {
            if (masked) dispatch_v<FastMath, true, true>(V, f); else dispatch_v<FastMath, true, false>(V, f);
        } else {
            if (masked) dispatch_v<FastMath, false, true>(V, f); else dispatch_v<FastMath, false, false>(V, f);
        }
    } else {
        if (run) {
            if (masked) dispatch_v<ExactMath, true, true>(V, f); else dispatch_v<ExactMath, true, false>(V, f);
        } else {
            if (masked) dispatch_v<ExactMath, false, true>(V, f); else dispatch_v<ExactMath, false, false>(V, f);
        }
    }
}

// Work items are (strip of 32*V columns) x (chunk of R rows), one per warp.  R is
// chosen so that all warps are resident at once (one full wave at the kernel's
// occupancy), which equalises the work of every SM; chunks keep >= 4 rows.
Plan make_plan(const swe_domain* d, int V, bool run) {
    Plan p;
    p.V = V;
    const int rows = d->dd.upd_hi - d->dd.upd_lo, cols = d->dd.cols;  // the rows the step updates
    p.nstrips = (cols + kWarp * V - 1) / (kWarp * V);
    // The occupancy query costs more than a small step: ask once per kernel instance.
    int& occ = const_cast<swe_domain*>(d)->occ_cache[V - 1][run ? 1 : 0];
    if (occ <= 0) {
        occ = 1;
        auto occ_of = [&](auto k) {
            int n = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, decltype(k)::fn(), kThreads, 0) == cudaSuccess && n > 0)
                occ = n;
        };
        dispatch(V, d->arith, run, d->masked, occ_of);
    }
    const int wpb = kThreads / kWarp;
    const int64_t warps_avail = (int64_t)occ * d->sms * wpb;
    int R = d->rows_per_warp_override;
    if (R <= 0) {
        const int64_t chunks = std::max<int64_t>(1, warps_avail / p.nstrips);
        R = (int)((rows + chunks - 1) / chunks);
        R = std::max(R, std::min(4, rows));
    }
    p.rows_per_warp = R;
    const int64_t chunks = (rows + R - 1) / R;
    const int64_t warps = chunks * p.nstrips;
    p.blocks = (int)((warps + wpb - 1) / wpb);
    return p;
}

void launch_step(const swe_domain* d, const Plan& pl, const StepLaunch& sl, bool run,
                 cudaStream_t st) {
    dispatch(pl.V, d->arith, run, d->masked, [&](auto k) { decltype(k)::launch(pl.blocks, sl, st); });
}

// 2-D grid of a per-cell kernel over rows x cols (for_cells): x over the
// columns, y over the rows, about 8 CTAs per SM (and about `per_thread` cells
// per thread on small planes).
dim3 cell_grid(int rows, int cols, int threads, int sms, int per_thread = 1) {
    const int64_t gx = std::max<int64_t>(1, std::min<int64_t>((cols + threads - 1) / threads, (int64_t)sms * 8));
    const int64_t want = std::max<int64_t>(1, ((int64_t)rows * cols + (int64_t)threads * per_thread - 1) /
                                                  ((int64_t)threads * per_thread) / gx);
    const int64_t gy = std::max<int64_t>(1, std::min<int64_t>({(int64_t)rows, want, ((int64_t)sms * 8 + gx - 1) / gx}));
    return dim3((unsigned)gx, (unsigned)gy);
}

dim3 reduce_grid(const swe_domain* d) {
    return cell_grid(d->dd.upd_hi - d->dd.upd_lo, d->dd.cols, kThreads, d->sms, 8);
}

int reduce_blocks(const swe_domain* d) {
    const dim3 g = reduce_grid(d);
    return (int)(g.x * g.y);
}

void launch_reduce(const swe_domain* d, const StateView& s, Control* ctl, cudaStream_t st) {
    const dim3 grid = reduce_grid(d);
    if (d->arith == SWE_ARITH_FAST)
        reduce_kernel<FastMath, kThreads><<<grid, kThreads, 0, st>>>(d->dd, s, ctl, d->rparts);
    else
        reduce_kernel<ExactMath, kThreads><<<grid, kThreads, 0, st>>>(d->dd, s, ctl, d->rparts);
}

int choose_vec(const void* const* ptrs, int n, int64_t pitch_a, int64_t pitch_b) {
    auto aligned = [&](int bytes) {
        for (int i = 0; i < n; ++i)
            if (reinterpret_cast<uintptr_t>(ptrs[i]) % bytes) return false;
        return true;
    };
    if (pitch_a % 2 == 0 && pitch_b % 2 == 0 && aligned(8)) return 2;
    return 1;
}

// Partials of the reductions (reduce_kernel); separate from the step slots so that
// a CFL query in the middle of a resident run leaves its ledger intact.
int ensure_rparts(swe_domain* d) {
    const int blocks = reduce_blocks(d);
    if (blocks <= d->rparts_cap) return SWE_OK;
    if (d->rparts) cudaFree(d->rparts);
    d->rparts = nullptr;
    SWE_CK(cudaMalloc(&d->rparts, sizeof(Partial) * (size_t)blocks));
    d->rparts_cap = blocks;
    return SWE_OK;
}

// Ledger slots of the run-mode steps for `blocks` CTAs (one per warp), and the
// reduction partials.
int ensure_parts(swe_domain* d, int blocks) {
    const int rrc = ensure_rparts(d);
    if (rrc) return rrc;
    if (blocks <= d->slots_cap) return SWE_OK;
    if (d->slots) cudaFree(d->slots);
    d->slots = nullptr;
    SWE_CK(cudaMalloc(&d->slots, sizeof(LedgerSlot) * kWarpsPerCta * (size_t)blocks));
    d->slots_cap = blocks;
    return SWE_OK;
}

// The bed and n^2 of the strip-boundary columns (when the domain keeps them;
// after creation and after every change of n^2).
int fill_edge_statics(swe_domain* d, cudaStream_t st) {
    if (!d->edge_stat) return SWE_OK;
    const int nb = (d->dd.cols + kEdgeStrip - 1) / kEdgeStrip + 1;
    edge_fill_kernel<<<dim3((unsigned)((d->dd.rows + 127) / 128), (unsigned)nb), 128, 0, st>>>(
        d->dd, StateView{nullptr, nullptr, nullptr, 0}, nullptr, d->edge_stat);
    SWE_CK(cudaGetLastError());
    return SWE_OK;
}

// The strip-boundary columns of the state in ping buffer 0 (a run's start).
int fill_edges(swe_domain* d, cudaStream_t st) {
    if (!d->edge_buf[0]) return SWE_OK;
    const int nb = (d->dd.cols + kEdgeStrip - 1) / kEdgeStrip + 1;
    edge_fill_kernel<<<dim3((unsigned)((d->dd.rows + 127) / 128), (unsigned)nb), 128, 0, st>>>(
        d->dd, StateView{d->ping[0][0], d->ping[0][1], d->ping[0][2], d->ppitch}, d->edge_buf[0], nullptr);
    SWE_CK(cudaGetLastError());
    return SWE_OK;
}

int ensure_ping(swe_domain* d) {
    if (d->ping[0][0]) return SWE_OK;
    d->ppitch = round_up(d->dd.cols, 128);
    const size_t plane = sizeof(float) * (size_t)d->ppitch * (size_t)d->dd.rows;
    for (int b = 0; b < 2; ++b)
        for (int f = 0; f < 3; ++f) {
            SWE_CK(cudaMalloc(&d->ping[b][f], plane));
            SWE_CK(cudaMemset(d->ping[b][f], 0, plane));
        }
    // The strip-boundary columns that the plain run-mode step keeps for the
    // next step (DomainDev::edge), allocated with the state buffers, before any
    // step graph is captured.  Not for row strips of a decomposed domain, whose
    // halo rows are exchanged outside the step.
    if (d->strip_total_rows < 0) {
        DomainDev& dd = d->dd;
        const int nb = (dd.cols + kEdgeStrip - 1) / kEdgeStrip + 1;
        dd.edge_rows = round_up(dd.rows, 32);
        const size_t n6 = sizeof(float) * (size_t)nb * 6 * (size_t)dd.edge_rows;
        const size_t n4 = sizeof(float) * (size_t)nb * 4 * (size_t)dd.edge_rows;
        for (int b = 0; b < 2; ++b) {
            SWE_CK(cudaMalloc(&d->edge_buf[b], n6));
            SWE_CK(cudaMemset(d->edge_buf[b], 0, n6));
        }
        SWE_CK(cudaMalloc(&d->edge_stat, n4));
        SWE_CK(cudaMemset(d->edge_stat, 0, n4));
        dd.edge[0] = d->edge_buf[0];
        dd.edge[1] = d->edge_buf[1];
        dd.edge_static = d->edge_stat;
        const int rc = fill_edge_statics(d, nullptr);
        if (rc) return rc;
        SWE_CK(cudaDeviceSynchronize());
    }
    return SWE_OK;
}

int check_state_ptrs(const void* a, const void* b, const void* c, int64_t pitch, int cols) {
    if (!a || !b || !c) return fail(SWE_ERR_INVALID, "state pointers must be non-null");
    if (pitch < cols) return fail(SWE_ERR_INVALID, "pitch must be >= cols");
    return SWE_OK;
}

int copy_plane(float* dst, int64_t dpitch, const float* src, int64_t spitch, int rows, int cols,
               cudaStream_t st) {
    SWE_CK(cudaMemcpy2DAsync(dst, sizeof(float) * dpitch, src, sizeof(float) * spitch,
                             sizeof(float) * cols, rows, cudaMemcpyDeviceToDevice, st));
    return SWE_OK;
}

// Load the initial state into ping buffer 0, upload the output times, write
// snapshot 0, reset the run control and launch the reduction that sets the
// clock, the first CFL dt and volume0.  Shared by swe_run, swe_advance and the
// ensemble.
int begin_run(swe_domain* d, StateView init, const float* times_host, int n_times, double t_start,
              int n_out, int max_steps, float* out_h, float* out_hu, float* out_hv, cudaStream_t st,
              const double* times64_host = nullptr, double* dt_log = nullptr, int defer_plan = 0) {
    const int rows = d->dd.rows, cols = d->dd.cols;
    d->resident = false;  // any run replaces a resident state
    int rc = ensure_ping(d);
    if (rc) return rc;
    rc = ensure_parts(d, reduce_blocks(d));
    if (rc) return rc;
    for (int f = 0; f < 3; ++f) {
        const float* src = f == 0 ? init.h : (f == 1 ? init.hu : init.hv);
        rc = copy_plane(d->ping[0][f], d->ppitch, src, init.pitch, rows, cols, st);
        if (rc) return rc;
    }
    rc = fill_edges(d, st);
    if (rc) return rc;
    if (n_times > d->times_cap) {
        if (d->times_dev) cudaFree(d->times_dev);
        d->times_dev = nullptr;
        SWE_CK(cudaMalloc(&d->times_dev, sizeof(float) * (size_t)n_times));
        d->times_cap = n_times;
    }
    // Output times (up to kInlineTimes: every advance, ensemble interval and
    // ordinary run) travel with the control block's launch parameters; longer
    // output lists are copied.
    static_assert(kInlineTimes <= 128, "one thread of control_init_kernel per inline time");
    RunTargets tg{};
    if (n_times <= kInlineTimes) {
        tg.n = n_times;
        tg.times = d->times_dev;
        for (int i = 0; i < n_times; ++i) tg.t[i] = times_host[i];
    } else {
        SWE_CK(cudaMemcpyAsync(d->times_dev, times_host, sizeof(float) * (size_t)n_times,
                               cudaMemcpyHostToDevice, st));
    }
    if (times64_host) {
        if (n_times > 2) return fail(SWE_ERR_INVALID, "float64 targets support one interval");
        if (!d->times64_dev) SWE_CK(cudaMalloc(&d->times64_dev, 2 * sizeof(double)));
        tg.times64 = d->times64_dev;
        for (int i = 0; i < n_times; ++i) tg.t64[i] = times64_host[i];
    }
    if (out_h) {
        float* outs[3] = {out_h, out_hu, out_hv};
        for (int f = 0; f < 3; ++f) {
            const float* src = f == 0 ? init.h : (f == 1 ? init.hu : init.hv);
            rc = copy_plane(outs[f], cols, src, init.pitch, rows, cols, st);
            if (rc) return rc;
        }
    }
    Control c0;
    std::memset(&c0, 0, sizeof(c0));
    c0.n_out = n_out;
    c0.max_steps = max_steps;
    c0.t_start = t_start;
    c0.times = d->times_dev;
    c0.times64 = times64_host ? d->times64_dev : nullptr;
    c0.done_counter = d->done_counter;
    c0.dt_log = dt_log;
    c0.defer_plan = defer_plan;
    c0.out_h = out_h;
    c0.out_hu = out_hu;
    c0.out_hv = out_hv;
    c0.out_plane = (int64_t)rows * cols;
    ControlHeadImage img;
    std::memcpy(&img, &c0, sizeof(img));
    control_init_kernel<<<1, 128, 0, st>>>(d->ctl, img, tg);
    SWE_CK(cudaGetLastError());
    StateView v0{d->ping[0][0], d->ping[0][1], d->ping[0][2], d->ppitch};
    launch_reduce(d, v0, d->ctl, st);
    SWE_CK(cudaGetLastError());
    // The step warps' ledger slots start the run at zero.
    SWE_CK(cudaMemsetAsync(d->slots, 0, sizeof(LedgerSlot) * kWarpsPerCta * (size_t)d->slots_cap, st));
    return SWE_OK;
}

// The run's ledger into the control block from the slots of the step warps of
// `ncta` CTAs.
int fold_ledger(swe_domain* d, int ncta, cudaStream_t st) {
    ledger_fold_kernel<kThreads><<<1, kThreads, 0, st>>>(d->dd, d->ctl, d->slots, ncta * kWarpsPerCta);
    SWE_CK(cudaGetLastError());
    return SWE_OK;
}

// Steps per poll of the run driver and at most per captured step graph.
constexpr int kChunk = 32;

// Run-mode launch of step k of a run (buffer parity k & 1).
StepLaunch run_launch(const swe_domain* d, const Plan& pl, int64_t k) {
    StepLaunch sl{};
    sl.d = d->dd;
    sl.ctl = d->ctl;
    sl.slots = d->slots;
    sl.nstrips = pl.nstrips;
    sl.rows_per_warp = pl.rows_per_warp;
    const int src = (int)(k & 1);
    sl.par = src;
    sl.in = StateView{d->ping[src][0], d->ping[src][1], d->ping[src][2], d->ppitch};
    sl.out = StateOut{d->ping[src ^ 1][0], d->ping[src ^ 1][1], d->ping[src ^ 1][2], d->ppitch};
    return sl;
}

// The graph of `len` (1..kChunk) run-mode steps starting from ping buffer
// `par`, captured on a private stream (the caller's stream may be the legacy
// default stream, which cannot be captured) on first use.  Its kernel
// parameters hold the domain record by value, so a change of the partials
// buffer, the rain scale or the plan re-captures every graph.
void drop_chunk_graphs(swe_domain* d) {
    for (auto& row : d->chunk_graph)
        for (auto& g : row)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
}

int chunk_graph(swe_domain* d, const Plan& pl, int par, int len, cudaGraphExec_t* out) {
    if (d->chunk_graph_slots != d->slots || d->chunk_graph_rain_scale != d->dd.rain_scale ||
        d->chunk_graph_rows != pl.rows_per_warp) {
        drop_chunk_graphs(d);
        d->chunk_graph_slots = d->slots;
        d->chunk_graph_rain_scale = d->dd.rain_scale;
        d->chunk_graph_rows = pl.rows_per_warp;
    }
    cudaGraphExec_t& slot = d->chunk_graph[par][len];
    if (slot) {
        *out = slot;
        return SWE_OK;
    }
    if (!d->cap_stream) SWE_CK(cudaStreamCreateWithFlags(&d->cap_stream, cudaStreamNonBlocking));
    SWE_CK(cudaStreamBeginCapture(d->cap_stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < len; ++k) launch_step(d, pl, run_launch(d, pl, par + k), true, d->cap_stream);
    cudaGraph_t g = nullptr;
    SWE_CK(cudaStreamEndCapture(d->cap_stream, &g));
    const cudaError_t err = cudaGraphInstantiate(&slot, g, 0);
    cudaGraphDestroy(g);
    if (err != cudaSuccess) {
        slot = nullptr;
        return fail(SWE_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(err));
    }
    // Uploaded now, ahead of its first launch.
    SWE_CK(cudaGraphUpload(slot, d->cap_stream));
    *out = slot;
    return SWE_OK;
}

// Enqueue steps k0 .. k0+n-1 of the current run as graphs of up to kChunk
// steps.  Every graph the steps need is captured before the first one is
// launched, so that the stream never waits for the host in between; with
// launch == false the graphs are only captured.
int enqueue_run_steps(swe_domain* d, int64_t k0, int64_t n, cudaStream_t st, bool launch = true) {
    const Plan pl = make_plan(d, d->run_vec, true);
    const int64_t end = k0 + n;
    for (int64_t k = k0; k < end; k += kChunk) {
        cudaGraphExec_t g = nullptr;
        const int rc = chunk_graph(d, pl, (int)(k & 1), (int)std::min<int64_t>(kChunk, end - k), &g);
        if (rc) return rc;
    }
    if (!launch) return SWE_OK;
    for (int64_t k = k0; k < end; k += kChunk) {
        cudaGraphExec_t g = nullptr;
        const int rc = chunk_graph(d, pl, (int)(k & 1), (int)std::min<int64_t>(kChunk, end - k), &g);
        if (rc) return rc;
        SWE_CK(cudaGraphLaunch(g, st));
    }
    SWE_CK(cudaGetLastError());
    return SWE_OK;
}

// Shared run driver for swe_run and swe_advance.
int run_driver(swe_domain* d, StateView init, const float* times_host, int n_times,
               double t_start, int n_out, int max_steps, float* out_h, float* out_hu,
               float* out_hv, swe_run_result* res, cudaStream_t st, int* final_buf,
               const double* times64_host = nullptr, double* dt_log = nullptr) {
    int rc = ensure_ping(d);
    if (rc) return rc;
    const Plan pl = make_plan(d, d->run_vec, true);
    rc = ensure_parts(d, std::max(pl.blocks, reduce_blocks(d)));
    if (rc) return rc;
    rc = begin_run(d, init, times_host, n_times, t_start, n_out, max_steps, out_h, out_hu, out_hv, st,
                   times64_host, dt_log);
    if (rc) return rc;
    int64_t launched = 0;
    d->launches = 1;
    d->timed_valid = false;
    if (d->timing) SWE_CK(cudaEventRecord(d->time_ev[0], st));
    const int K = kChunk;
    int chunk = 0;
    bool finished = false;
    while (!finished) {
        const int64_t todo = std::min<int64_t>(K, (int64_t)max_steps - launched);
        rc = enqueue_run_steps(d, launched, todo, st);
        if (rc) return rc;
        launched += todo;
        d->launches += todo;
        const int slot = chunk & 1;
        SWE_CK(cudaMemcpyAsync(&d->ctl_host[slot], d->ctl, kControlHead, cudaMemcpyDeviceToHost, st));
        SWE_CK(cudaEventRecord(d->poll_ev[slot], st));
        if (launched >= max_steps) break;
        if (chunk > 0) {
            SWE_CK(cudaEventSynchronize(d->poll_ev[slot ^ 1]));
            if (d->ctl_host[slot ^ 1].done) finished = true;
        }
        ++chunk;
    }
    if (d->timing) {
        // The end event follows the last step kernel; poll copies in between are ~1 us each.
        SWE_CK(cudaEventRecord(d->time_ev[1], st));
        d->timed_steps = launched;
        d->timed_valid = true;
    }
    rc = fold_ledger(d, pl.blocks, st);
    if (rc) return rc;
    SWE_CK(cudaStreamSynchronize(st));
    SWE_CK(cudaMemcpy(&d->ctl_host[0], d->ctl, kControlHead, cudaMemcpyDeviceToHost));
    const Control& c = d->ctl_host[0];
    res->final_time_s = c.t;
    res->outputs_written = c.idx;
    res->steps_used = c.steps;
    res->status = c.status ? c.status : (c.idx >= n_out ? SWE_OK : SWE_ERR_MAX_STEPS);
    res->reserved = 0;
    for (int i = 0; i < 6; ++i) res->ledger[i] = c.ledger[i];
    if (final_buf) *final_buf = c.steps & 1;
    return SWE_OK;
}

void free_domain(swe_domain* d) {
    if (!d) return;
    cudaFree(d->bed);
    cudaFree(d->nm);
    cudaFree(d->mult);
    cudaFree(d->rain);
    cudaFree(d->ctl);
    cudaFree(d->ctl_scratch);
    if (d->ctl_host) cudaFreeHost(d->ctl_host);
    cudaFree(d->slots);
    cudaFree(d->rparts);
    for (int b = 0; b < 2; ++b)
        for (int f = 0; f < 3; ++f) cudaFree(d->ping[b][f]);
    cudaFree(d->edge_buf[0]);
    cudaFree(d->edge_buf[1]);
    cudaFree(d->edge_stat);
    cudaFree(d->times_dev);
    for (int q = 0; q < 3; ++q) cudaFree(d->lupd[q]);
    cudaFree(d->times64_dev);
    cudaFree(d->next_scratch);
    cudaFree(d->next_scratch2);
    cudaFree(d->seg2);
    for (cudaEvent_t e : d->seg_ev)
        if (e) cudaEventDestroy(e);
    if (d->aux_stream) cudaStreamDestroy(d->aux_stream);
    cudaFree(d->corr_sums);
    cudaFree(d->corr_prov);
    for (int i = 0; i < 2; ++i) {
        if (d->poll_ev[i]) cudaEventDestroy(d->poll_ev[i]);
        if (d->time_ev[i]) cudaEventDestroy(d->time_ev[i]);
    }
    drop_chunk_graphs(d);
    if (d->cap_stream) cudaStreamDestroy(d->cap_stream);
    cudaFree(d->snap_dev);
    if (d->copy_stream) cudaStreamDestroy(d->copy_stream);
    if (d->snap_ev) cudaEventDestroy(d->snap_ev);
    delete d;
}

__global__ void pack_static_kernel(const float* bed, const float* man, const uint8_t* mask,
                                   const float* mult, int rows, int cols, int64_t pitch,
                                   float* bed_o, float* nm_o, float* mult_o, int* any_inactive) {
    const int64_t n = (int64_t)rows * pitch;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(i / pitch), c = (int)(i - (int64_t)r * pitch);
        const int cc = c < cols ? c : cols - 1;
        const int64_t j = (int64_t)r * cols + cc;
        const float n_ = man[j];
        const float n2 = __fmul_rn(n_, n_);  // manning_n**2 in float32
        const float n2a = fabsf(n2);
        bed_o[i] = bed[j];
        // The domain mask rides in the sign bit: set = inactive.
        nm_o[i] = mask[j] ? n2a : __int_as_float(__float_as_int(n2a) | (int)0x80000000);
        if (!mask[j]) *any_inactive = 1;
        if (mult_o) mult_o[i] = mult[j];
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Batched ensemble (swe_ensemble_*)
// ---------------------------------------------------------------------------
struct swe_ensemble {
    std::vector<swe_domain*> doms;
    int arith = SWE_ARITH_FAST;
    bool masked = false;
    int rows_per_warp = 128;  // provisional: swe_ensemble_create sets ens_auto_rows (B200Ensemble.autotune measures)
    int sms = 148;
    MemberDev* members_dev = nullptr;
    int members_cap = 0;
    int2* items_dev = nullptr;
    int items_cap = 0;
    int n_items = 0;
    int grid = 1;
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_k = 0;
    cudaEvent_t time_ev[2] = {nullptr, nullptr};
    bool timing = false;
    bool timed_valid = false;
    int64_t timed_steps = 0;
    int64_t launches = 0;
    unsigned* done_counter = nullptr;       // device: members finished in advance_to
    unsigned* done_host = nullptr;          // pinned: two polled copies of it
    cudaEvent_t poll_ev[2] = {nullptr, nullptr};
    // Member table in the kernel's parameter space (up to kEnsParamMembers
    // members; SWE_ENS_PARAM_TABLE=0 keeps the table in global memory).
    std::unique_ptr<EnsParams> params;
    std::vector<int> member_ncta;  // step CTAs (ledger slots) of each member
};

namespace {

template <class M, bool MASKED>
void ens_launch_t(const swe_ensemble* e, int parity, cudaStream_t st) {
    cudaLaunchConfig_t cfg = pdl_config(e->grid, st);
    cudaLaunchAttribute attr[1];
    attach_pdl(cfg, attr);
    if (e->params) {
        e->params->parity = parity;
        cudaLaunchKernelEx(&cfg, ensemble_step_kernel_p<M, kThreads, MASKED>, *e->params);
    } else {
        cudaLaunchKernelEx(&cfg, ensemble_step_kernel<M, kThreads, MASKED>, (const MemberDev*)e->members_dev,
                           (const int2*)e->items_dev, e->n_items, parity);
    }
}

void ens_launch(const swe_ensemble* e, int parity, cudaStream_t st) {
    if (e->arith == SWE_ARITH_FAST) {
        if (e->masked) ens_launch_t<FastMath, true>(e, parity, st); else ens_launch_t<FastMath, false>(e, parity, st);
    } else {
        if (e->masked) ens_launch_t<ExactMath, true>(e, parity, st); else ens_launch_t<ExactMath, false>(e, parity, st);
    }
}

int ens_occupancy(const swe_ensemble* e) {
    const void* fn = nullptr;
    if (e->params) {
        if (e->arith == SWE_ARITH_FAST)
            fn = e->masked ? reinterpret_cast<const void*>(&ensemble_step_kernel_p<FastMath, kThreads, true>)
                           : reinterpret_cast<const void*>(&ensemble_step_kernel_p<FastMath, kThreads, false>);
        else
            fn = e->masked ? reinterpret_cast<const void*>(&ensemble_step_kernel_p<ExactMath, kThreads, true>)
                           : reinterpret_cast<const void*>(&ensemble_step_kernel_p<ExactMath, kThreads, false>);
    } else if (e->arith == SWE_ARITH_FAST)
        fn = e->masked ? reinterpret_cast<const void*>(&ensemble_step_kernel<FastMath, kThreads, true>)
                       : reinterpret_cast<const void*>(&ensemble_step_kernel<FastMath, kThreads, false>);
    else
        fn = e->masked ? reinterpret_cast<const void*>(&ensemble_step_kernel<ExactMath, kThreads, true>)
                       : reinterpret_cast<const void*>(&ensemble_step_kernel<ExactMath, kThreads, false>);
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kThreads, 0) != cudaSuccess || n < 1) n = 1;
    return n;
}

// Default rows per warp: the step of a batch that fits the persistent grid in
// one round takes about as long as its longest march, so the default is the
// smallest march (at least 32 rows) whose work items all fit in one round of
// the grid; when even 1024-row marches need more than one round, 256.
int ens_occupancy(const swe_ensemble* e);
int ens_auto_rows(const swe_ensemble* e) {
    const int wpb = kThreads / kWarp;
    const int64_t slots = (int64_t)ens_occupancy(e) * e->sms;
    auto items = [&](int R) {
        int64_t n = 0;
        for (const swe_domain* d : e->doms) {
            const int64_t nstrips = (d->dd.cols + 2 * kWarp - 1) / (2 * kWarp);
            const int64_t chunks = (d->dd.rows + R - 1) / R;
            n += (chunks * nstrips + wpb - 1) / wpb;
        }
        return n;
    };
    if (items(1024) > slots) return 256;
    int lo = 32, hi = 1024;  // items(hi) <= slots; items is non-increasing in R
    if (items(lo) <= slots) return lo;
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (items(mid) <= slots) hi = mid; else lo = mid;
    }
    return hi;
}

// Member table and work list for the current rows-per-warp.
int ens_rebuild(swe_ensemble* e) {
    const int wpb = kThreads / kWarp;
    const int R = e->rows_per_warp;
    std::vector<MemberDev> md(e->doms.size());
    std::vector<int2> items;
    for (size_t m = 0; m < e->doms.size(); ++m) {
        swe_domain* d = e->doms[m];
        int rc = ensure_ping(d);
        if (rc) return rc;
        const int nstrips = (d->dd.cols + 2 * kWarp - 1) / (2 * kWarp);
        const int chunks = (d->dd.rows + R - 1) / R;
        const int ncta = (int)(((int64_t)chunks * nstrips + wpb - 1) / wpb);
        rc = ensure_parts(d, std::max(ncta, reduce_blocks(d)));
        if (rc) return rc;
        MemberDev& x = md[m];
        x.d = d->dd;
        for (int b = 0; b < 2; ++b)
            for (int f = 0; f < 3; ++f) x.buf[b][f] = d->ping[b][f];
        x.pitch = d->ppitch;
        x.ctl = d->ctl;
        x.slots = d->slots;
        x.nstrips = nstrips;
        x.rows_per_warp = R;
        x.ncta = ncta;
        for (int c = 0; c < ncta; ++c) items.push_back(make_int2((int)m, c));
        e->member_ncta.resize(e->doms.size());
        e->member_ncta[m] = ncta;
    }
    if ((int)md.size() > e->members_cap) {
        cudaFree(e->members_dev);
        e->members_dev = nullptr;
        SWE_CK(cudaMalloc(&e->members_dev, sizeof(MemberDev) * md.size()));
        e->members_cap = (int)md.size();
    }
    if ((int)items.size() > e->items_cap) {
        cudaFree(e->items_dev);
        e->items_dev = nullptr;
        SWE_CK(cudaMalloc(&e->items_dev, sizeof(int2) * items.size()));
        e->items_cap = (int)items.size();
    }
    SWE_CK(cudaMemcpy(e->members_dev, md.data(), sizeof(MemberDev) * md.size(), cudaMemcpyHostToDevice));
    SWE_CK(cudaMemcpy(e->items_dev, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice));
    e->n_items = (int)items.size();
    const char* pt = std::getenv("SWE_ENS_PARAM_TABLE");
    e->params.reset();
    if ((int)md.size() <= kEnsParamMembers && !(pt && pt[0] == '0')) {
        e->params.reset(new EnsParams());
        std::memset(e->params.get(), 0, sizeof(EnsParams));
        int b = 0;
        for (size_t m = 0; m < md.size(); ++m) {
            e->params->m[m] = md[m];
            e->params->cta_begin[m] = b;
            b += md[m].ncta;
        }
        e->params->cta_begin[md.size()] = b;
        e->params->n_members = (int)md.size();
        e->params->n_items = b;
    }
    e->grid = std::max(1, std::min(e->n_items, ens_occupancy(e) * e->sms));
    if (e->graph) {
        cudaGraphExecDestroy(e->graph);
        e->graph = nullptr;
        e->graph_k = 0;
    }
    return SWE_OK;
}

// CUDA graph of K consecutive ensemble steps (parity alternating, K even).
int ens_graph(swe_ensemble* e, int K) {
    if (e->graph && e->graph_k == K) return SWE_OK;
    if (e->graph) {
        cudaGraphExecDestroy(e->graph);
        e->graph = nullptr;
    }
    if (!e->cap_stream) SWE_CK(cudaStreamCreateWithFlags(&e->cap_stream, cudaStreamNonBlocking));
    SWE_CK(cudaStreamBeginCapture(e->cap_stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < K; ++k) ens_launch(e, k & 1, e->cap_stream);
    cudaGraph_t g = nullptr;
    SWE_CK(cudaStreamEndCapture(e->cap_stream, &g));
    const cudaError_t err = cudaGraphInstantiate(&e->graph, g, 0);
    cudaGraphDestroy(g);
    if (err != cudaSuccess) return fail(SWE_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(err));
    e->graph_k = K;
    return SWE_OK;
}

// Reads every member's Control block, fills its run result and copies its
// final planes to the caller's buffers.  Error statuses: any member's, the
// first one met; a member short of its target counts only when need_target.
int ens_collect(swe_ensemble* e, float* const* h, float* const* hu, float* const* hv, const int64_t* pitch,
                swe_run_result* results, cudaStream_t st, bool need_target) {
    const int n = (int)e->doms.size();
    // Every member's ledger fold and control-block read are queued first and
    // waited for once; the final states are then copied out in stream order.
    for (int m = 0; m < n; ++m) {
        swe_domain* d = e->doms[m];
        const int rc = fold_ledger(d, e->member_ncta[m], st);
        if (rc) return rc;
        SWE_CK(cudaMemcpyAsync(&d->ctl_host[0], d->ctl, kControlHead, cudaMemcpyDeviceToHost, st));
    }
    SWE_CK(cudaStreamSynchronize(st));
    int status = SWE_OK;
    for (int m = 0; m < n; ++m) {
        swe_domain* d = e->doms[m];
        const Control& c = d->ctl_host[0];
        swe_run_result& r = results[m];
        r.final_time_s = c.t;
        r.outputs_written = c.idx;
        r.steps_used = c.steps;
        r.status = c.status;
        r.reserved = 0;
        for (int i = 0; i < 6; ++i) r.ledger[i] = c.ledger[i];
        if (c.status && !status) status = c.status;
        if (need_target && !c.done && !status) status = SWE_ERR_MAX_STEPS;
        float* outs[3] = {h[m], hu[m], hv[m]};
        const int fb = c.steps & 1;
        for (int f = 0; f < 3; ++f) {
            const int rc = copy_plane(outs[f], pitch[m], d->ping[fb][f], d->ppitch, d->dd.rows, d->dd.cols, st);
            if (rc) return rc;
        }
    }
    if (status == SWE_ERR_NONFINITE) return fail(SWE_ERR_NONFINITE, "non-finite values reached a member's CFL reduction");
    if (status == SWE_ERR_MAX_STEPS) return fail(status, "an ensemble member did not reach its target time");
    if (status) return fail(status, "an ensemble member stopped with an error status");
    return SWE_OK;
}


void free_ensemble(swe_ensemble* e) {
    if (!e) return;
    for (auto* d : e->doms) free_domain(d);
    cudaFree(e->members_dev);
    cudaFree(e->items_dev);
    if (e->graph) cudaGraphExecDestroy(e->graph);
    if (e->cap_stream) cudaStreamDestroy(e->cap_stream);
    for (int i = 0; i < 2; ++i) {
        if (e->time_ev[i]) cudaEventDestroy(e->time_ev[i]);
        if (e->poll_ev[i]) cudaEventDestroy(e->poll_ev[i]);
    }
    cudaFree(e->done_counter);
    cudaFreeHost(e->done_host);
    delete e;
}

}  // namespace

// ---------------------------------------------------------------------------
// Allocation-free CFL reduction (swe_max_inverse_dt_noalloc)
// ---------------------------------------------------------------------------
// Some callers cannot call cudaMalloc at the point where they need a CFL time
// step: code that runs under a framework's caching allocator (PyTorch's holds
// the device memory it has reserved, so a direct cudaMalloc can fail although
// the pool has room), and time-stepping loops that forbid allocation once they
// are running.  For them this variant of the CFL reduction takes every input
// and the output from the caller and keeps its scratch -- one partial maximum
// per CTA and the last-CTA ticket -- in a fixed file-scope device array, so it
// allocates nothing.  The array is loaded with the library on every GPU that
// uses it and stays until the process exits.
namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocCellsPerBlock = 2048;  // 8 cells per thread
constexpr int kNoAllocMaxBlocks = SWE_NOALLOC_MAX_CELLS / kNoAllocCellsPerBlock;
constexpr int kNoAllocMaxDevices = 64;
static_assert(SWE_NOALLOC_MAX_CELLS % kNoAllocCellsPerBlock == 0, "limit must be whole CTAs");

struct NoAllocScratch {
    float block_max[kNoAllocMaxBlocks];  // 32 KiB of per-CTA partial maxima
    unsigned ticket;                     // last-CTA counter, zero between calls
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

__global__ void __launch_bounds__(kNoAllocThreads)
max_inverse_dt_noalloc_kernel(const float* __restrict__ h, const float* __restrict__ hu,
                              const float* __restrict__ hv, int64_t pitch,
                              const uint8_t* __restrict__ mask, int rows, int cols, Consts k,
                              NoAllocScratch* scratch, float* out) {
    __shared__ float s_max[kNoAllocThreads / kWarp];
    __shared__ bool s_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t n = (int64_t)rows * cols;
    const int64_t base = (int64_t)blockIdx.x * kNoAllocCellsPerBlock;
    float m = 0.f;
    for (int q = threadIdx.x; q < kNoAllocCellsPerBlock; q += kNoAllocThreads) {
        const int64_t i = base + q;
        if (i >= n) break;
        const int r = (int)(i / cols), c = (int)(i - (int64_t)r * cols);
        const int64_t o = (int64_t)r * pitch + c;
        float u, v;
        const float hh = h[o];
        ExactMath::vel2(hu[o], hv[o], hh, k.dry, u, v);
        const float w = ExactMath::sqrt(ExactMath::mul(k.g, fmaxf(hh, 0.0f)));
        const float inv = ExactMath::add(ExactMath::div(ExactMath::add(fabsf(u), w), k.dx),
                                         ExactMath::div(ExactMath::add(fabsf(v), w), k.dy));
        m = nan_max(m, mask[i] ? inv : 0.0f);
    }
    m = warp_max(m);
    if (lane == 0) s_max[warp] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        float b = s_max[0];
        for (int w = 1; w < kNoAllocThreads / kWarp; ++w) b = nan_max(b, s_max[w]);
        scratch->block_max[blockIdx.x] = b;
        __threadfence();
        s_last = atomicAdd(&scratch->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const volatile float* bm = scratch->block_max;
    float a = 0.f;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += kNoAllocThreads) a = nan_max(a, bm[b]);
    a = warp_max(a);
    __syncthreads();
    if (lane == 0) s_max[warp] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        float r = s_max[0];
        for (int w = 1; w < kNoAllocThreads / kWarp; ++w) r = nan_max(r, s_max[w]);
        *out = r;
        scratch->ticket = 0u;  // leave the counter at zero for the next call
    }
}

// Device address of g_noalloc_scratch, looked up once per device.
int noalloc_scratch(NoAllocScratch** out) {
    static std::mutex mu;
    static NoAllocScratch* addr[kNoAllocMaxDevices] = {};
    int dev = 0;
    SWE_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(SWE_ERR_INVALID, "device index out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        SWE_CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        addr[dev] = static_cast<NoAllocScratch*>(p);
    }
    *out = addr[dev];
    return SWE_OK;
}

}  // namespace

namespace {
// Depth at flat cell indices (rows*cols numbering) of a pitched plane.
// Clock at the start of step k of a fixed-dt (dts == null) or logged-dt rollout:
// t_{k+1} = t_k + dt_k in float64, the accumulation the run-mode clock uses.
double step_time(int k, double dt, double t0, const double* dts) {
    double t = t0;
    for (int j = 0; j < k; ++j) t += dts ? dts[j] : dt;
    return t;
}

__global__ void gauge_gather_kernel(const float* h, int64_t pitch, int cols, const int64_t* idx, int n,
                                    float* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int64_t k = idx[i];
        out[i] = h[(k / cols) * pitch + (k % cols)];
    }
}

// lam_h[idx[i]] += g[i] (atomic: gauges may repeat).
__global__ void gauge_inject_kernel(float* lam_h, int64_t pitch, int cols, const int64_t* idx, int n,
                                    const float* g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int64_t k = idx[i];
        atomicAdd(&lam_h[(k / cols) * pitch + (k % cols)], g[i]);
    }
}

// Replace n^2 in the packed plane, keeping the mask in the sign bit.
__global__ void repack_manning_kernel(const float* n, int rows, int cols, int64_t pitch, float* nm) {
    const int64_t total = (int64_t)rows * pitch;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(i / pitch), c = (int)(i - (int64_t)r * pitch);
        const int cc = c < cols ? c : cols - 1;
        const float v = n[(int64_t)r * cols + cc];
        const float n2 = fabsf(__fmul_rn(v, v));
        const bool inactive = signbit(nm[i]);
        nm[i] = inactive ? __int_as_float(__float_as_int(n2) | (int)0x80000000) : n2;
    }
}
}  // namespace

extern "C" {

const char* swe_version(void) { return "swe_b200 0.1.0 sm_100a"; }

int swe_last_error(char* buf, size_t n) {
    if (buf && n) {
        const size_t k = std::min(n - 1, g_err.size());
        std::memcpy(buf, g_err.data(), k);
        buf[k] = '\0';
    }
    return (int)g_err.size();
}

int swe_domain_create(const swe_domain_desc* desc, swe_domain_t* out) {
    if (!desc || !out) return fail(SWE_ERR_INVALID, "null descriptor or output handle");
    *out = nullptr;
    const swe_domain_desc& q = *desc;
    if (q.rows < 1 || q.cols < 1) return fail(SWE_ERR_INVALID, "rows and cols must be >= 1");
    if (!(q.dx > 0) || !(q.dy > 0)) return fail(SWE_ERR_INVALID, "dx and dy must be positive");
    if (!(q.max_dt > 0)) return fail(SWE_ERR_INVALID, "max_dt must be positive");
    if (!(q.dry_tolerance >= 0)) return fail(SWE_ERR_INVALID, "dry_tolerance must be >= 0");
    if (q.n_rain < 1 || !q.rain_times || !q.rain_rates)
        return fail(SWE_ERR_INVALID, "the hyetograph needs at least one (time, rate) pair");
    for (int i = 0; i < 4; ++i)
        if (q.boundary[i] != SWE_REFLECTIVE && q.boundary[i] != SWE_OPEN)
            return fail(SWE_ERR_INVALID, "boundary codes must be 0 (reflective) or 1 (open)");
    if (!q.bed || !q.manning_n || !q.domain_mask)
        return fail(SWE_ERR_INVALID, "bed, manning_n and domain_mask are required");
    if (q.arithmetic != SWE_ARITH_EXACT && q.arithmetic != SWE_ARITH_FAST)
        return fail(SWE_ERR_INVALID, "arithmetic must be SWE_ARITH_EXACT or SWE_ARITH_FAST");
    int dev = 0;
    SWE_CK(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    SWE_CK(cudaGetDeviceProperties(&prop, dev));
    if (prop.major != 10)
        return fail(SWE_ERR_NO_DEVICE, std::string("this build targets sm_100a; device is ") + prop.name);

    swe_domain* d = new swe_domain();
    d->device = dev;
    d->sms = prop.multiProcessorCount;
    d->arith = q.arithmetic;
    // Runs use the paired-lane kernel in both arithmetics (exact arithmetic keeps
    // its operations scalar, but the paired march still measured 5.7 % faster on
    // the 2048^2 urban step than one cell per lane; the results are the same).
    d->run_vec = 2;
    if (const char* e = std::getenv("SWE_ROWS_PER_WARP")) d->rows_per_warp_override = std::atoi(e);
    if (const char* e = std::getenv("SWE_RUN_VEC")) {
        const int v = std::atoi(e);
        if (v == 1 || v == 2) d->run_vec = v;
    }
    const int rows = q.rows, cols = q.cols;
    const int64_t pitch = round_up(cols, 128);
    // The step kernels address a plane with 32-bit element offsets.
    if ((int64_t)(rows + 2) * pitch >= (int64_t(1) << 31))
        return fail(SWE_ERR_INVALID, "domain too large: a plane must hold fewer than 2^31 elements");
    const size_t plane = sizeof(float) * (size_t)pitch * rows;
    const size_t n = (size_t)rows * cols;
    auto bail = [&](int code) { free_domain(d); return code; };
    cudaError_t e;
#define SWE_CK2(expr)                                                                          \
    do {                                                                                       \
        e = (expr);                                                                            \
        if (e != cudaSuccess)                                                                  \
            return bail(fail(SWE_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e))); \
    } while (0)
    SWE_CK2(cudaMalloc(&d->bed, plane));
    SWE_CK2(cudaMalloc(&d->nm, plane));
    if (q.rainfall_multiplier) SWE_CK2(cudaMalloc(&d->mult, plane));
    // Stage the inputs on the device, then pack.
    const float *bed_s = q.bed, *man_s = q.manning_n, *mult_s = q.rainfall_multiplier;
    const uint8_t* mask_s = q.domain_mask;
    void* staging = nullptr;
    if (q.fields_on_host) {
        const size_t bytes = n * (3 * sizeof(float) + 1) + 256;
        SWE_CK2(cudaMalloc(&staging, bytes));
        char* p = static_cast<char*>(staging);
        SWE_CK2(cudaMemcpy(p, q.bed, n * sizeof(float), cudaMemcpyHostToDevice));
        bed_s = reinterpret_cast<const float*>(p);
        p += n * sizeof(float);
        SWE_CK2(cudaMemcpy(p, q.manning_n, n * sizeof(float), cudaMemcpyHostToDevice));
        man_s = reinterpret_cast<const float*>(p);
        p += n * sizeof(float);
        if (q.rainfall_multiplier) {
            SWE_CK2(cudaMemcpy(p, q.rainfall_multiplier, n * sizeof(float), cudaMemcpyHostToDevice));
            mult_s = reinterpret_cast<const float*>(p);
        }
        p += n * sizeof(float);
        SWE_CK2(cudaMemcpy(p, q.domain_mask, n, cudaMemcpyHostToDevice));
        mask_s = reinterpret_cast<const uint8_t*>(p);
    }
    int* flag = nullptr;
    SWE_CK2(cudaMalloc(&flag, sizeof(int)));
    SWE_CK2(cudaMemset(flag, 0, sizeof(int)));
    pack_static_kernel<<<std::min<int64_t>((rows * pitch + 255) / 256, 4096), 256>>>(
        bed_s, man_s, mask_s, mult_s, rows, cols, pitch, d->bed, d->nm, d->mult, flag);
    SWE_CK2(cudaGetLastError());
    int any_inactive = 1;
    SWE_CK2(cudaMemcpy(&any_inactive, flag, sizeof(int), cudaMemcpyDeviceToHost));
    cudaFree(flag);
    d->masked = any_inactive != 0;
    if (staging) cudaFree(staging);
    // Hyetograph as float64 (np.interp converts the float32 table to float64).
    d->rain_t.resize(q.n_rain);
    d->rain_r.resize(q.n_rain);
    for (int i = 0; i < q.n_rain; ++i) {
        d->rain_t[i] = (double)q.rain_times[i];
        d->rain_r[i] = (double)q.rain_rates[i];
    }
    SWE_CK2(cudaMalloc(&d->rain, sizeof(double) * 2 * q.n_rain));
    SWE_CK2(cudaMemcpy(d->rain, d->rain_t.data(), sizeof(double) * q.n_rain, cudaMemcpyHostToDevice));
    SWE_CK2(cudaMemcpy(d->rain + q.n_rain, d->rain_r.data(), sizeof(double) * q.n_rain,
                       cudaMemcpyHostToDevice));
    SWE_CK2(cudaMalloc(&d->ctl, sizeof(Control)));
    SWE_CK2(cudaMalloc(&d->ctl_scratch, sizeof(Control)));
    SWE_CK2(cudaMemset(d->ctl, 0, sizeof(Control)));
    SWE_CK2(cudaMemset(d->ctl_scratch, 0, sizeof(Control)));
    SWE_CK2(cudaMallocHost(&d->ctl_host, 2 * sizeof(Control)));
    for (int i = 0; i < 2; ++i) SWE_CK2(cudaEventCreateWithFlags(&d->poll_ev[i], cudaEventDisableTiming));
#undef SWE_CK2

    DomainDev& dd = d->dd;
    dd.rows = rows;
    dd.cols = cols;
    dd.spitch = pitch;
    dd.bed = d->bed;
    dd.nm = d->nm;
    dd.mult = d->mult;
    for (int i = 0; i < 4; ++i) dd.bnd[i] = q.boundary[i];
    dd.k.g = (float)q.gravity;
    dd.k.half_g = (float)(0.5 * q.gravity);
    dd.k.dry = (float)q.dry_tolerance;
    dd.k.dx = (float)q.dx;
    dd.k.dy = (float)q.dy;
    {
        // An exact power of two within float range: its reciprocal is exact too.
        auto pow2 = [](float v) {
            int e = 0;
            return v > 0.f && std::frexp(v, &e) == 0.5f && e > -120 && e < 120;
        };
        dd.k.pow2 = pow2(dd.k.dx) && pow2(dd.k.dy) ? 1 : 0;
    }
    dd.k.eps = (float)1.0e-12;
    dd.k.expo = (float)(7.0 / 3.0);
    dd.dx = q.dx;
    dd.dy = q.dy;
    dd.g = q.gravity;
    dd.cfl = q.cfl;
    dd.max_dt = q.max_dt;
    dd.default_rain = q.default_rainfall;
    dd.rain_t = d->rain;
    dd.rain_r = d->rain + q.n_rain;
    dd.n_rain = q.n_rain;
    dd.rain_x0 = d->rain_t.front();
    dd.rain_xn = d->rain_t.back();
    dd.rain_yn = d->rain_r.back();
    dd.rain_scale = 1.0;
    dd.upd_lo = 0;
    dd.upd_hi = q.rows;
    *out = d;
    return SWE_OK;
}

int swe_domain_destroy(swe_domain_t d) {
    if (!d) return SWE_OK;
    cudaDeviceSynchronize();
    free_domain(d);
    return SWE_OK;
}

int swe_rainfall_rate(swe_domain_t d, double time_s, double* rate_out) {
    if (!d || !rate_out) return fail(SWE_ERR_INVALID, "null argument");
    *rate_out = d->dd.rain_scale * host_rain_rate(d->rain_t, d->rain_r, d->dd.default_rain, time_s);
    return SWE_OK;
}

int swe_domain_set_rain_scale(swe_domain_t d, double scale) {
    if (!d) return fail(SWE_ERR_INVALID, "null domain");
    if (!(scale >= 0.0) || !std::isfinite(scale)) return fail(SWE_ERR_INVALID, "rain scale must be finite and >= 0");
    d->dd.rain_scale = scale;
    return SWE_OK;
}

int swe_domain_set_manning(swe_domain_t d, const float* manning_n, int32_t on_host, void* stream) {
    if (!d || !manning_n) return fail(SWE_ERR_INVALID, "null argument");
    const int rows = d->dd.rows, cols = d->dd.cols;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const float* src = manning_n;
    float* staged = nullptr;
    if (on_host) {
        SWE_CK(cudaMalloc(&staged, sizeof(float) * (size_t)rows * cols));
        SWE_CK(cudaMemcpyAsync(staged, manning_n, sizeof(float) * (size_t)rows * cols, cudaMemcpyHostToDevice, st));
        src = staged;
    }
    const int64_t n = (int64_t)rows * d->dd.spitch;
    repack_manning_kernel<<<(int)std::min<int64_t>((n + 255) / 256, 4096), 256, 0, st>>>(src, rows, cols, d->dd.spitch, d->nm);
    SWE_CK(cudaGetLastError());
    const int erc = fill_edge_statics(d, st);
    if (erc) return erc;
    if (staged) {
        SWE_CK(cudaStreamSynchronize(st));
        cudaFree(staged);
    }
    return SWE_OK;
}

namespace {

// One reverse step; `next` (U_{k+1}, or null) lets the cell part skip the face recompute.
int adjoint_step_impl(swe_domain* d, const float* h, const float* hu, const float* hv, int64_t pitch,
                      const float* next, int64_t next_pitch, int64_t next_plane,
                      const float* lam_h, const float* lam_hu, const float* lam_hv, int64_t lam_pitch,
                      float* lam_h_out, float* lam_hu_out, float* lam_hv_out, int64_t out_pitch,
                      float* grad_n2, double* grad_rain_scale, double dt, double time_s, cudaStream_t st) {
    const int rows = d->dd.rows;
    if (!d->lupd[0]) {
        d->lpitch = round_up(d->dd.cols, 128);
        for (int q = 0; q < 3; ++q) SWE_CK(cudaMalloc(&d->lupd[q], sizeof(float) * (size_t)d->lpitch * rows));
    }
    const double rate = host_rain_rate(d->rain_t, d->rain_r, d->dd.default_rain, time_s);
    AdjLaunch al{};
    al.d = d->dd;
    al.in = StateView{h, hu, hv, pitch};
    al.next = next ? StateView{next, next + next_plane, next + 2 * next_plane, next_pitch}
                   : StateView{nullptr, nullptr, nullptr, 0};
    al.lam = StateView{lam_h, lam_hu, lam_hv, lam_pitch};
    al.lam_out = StateOut{lam_h_out, lam_hu_out, lam_hv_out, out_pitch};
    for (int q = 0; q < 3; ++q) al.lupd[q] = d->lupd[q];
    al.lpitch = d->lpitch;
    al.grad_n2 = grad_n2;
    al.grad_rain = grad_rain_scale;
    al.s.dt = (float)dt;
    const volatile double dr = dt * (d->dd.rain_scale * rate);
    const volatile double dg = dt * d->dd.g;
    const volatile double dru = dt * rate;
    al.s.dt_rain = (float)dr;
    al.s.dt_g = (float)dg;
    al.dt_rate = (float)dru;
    al.k = AdjConsts{d->dd.k.g, d->dd.k.half_g, d->dd.k.dry, d->dd.k.eps, d->dd.k.dx, d->dd.k.dy};
    al.rdx = 1.0f / d->dd.k.dx;
    al.rdy = 1.0f / d->dd.k.dy;
    const int64_t n = (int64_t)rows * d->dd.cols;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((n + kThreads - 1) / kThreads, (int64_t)d->sms * 16));
    const bool aliased = lam_h_out == lam_h || lam_hu_out == lam_hu || lam_hv_out == lam_hv;
    if (!aliased) {
        // One fused kernel (its halo reads of lam need lam_out elsewhere).
        static std::once_flag attr_once[2];
        std::call_once(attr_once[next ? 1 : 0], [&] {
            if (next)
                cudaFuncSetAttribute(adj_tile_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sizeof(AdjTileSmem));
            else
                cudaFuncSetAttribute(adj_tile_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sizeof(AdjTileSmem));
        });
        const int64_t tiles = (int64_t)((d->dd.cols + kFTW - 1) / kFTW) * ((rows + kFTH - 1) / kFTH);
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)d->sms * 4));
        if (next)
            adj_tile_kernel<true><<<grid, kFThreads, sizeof(AdjTileSmem), st>>>(al);
        else
            adj_tile_kernel<false><<<grid, kFThreads, sizeof(AdjTileSmem), st>>>(al);
    } else {
        if (next)
            adj_cell_kernel<kThreads, true><<<blocks, kThreads, 0, st>>>(al);
        else
            adj_cell_kernel<kThreads, false><<<blocks, kThreads, 0, st>>>(al);
        const int64_t tiles = (int64_t)((d->dd.cols + kAdjTW - 1) / kAdjTW) * ((rows + kAdjTH - 1) / kAdjTH);
        adj_face_tile_kernel<<<(int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)d->sms * 8)),
                               kAdjTW * kAdjTH, 0, st>>>(al);
    }
    SWE_CK(cudaGetLastError());
    return SWE_OK;
}

}  // namespace

int swe_adjoint_step(swe_domain_t d, const float* h, const float* hu, const float* hv, int64_t pitch,
                     const float* lam_h, const float* lam_hu, const float* lam_hv, int64_t lam_pitch,
                     float* lam_h_out, float* lam_hu_out, float* lam_hv_out, int64_t out_pitch,
                     float* grad_n2, double* grad_rain_scale, double dt, double time_s, void* stream) {
    if (!d || !grad_n2 || !grad_rain_scale) return fail(SWE_ERR_INVALID, "null argument");
    int rc = check_state_ptrs(h, hu, hv, pitch, d->dd.cols);
    if (rc) return rc;
    rc = check_state_ptrs(lam_h, lam_hu, lam_hv, lam_pitch, d->dd.cols);
    if (rc) return rc;
    rc = check_state_ptrs(lam_h_out, lam_hu_out, lam_hv_out, out_pitch, d->dd.cols);
    if (rc) return rc;
    return adjoint_step_impl(d, h, hu, hv, pitch, nullptr, 0, 0, lam_h, lam_hu, lam_hv, lam_pitch, lam_h_out,
                             lam_hu_out, lam_hv_out, out_pitch, grad_n2, grad_rain_scale, dt, time_s,
                             static_cast<cudaStream_t>(stream));
}

int swe_step(swe_domain_t d, const float* h, const float* hu, const float* hv, int64_t pitch_in,
             float* h_out, float* hu_out, float* hv_out, int64_t pitch_out, double dt,
             double time_s, void* stream) {
    if (!d) return fail(SWE_ERR_INVALID, "null domain");
    int rc = check_state_ptrs(h, hu, hv, pitch_in, d->dd.cols);
    if (rc) return rc;
    rc = check_state_ptrs(h_out, hu_out, hv_out, pitch_out, d->dd.cols);
    if (rc) return rc;
    const void* ins[3] = {h, hu, hv};
    const void* outs[3] = {h_out, hu_out, hv_out};
    for (auto a : ins)
        for (auto b : outs)
            if (a == b) return fail(SWE_ERR_INVALID, "step outputs must not alias its inputs");
    if ((int64_t)d->dd.rows * std::max(pitch_in, pitch_out) >= (int64_t(1) << 31))
        return fail(SWE_ERR_INVALID, "state planes must hold fewer than 2^31 elements");
    const void* all[6] = {h, hu, hv, h_out, hu_out, hv_out};
    const int V = choose_vec(all, 6, pitch_in, pitch_out);
    const Plan pl = make_plan(d, V, false);
    const volatile double rate = d->dd.rain_scale * host_rain_rate(d->rain_t, d->rain_r, d->dd.default_rain, time_s);
    StepLaunch sl{};
    sl.d = d->dd;
    sl.in = StateView{h, hu, hv, pitch_in};
    sl.out = StateOut{h_out, hu_out, hv_out, pitch_out};
    sl.s.dt = (float)dt;
    const volatile double dr = dt * rate;
    const volatile double dg = dt * d->dd.g;
    sl.s.dt_rain = (float)dr;
    sl.s.dt_g = (float)dg;
    sl.ctl = nullptr;
    sl.slots = nullptr;
    sl.nstrips = pl.nstrips;
    sl.rows_per_warp = pl.rows_per_warp;
    launch_step(d, pl, sl, false, static_cast<cudaStream_t>(stream));
    SWE_CK(cudaGetLastError());
    return SWE_OK;
}

int swe_max_inverse_dt(swe_domain_t d, const float* h, const float* hu, const float* hv,
                       int64_t pitch, float* max_inverse_dt_out, void* stream) {
    if (!d || !max_inverse_dt_out) return fail(SWE_ERR_INVALID, "null argument");
    int rc = check_state_ptrs(h, hu, hv, pitch, d->dd.cols);
    if (rc) return rc;
    rc = ensure_parts(d, reduce_blocks(d));
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    SWE_CK(cudaMemsetAsync(d->ctl_scratch, 0, sizeof(Control), st));
    launch_reduce(d, StateView{h, hu, hv, pitch}, d->ctl_scratch, st);
    SWE_CK(cudaGetLastError());
    SWE_CK(cudaMemcpyAsync(&d->ctl_host[0], d->ctl_scratch, kControlHead, cudaMemcpyDeviceToHost, st));
    SWE_CK(cudaStreamSynchronize(st));
    *max_inverse_dt_out = d->ctl_host[0].maxinv;
    return SWE_OK;
}

int swe_cfl_dt(swe_domain_t d, const float* h, const float* hu, const float* hv, int64_t pitch,
               double* dt_out, void* stream) {
    if (!dt_out) return fail(SWE_ERR_INVALID, "null argument");
    float m = 0.f;
    const int rc = swe_max_inverse_dt(d, h, hu, hv, pitch, &m, stream);
    if (rc) return rc;
    const double md = (double)m;
    if (md > 0.0) {
        const double c = d->dd.cfl / md;
        *dt_out = c < d->dd.max_dt ? c : d->dd.max_dt;
    } else {
        *dt_out = d->dd.max_dt;
    }
    return SWE_OK;
}

int swe_run(swe_domain_t d, const float* h0, const float* hu0, const float* hv0, int64_t pitch_in,
            const float* output_times, int32_t n_out, int32_t max_steps, float* out_h,
            float* out_hu, float* out_hv, swe_run_result* result, void* stream) {
    if (!d || !result) return fail(SWE_ERR_INVALID, "null argument");
    int rc = check_state_ptrs(h0, hu0, hv0, pitch_in, d->dd.cols);
    if (rc) return rc;
    if (!output_times || n_out < 1)
        return fail(SWE_ERR_INVALID, "Output times must be one-dimensional, start at zero, and increase.");
    if (output_times[0] != 0.0f)
        return fail(SWE_ERR_INVALID, "Output times must be one-dimensional, start at zero, and increase.");
    for (int i = 1; i < n_out; ++i)
        if (!(output_times[i] > output_times[i - 1]))
            return fail(SWE_ERR_INVALID, "Output times must be one-dimensional, start at zero, and increase.");
    if (max_steps < 0) return fail(SWE_ERR_INVALID, "max_steps must be >= 0");
    if (!out_h || !out_hu || !out_hv) return fail(SWE_ERR_INVALID, "output buffers are required");
    rc = run_driver(d, StateView{h0, hu0, hv0, pitch_in}, output_times, n_out,
                    (double)output_times[0], n_out, max_steps, out_h, out_hu, out_hv, result,
                    static_cast<cudaStream_t>(stream), nullptr);
    if (rc) return rc;
    if (result->status == SWE_ERR_MAX_STEPS) {
        char msg[256];
        std::snprintf(msg, sizeof msg, "max_steps=%d wrote %d/%d outputs; last time=%.3f s.",
                      max_steps, result->outputs_written, n_out, result->final_time_s);
        return fail(SWE_ERR_MAX_STEPS, msg);
    }
    if (result->status == SWE_ERR_NONFINITE)
        return fail(SWE_ERR_NONFINITE, "non-finite values reached the CFL reduction");
    return SWE_OK;
}

int swe_run_host(swe_domain_t d, const float* h0, const float* hu0, const float* hv0, int64_t pitch_in,
                 const float* output_times, int32_t n_out, int32_t max_steps, float* out_h, float* out_hu,
                 float* out_hv, swe_run_result* result, void* stream) {
    if (!d || !result) return fail(SWE_ERR_INVALID, "null argument");
    int rc = check_state_ptrs(h0, hu0, hv0, pitch_in, d->dd.cols);
    if (rc) return rc;
    if (!output_times || n_out < 1 || output_times[0] != 0.0f)
        return fail(SWE_ERR_INVALID, "Output times must be one-dimensional, start at zero, and increase.");
    for (int i = 1; i < n_out; ++i)
        if (!(output_times[i] > output_times[i - 1]))
            return fail(SWE_ERR_INVALID, "Output times must be one-dimensional, start at zero, and increase.");
    if (max_steps < 0) return fail(SWE_ERR_INVALID, "max_steps must be >= 0");
    if (!out_h || !out_hu || !out_hv) return fail(SWE_ERR_INVALID, "output buffers are required");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int rows = d->dd.rows, cols = d->dd.cols;
    const int64_t plane = (int64_t)rows * cols;
    rc = ensure_ping(d);
    if (rc) return rc;
    const Plan pl = make_plan(d, d->run_vec, true);
    rc = ensure_parts(d, std::max(pl.blocks, reduce_blocks(d)));
    if (rc) return rc;
    // Device staging: the initial state in ping buffer 1 and one plane triple per output.
    const int64_t need = (int64_t)n_out * 3 * plane;
    if (need > d->snap_cap) {
        cudaFree(d->snap_dev);
        d->snap_dev = nullptr;
        d->snap_cap = 0;
        SWE_CK(cudaMalloc(&d->snap_dev, sizeof(float) * (size_t)need));
        d->snap_cap = need;
    }
    if (!d->copy_stream) SWE_CK(cudaStreamCreateWithFlags(&d->copy_stream, cudaStreamNonBlocking));
    if (!d->snap_ev) SWE_CK(cudaEventCreateWithFlags(&d->snap_ev, cudaEventDisableTiming));
    const float* hin[3] = {h0, hu0, hv0};
    for (int f = 0; f < 3; ++f)
        SWE_CK(cudaMemcpy2DAsync(d->ping[1][f], sizeof(float) * d->ppitch, hin[f], sizeof(float) * pitch_in,
                                 sizeof(float) * cols, rows, cudaMemcpyHostToDevice, st));
    float* sh = d->snap_dev;
    float* shu = sh + (int64_t)n_out * plane;
    float* shv = shu + (int64_t)n_out * plane;
    rc = begin_run(d, StateView{d->ping[1][0], d->ping[1][1], d->ping[1][2], d->ppitch}, output_times, n_out,
                   (double)output_times[0], n_out, max_steps, sh, shu, shv, st);
    if (rc) return rc;
    float* host[3] = {out_h, out_hu, out_hv};
    float* dev[3] = {sh, shu, shv};
    int copied = 0;
    // Copies output k to the host on the copy stream once `ev` (recorded after it was written) has passed.
    auto copy_out = [&](int upto, cudaEvent_t ev) -> int {
        if (upto <= copied) return SWE_OK;
        SWE_CK(cudaStreamWaitEvent(d->copy_stream, ev, 0));
        for (int f = 0; f < 3; ++f)
            SWE_CK(cudaMemcpyAsync(host[f] + (int64_t)copied * plane, dev[f] + (int64_t)copied * plane,
                                   sizeof(float) * (size_t)(upto - copied) * plane, cudaMemcpyDeviceToHost,
                                   d->copy_stream));
        copied = upto;
        return SWE_OK;
    };
    SWE_CK(cudaEventRecord(d->snap_ev, st));
    rc = copy_out(1, d->snap_ev);  // output 0 is the initial state
    if (rc) return rc;
    d->launches = 1;
    d->timed_valid = false;
    int64_t launched = 0;
    int chunk = 0;
    for (;;) {
        const int64_t todo = std::min<int64_t>(kChunk, (int64_t)max_steps - launched);
        rc = enqueue_run_steps(d, launched, todo, st);
        if (rc) return rc;
        launched += todo;
        d->launches += todo;
        const int slot = chunk & 1;
        SWE_CK(cudaMemcpyAsync(&d->ctl_host[slot], d->ctl, kControlHead, cudaMemcpyDeviceToHost, st));
        SWE_CK(cudaEventRecord(d->poll_ev[slot], st));
        if (launched >= max_steps) break;
        if (chunk > 0) {
            // The previous chunk has finished: outputs it recorded go to the host
            // while the chunk just queued runs.
            SWE_CK(cudaEventSynchronize(d->poll_ev[slot ^ 1]));
            const Control& c = d->ctl_host[slot ^ 1];
            rc = copy_out(std::min(c.idx, n_out), d->poll_ev[slot ^ 1]);
            if (rc) return rc;
            if (c.done) break;
        }
        ++chunk;
    }
    rc = fold_ledger(d, pl.blocks, st);
    if (rc) return rc;
    SWE_CK(cudaStreamSynchronize(st));
    SWE_CK(cudaMemcpy(&d->ctl_host[0], d->ctl, kControlHead, cudaMemcpyDeviceToHost));
    const Control& c = d->ctl_host[0];
    SWE_CK(cudaEventRecord(d->snap_ev, st));
    rc = copy_out(std::min(c.idx, n_out), d->snap_ev);
    if (rc) return rc;
    SWE_CK(cudaStreamSynchronize(d->copy_stream));
    result->final_time_s = c.t;
    result->outputs_written = c.idx;
    result->steps_used = c.steps;
    result->status = c.status ? c.status : (c.idx >= n_out ? SWE_OK : SWE_ERR_MAX_STEPS);
    result->reserved = 0;
    for (int i = 0; i < 6; ++i) result->ledger[i] = c.ledger[i];
    if (result->status == SWE_ERR_MAX_STEPS) {
        char msg[256];
        std::snprintf(msg, sizeof msg, "max_steps=%d wrote %d/%d outputs; last time=%.3f s.", max_steps,
                      result->outputs_written, n_out, result->final_time_s);
        return fail(SWE_ERR_MAX_STEPS, msg);
    }
    if (result->status == SWE_ERR_NONFINITE) return fail(SWE_ERR_NONFINITE, "non-finite values reached the CFL reduction");
    return SWE_OK;
}

int swe_advance(swe_domain_t d, float* h, float* hu, float* hv, int64_t pitch, int32_t n_steps,
                double start_s, swe_run_result* result, void* stream) {
    if (!d || !result) return fail(SWE_ERR_INVALID, "null argument");
    int rc = check_state_ptrs(h, hu, hv, pitch, d->dd.cols);
    if (rc) return rc;
    if (n_steps < 0) return fail(SWE_ERR_INVALID, "n_steps must be >= 0");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const float times[2] = {(float)start_s, INFINITY};
    int fb = 0;
    rc = run_driver(d, StateView{h, hu, hv, pitch}, times, 2, start_s, 2, n_steps, nullptr,
                    nullptr, nullptr, result, st, &fb);
    if (rc) return rc;
    if (result->status == SWE_ERR_NONFINITE)
        return fail(SWE_ERR_NONFINITE, "non-finite values reached the CFL reduction");
    result->status = SWE_OK;
    float* outs[3] = {h, hu, hv};
    for (int f = 0; f < 3; ++f) {
        rc = copy_plane(outs[f], pitch, d->ping[fb][f], d->ppitch, d->dd.rows, d->dd.cols, st);
        if (rc) return rc;
    }
    SWE_CK(cudaStreamSynchronize(st));
    return SWE_OK;
}

int64_t swe_last_launch_count(swe_domain_t d) { return d ? d->launches : -1; }

int swe_resident_load(swe_domain_t d, const float* h, const float* hu, const float* hv, int64_t pitch,
                      double start_s, void* stream) {
    if (!d) return fail(SWE_ERR_INVALID, "null domain");
    int rc = check_state_ptrs(h, hu, hv, pitch, d->dd.cols);
    if (rc) return rc;
    if (!std::isfinite(start_s)) return fail(SWE_ERR_INVALID, "start time must be finite");
    rc = ensure_ping(d);
    if (rc) return rc;
    rc = ensure_parts(d, std::max(make_plan(d, d->run_vec, true).blocks, reduce_blocks(d)));
    if (rc) return rc;
    // An open-ended run: no output target within reach and no step cap, so the
    // control block stops the steps only on a non-finite CFL maximum.
    const float times[2] = {(float)start_s, INFINITY};
    rc = begin_run(d, StateView{h, hu, hv, pitch}, times, 2, start_s, 2, INT32_MAX, nullptr, nullptr, nullptr,
                   static_cast<cudaStream_t>(stream));
    if (rc) return rc;
    d->resident = true;
    d->resident_steps = 0;
    d->launches = 1;
    return SWE_OK;
}

int swe_resident_steps(swe_domain_t d, int32_t n_steps, void* stream) {
    if (!d) return fail(SWE_ERR_INVALID, "null domain");
    if (!d->resident) return fail(SWE_ERR_INVALID, "no resident state: call swe_resident_load first");
    if (n_steps < 0) return fail(SWE_ERR_INVALID, "n_steps must be >= 0");
    const int rc = enqueue_run_steps(d, d->resident_steps, n_steps, static_cast<cudaStream_t>(stream));
    if (rc) return rc;
    d->resident_steps += n_steps;
    d->launches = n_steps;
    return SWE_OK;
}

int swe_resident_prepare(swe_domain_t d, int32_t n_steps) {
    if (!d) return fail(SWE_ERR_INVALID, "null domain");
    if (!d->resident) return fail(SWE_ERR_INVALID, "no resident state: call swe_resident_load first");
    if (n_steps < 0) return fail(SWE_ERR_INVALID, "n_steps must be >= 0");
    // Both starting buffers: the steps may follow an odd number of other steps.
    const int rc = enqueue_run_steps(d, d->resident_steps, n_steps, nullptr, false);
    if (rc) return rc;
    return enqueue_run_steps(d, d->resident_steps + 1, n_steps, nullptr, false);
}

int swe_resident_store(swe_domain_t d, float* h, float* hu, float* hv, int64_t pitch, swe_run_result* result,
                       void* stream) {
    if (!d || !result) return fail(SWE_ERR_INVALID, "null argument");
    if (!d->resident) return fail(SWE_ERR_INVALID, "no resident state: call swe_resident_load first");
    int rc = check_state_ptrs(h, hu, hv, pitch, d->dd.cols);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int fb = (int)(d->resident_steps & 1);
    float* outs[3] = {h, hu, hv};
    for (int f = 0; f < 3; ++f) {
        rc = copy_plane(outs[f], pitch, d->ping[fb][f], d->ppitch, d->dd.rows, d->dd.cols, st);
        if (rc) return rc;
    }
    rc = fold_ledger(d, make_plan(d, d->run_vec, true).blocks, st);
    if (rc) return rc;
    SWE_CK(cudaMemcpyAsync(&d->ctl_host[0], d->ctl, kControlHead, cudaMemcpyDeviceToHost, st));
    SWE_CK(cudaStreamSynchronize(st));
    const Control& c = d->ctl_host[0];
    result->final_time_s = c.t;
    result->outputs_written = 0;
    result->steps_used = c.steps;
    result->status = c.status;
    result->reserved = 0;
    for (int i = 0; i < 6; ++i) result->ledger[i] = c.ledger[i];
    if (c.status == SWE_ERR_NONFINITE) return fail(SWE_ERR_NONFINITE, "non-finite values reached the CFL reduction");
    return SWE_OK;
}

int swe_advance_to(swe_domain_t d, float* h, float* hu, float* hv, int64_t pitch, double t_start,
                   double t_target, int32_t max_steps, double* dt_log, swe_run_result* result, void* stream) {
    if (!d || !result) return fail(SWE_ERR_INVALID, "null argument");
    int rc = check_state_ptrs(h, hu, hv, pitch, d->dd.cols);
    if (rc) return rc;
    if (!(t_target >= t_start) || max_steps < 0) return fail(SWE_ERR_INVALID, "need t_target >= t_start and max_steps >= 0");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const float times[2] = {(float)t_start, (float)t_target};
    const double times64[2] = {t_start, t_target};
    int fb = 0;
    rc = run_driver(d, StateView{h, hu, hv, pitch}, times, 2, t_start, 2, max_steps, nullptr, nullptr, nullptr,
                    result, st, &fb, times64, dt_log);
    if (rc) return rc;
    float* outs[3] = {h, hu, hv};
    for (int f = 0; f < 3; ++f) {
        rc = copy_plane(outs[f], pitch, d->ping[fb][f], d->ppitch, d->dd.rows, d->dd.cols, st);
        if (rc) return rc;
    }
    SWE_CK(cudaStreamSynchronize(st));
    if (result->status == SWE_ERR_NONFINITE) return fail(SWE_ERR_NONFINITE, "non-finite values reached the CFL reduction");
    if (result->status == SWE_ERR_MAX_STEPS) {
        char msg[160];
        std::snprintf(msg, sizeof msg, "max_steps=%d did not reach t=%.6f s (stopped at %.6f s)", max_steps,
                      t_target, result->final_time_s);
        return fail(SWE_ERR_MAX_STEPS, msg);
    }
    return SWE_OK;
}

int swe_network_features(swe_domain_t d, const float* h, const float* hu, const float* hv, int64_t pitch,
                         int32_t layout, const float* mean, const float* stddev, float rain_feature,
                         const float* terrain, const float* roughness, void* out, int32_t out_bf16,
                         void* stream) {
    if (!d || !out || !mean || !stddev) return fail(SWE_ERR_INVALID, "null argument");
    int rc = check_state_ptrs(h, hu, hv, pitch, d->dd.cols);
    if (rc) return rc;
    if (layout != kFeatRef6 && layout != kFeatState5) return fail(SWE_ERR_INVALID, "unknown feature layout");
    FeatureArgs a{};
    a.rows = d->dd.rows;
    a.cols = d->dd.cols;
    a.s = StateView{h, hu, hv, pitch};
    a.nm = d->nm;
    a.bed = d->bed;
    a.spitch = d->dd.spitch;
    a.terrain = terrain;
    a.roughness = roughness;
    const int nstat = layout == kFeatRef6 ? 3 : 5;
    for (int q = 0; q < 5; ++q) {
        a.mean[q] = q < nstat ? mean[q] : 0.f;
        const float sd = q < nstat ? stddev[q] : 1.f;
        if (!(sd > 0.f)) return fail(SWE_ERR_INVALID, "standard deviations must be positive");
        a.stdv[q] = sd;
    }
    a.rain_feature = rain_feature;
    a.dry = d->dd.k.dry;
    a.layout = layout;
    a.channels = layout == kFeatRef6 ? 6 : 5;
    a.out = out;
    a.out_bf16 = out_bf16 ? 1 : 0;
    features_kernel<<<cell_grid(a.rows, a.cols, 256, d->sms), 256, 0, static_cast<cudaStream_t>(stream)>>>(a);
    SWE_CK(cudaGetLastError());
    return SWE_OK;
}

int swe_output_fields(swe_domain_t d, const float* h, const float* hu, const float* hv, int64_t pitch,
                      float* depth, float* x_velocity, float* y_velocity, float* speed, int64_t out_pitch,
                      void* stream) {
    if (!d || !depth || !x_velocity || !y_velocity || !speed) return fail(SWE_ERR_INVALID, "null argument");
    int rc = check_state_ptrs(h, hu, hv, pitch, d->dd.cols);
    if (rc) return rc;
    if (out_pitch < d->dd.cols) return fail(SWE_ERR_INVALID, "output pitch smaller than the column count");
    SchemaArgs a{};
    a.rows = d->dd.rows;
    a.cols = d->dd.cols;
    a.s = StateView{h, hu, hv, pitch};
    a.nm = d->nm;
    a.spitch = d->dd.spitch;
    a.dry = d->dd.k.dry;
    a.depth = depth;
    a.u = x_velocity;
    a.v = y_velocity;
    a.speed = speed;
    a.out_pitch = out_pitch;
    schema_kernel<<<cell_grid(a.rows, a.cols, 256, d->sms), 256, 0, static_cast<cudaStream_t>(stream)>>>(a);
    SWE_CK(cudaGetLastError());
    return SWE_OK;
}

int swe_bias_act_nhwc(void* y, int64_t n, int32_t channels, const float* bias, int32_t relu, int32_t bf16,
                      int32_t device, void* stream) {
    if (!y || !bias || n < 0 || channels < 1 || n % channels) return fail(SWE_ERR_INVALID, "bad bias/activation arguments");
    if (n == 0) return SWE_OK;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool vec = bf16 && channels % 8 == 0 && reinterpret_cast<uintptr_t>(y) % 16 == 0;
    const int64_t work = vec ? n / 8 : n;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, (int64_t)sms * 16));
    auto* yb = static_cast<__nv_bfloat16*>(y);
    auto* yf = static_cast<float*>(y);
    if (vec) {
        if (relu) bias_act_bf16x8_kernel<true><<<blocks, 256, 0, st>>>(yb, work, channels, bias);
        else bias_act_bf16x8_kernel<false><<<blocks, 256, 0, st>>>(yb, work, channels, bias);
    } else if (bf16) {
        if (relu) bias_act_scalar_kernel<__nv_bfloat16, true><<<blocks, 256, 0, st>>>(yb, n, channels, bias);
        else bias_act_scalar_kernel<__nv_bfloat16, false><<<blocks, 256, 0, st>>>(yb, n, channels, bias);
    } else {
        if (relu) bias_act_scalar_kernel<float, true><<<blocks, 256, 0, st>>>(yf, n, channels, bias);
        else bias_act_scalar_kernel<float, false><<<blocks, 256, 0, st>>>(yf, n, channels, bias);
    }
    SWE_CK(cudaGetLastError());
    return SWE_OK;
}

int swe_apply_correction(swe_domain_t d, const float* h, const float* hu, const float* hv, int64_t pitch,
                         const void* residual, int32_t residual_bf16, int64_t res_stride_row,
                         int64_t res_stride_col, int64_t res_stride_channel, int32_t res_channels,
                         const float* clip_limits, double relaxation, float* h_out, float* hu_out,
                         float* hv_out, int64_t out_pitch, void* stream) {
    if (!d || !residual) return fail(SWE_ERR_INVALID, "null argument");
    int rc = check_state_ptrs(h, hu, hv, pitch, d->dd.cols);
    if (rc) return rc;
    rc = check_state_ptrs(h_out, hu_out, hv_out, out_pitch, d->dd.cols);
    if (rc) return rc;
    if (res_channels != 1 && res_channels != 3) return fail(SWE_ERR_INVALID, "residual must have 1 or 3 channels");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!d->corr_sums) SWE_CK(cudaMalloc(&d->corr_sums, 2 * sizeof(double)));
    if (!d->corr_prov) SWE_CK(cudaMalloc(&d->corr_prov, sizeof(float) * (size_t)d->dd.spitch * d->dd.rows));
    SWE_CK(cudaMemsetAsync(d->corr_sums, 0, 2 * sizeof(double), st));
    CorrectionArgs a{};
    a.rows = d->dd.rows;
    a.cols = d->dd.cols;
    a.s = StateView{h, hu, hv, pitch};
    a.out = StateOut{h_out, hu_out, hv_out, out_pitch};
    a.prov = d->corr_prov;
    a.prov_pitch = d->dd.spitch;
    a.nm = d->nm;
    a.spitch = d->dd.spitch;
    a.res = residual;
    a.rs_r = res_stride_row;
    a.rs_c = res_stride_col;
    a.rs_ch = res_stride_channel;
    a.res_channels = res_channels;
    a.res_bf16 = residual_bf16 ? 1 : 0;
    for (int q = 0; q < 3; ++q) {
        a.lim[q] = (clip_limits && q < res_channels) ? clip_limits[q] : INFINITY;
        if (!(a.lim[q] >= 0.f)) return fail(SWE_ERR_INVALID, "clip limits must be >= 0");
    }
    a.relax = (float)relaxation;
    a.dry = d->dd.k.dry;
    a.eps = 1.1920929e-07f;  // float32 machine epsilon (jnp.finfo(float32).eps)
    a.sums = d->corr_sums;
    const dim3 grid = cell_grid(a.rows, a.cols, 256, d->sms);
    correction_sums_kernel<<<grid, 256, 0, st>>>(a);
    correction_apply_kernel<<<grid, 256, 0, st>>>(a);
    SWE_CK(cudaGetLastError());
    return SWE_OK;
}


int swe_rollout_forward(swe_domain_t d, float* h, float* hu, float* hv, int64_t pitch, int32_t n_steps,
                        double dt, double t0, const double* dts, const int64_t* gauge_index, int32_t n_gauges,
                        int32_t obs_every, float* obs, float* ckpt, int32_t ckpt_every, void* stream) {
    if (!d) return fail(SWE_ERR_INVALID, "null domain");
    int rc = check_state_ptrs(h, hu, hv, pitch, d->dd.cols);
    if (rc) return rc;
    if (n_steps < 0 || (n_gauges > 0 && (!gauge_index || !obs || obs_every < 1)) || (ckpt && ckpt_every < 1))
        return fail(SWE_ERR_INVALID, "bad rollout arguments");
    rc = ensure_ping(d);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int rows = d->dd.rows, cols = d->dd.cols;
    float* user[3] = {h, hu, hv};
    for (int f = 0; f < 3; ++f) {
        rc = copy_plane(d->ping[0][f], d->ppitch, user[f], pitch, rows, cols, st);
        if (rc) return rc;
    }
    const int64_t plane = (int64_t)rows * cols;
    for (int k = 0; k < n_steps; ++k) {
        const int src = k & 1;
        const double t = step_time(k, dt, t0, dts), dtk = dts ? dts[k] : dt;
        if (ckpt && k % ckpt_every == 0) {
            float* dst = ckpt + (int64_t)(k / ckpt_every) * 3 * plane;
            for (int f = 0; f < 3; ++f) {
                rc = copy_plane(dst + f * plane, cols, d->ping[src][f], d->ppitch, rows, cols, st);
                if (rc) return rc;
            }
        }
        rc = swe_step(d, d->ping[src][0], d->ping[src][1], d->ping[src][2], d->ppitch, d->ping[src ^ 1][0],
                      d->ping[src ^ 1][1], d->ping[src ^ 1][2], d->ppitch, dtk, t, stream);
        if (rc) return rc;
        if (n_gauges > 0 && (k + 1) % obs_every == 0) {
            gauge_gather_kernel<<<(n_gauges + 127) / 128, 128, 0, st>>>(
                d->ping[src ^ 1][0], d->ppitch, cols, gauge_index, n_gauges,
                obs + (int64_t)((k + 1) / obs_every - 1) * n_gauges);
        }
    }
    const int fb = n_steps & 1;
    for (int f = 0; f < 3; ++f) {
        rc = copy_plane(user[f], pitch, d->ping[fb][f], d->ppitch, rows, cols, st);
        if (rc) return rc;
    }
    SWE_CK(cudaGetLastError());
    return SWE_OK;
}

int swe_rollout_backward(swe_domain_t d, const float* ckpt, int32_t ckpt_every, int32_t n_steps, double dt,
                         double t0, const double* dts, const int64_t* gauge_index, int32_t n_gauges,
                         int32_t obs_every, const float* grad_obs, float* lam_h, float* lam_hu, float* lam_hv,
                         int64_t lam_pitch, int32_t lam_in, float* grad_n2, double* grad_rain_scale, float* seg,
                         void* stream) {
    if (!d || !ckpt || !seg || ckpt_every < 1 || n_steps < 0) return fail(SWE_ERR_INVALID, "bad rollout arguments");
    if (n_gauges > 0 && (!gauge_index || !grad_obs || obs_every < 1)) return fail(SWE_ERR_INVALID, "bad gauge arguments");
    int rc = check_state_ptrs(lam_h, lam_hu, lam_hv, lam_pitch, d->dd.cols);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int rows = d->dd.rows, cols = d->dd.cols;
    const int64_t plane = (int64_t)rows * cols;
    if (!d->next_scratch) SWE_CK(cudaMalloc(&d->next_scratch, sizeof(float) * 3 * (size_t)plane));
    if (!d->lupd[0]) {
        d->lpitch = round_up(d->dd.cols, 128);
        for (int q = 0; q < 3; ++q) SWE_CK(cudaMalloc(&d->lupd[q], sizeof(float) * (size_t)d->lpitch * rows));
    }
    float* lam[3] = {lam_h, lam_hu, lam_hv};
    float* alt[3] = {d->lupd[0], d->lupd[1], d->lupd[2]};  // the other half of the lam ping-pong
    int cur = 0;  // 0: dL/dU of the current step is in lam, 1: in alt
    if (!lam_in)
        for (int f = 0; f < 3; ++f)
            SWE_CK(cudaMemset2DAsync(lam[f], sizeof(float) * lam_pitch, 0, sizeof(float) * cols, rows, st));
    const int nseg = n_steps > 0 ? (n_steps + ckpt_every - 1) / ckpt_every : 0;
    // Two segment buffers: the caller's `seg` and one of the domain's.  Segment
    // s-1 is recomputed on the domain's auxiliary stream while segment s is
    // reversed on the caller's stream (events order the reuse of a buffer), so
    // the recomputation overlaps the reverse steps instead of following them.
    const int64_t seg_floats = (int64_t)ckpt_every * 3 * plane;
    if (nseg > 1 && d->seg2_cap < seg_floats) {
        if (d->seg2) cudaFree(d->seg2);
        d->seg2 = nullptr;
        d->seg2_cap = 0;
        SWE_CK(cudaMalloc(&d->seg2, sizeof(float) * (size_t)seg_floats));
        d->seg2_cap = seg_floats;
    }
    if (!d->next_scratch2) SWE_CK(cudaMalloc(&d->next_scratch2, sizeof(float) * 3 * (size_t)plane));
    if (!d->aux_stream) SWE_CK(cudaStreamCreateWithFlags(&d->aux_stream, cudaStreamNonBlocking));
    for (cudaEvent_t& e : d->seg_ev)
        if (!e) SWE_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    cudaStream_t aux = d->aux_stream;
    cudaEvent_t ev_start = d->seg_ev[0], ev_end = d->seg_ev[5];
    cudaEvent_t* ev_rec = d->seg_ev + 1;   // segment buffer b recomputed
    cudaEvent_t* ev_used = d->seg_ev + 3;  // segment buffer b reversed (free again)
    float* segbuf[2] = {seg, d->seg2};
    float* nxtbuf[2] = {d->next_scratch, d->next_scratch2};
    // Recompute segment sgi's states U_k0 .. U_{k1-1} into segbuf[b] and U_{k1},
    // the output of its last step, into nxtbuf[b] (so that every reverse step can
    // rebuild its cell updates from its own output), on the auxiliary stream.
    auto recompute = [&](int sgi, int b) -> int {
        const int k0 = sgi * ckpt_every;
        const int k1 = std::min(k0 + ckpt_every, n_steps);
        float* sb = segbuf[b];
        SWE_CK(cudaMemcpyAsync(sb, ckpt + (int64_t)sgi * 3 * plane, sizeof(float) * 3 * plane,
                               cudaMemcpyDeviceToDevice, aux));
        for (int k = k0; k < k1; ++k) {
            const float* a = sb + (int64_t)(k - k0) * 3 * plane;
            float* o = k + 1 < k1 ? sb + (int64_t)(k + 1 - k0) * 3 * plane : nxtbuf[b];
            const int src = swe_step(d, a, a + plane, a + 2 * plane, cols, o, o + plane, o + 2 * plane, cols,
                                     dts ? dts[k] : dt, step_time(k, dt, t0, dts), aux);
            if (src) return src;
        }
        SWE_CK(cudaEventRecord(ev_rec[b], aux));
        return SWE_OK;
    };
    SWE_CK(cudaEventRecord(ev_start, st));  // the checkpoints and lam are ready on the caller's stream
    SWE_CK(cudaStreamWaitEvent(aux, ev_start, 0));
    // On every return the caller's stream waits for the auxiliary stream, so no
    // recomputation is left running into the caller's buffers after an error.
    auto join = [&](int status) {
        cudaEventRecord(ev_end, aux);
        cudaStreamWaitEvent(st, ev_end, 0);
        return status;
    };
    if (nseg > 0) {
        rc = recompute(nseg - 1, 0);
        if (rc) return join(rc);
    }
    for (int i = 0; i < nseg; ++i) {
        const int sgi = nseg - 1 - i, b = i & 1;
        const int k0 = sgi * ckpt_every;
        const int k1 = std::min(k0 + ckpt_every, n_steps);
        if (sgi > 0) {
            if (i >= 1 && cudaStreamWaitEvent(aux, ev_used[b ^ 1], 0) != cudaSuccess)  // buffer b^1 reversed
                return join(fail(SWE_ERR_CUDA, "cudaStreamWaitEvent failed"));
            rc = recompute(sgi - 1, b ^ 1);
            if (rc) return join(rc);
        }
        if (cudaStreamWaitEvent(st, ev_rec[b], 0) != cudaSuccess)
            return join(fail(SWE_ERR_CUDA, "cudaStreamWaitEvent failed"));
        const float* sb = segbuf[b];
        for (int k = k1 - 1; k >= k0; --k) {
            // dL/dU_{k+1} is in buffer `cur`; dL/dU_k goes to the other one (the fused
            // reverse step reads its neighbours' lam while it writes lam_out).
            float* const* src = cur ? alt : lam;
            float* const* dst = cur ? lam : alt;
            const int64_t sp = cur ? d->lpitch : lam_pitch, dp = cur ? lam_pitch : d->lpitch;
            if (n_gauges > 0 && (k + 1) % obs_every == 0) {
                gauge_inject_kernel<<<(n_gauges + 127) / 128, 128, 0, st>>>(
                    src[0], sp, cols, gauge_index, n_gauges, grad_obs + (int64_t)((k + 1) / obs_every - 1) * n_gauges);
            }
            const float* a = sb + (int64_t)(k - k0) * 3 * plane;
            const float* nx = k + 1 < k1 ? sb + (int64_t)(k + 1 - k0) * 3 * plane : nxtbuf[b];
            rc = adjoint_step_impl(d, a, a + plane, a + 2 * plane, cols, nx, cols, plane, src[0], src[1], src[2], sp,
                                   dst[0], dst[1], dst[2], dp, grad_n2, grad_rain_scale, dts ? dts[k] : dt,
                                   step_time(k, dt, t0, dts), st);
            if (rc) return join(rc);
            cur ^= 1;
        }
        if (cudaEventRecord(ev_used[b], st) != cudaSuccess) return join(fail(SWE_ERR_CUDA, "cudaEventRecord failed"));
    }
    join(SWE_OK);  // every recomputation is behind the caller's stream
    if (cur) {  // the result is in the alternate buffers: copy it to the caller's lam planes
        for (int f = 0; f < 3; ++f) {
            rc = copy_plane(lam[f], lam_pitch, alt[f], d->lpitch, rows, cols, st);
            if (rc) return rc;
        }
    }
    SWE_CK(cudaGetLastError());
    return SWE_OK;
}


int swe_ensemble_create(const swe_domain_desc* descs, int32_t n_members, swe_ensemble_t* out) {
    if (!descs || !out || n_members < 1) return fail(SWE_ERR_INVALID, "need at least one member descriptor");
    *out = nullptr;
    for (int m = 1; m < n_members; ++m)
        if (descs[m].arithmetic != descs[0].arithmetic)
            return fail(SWE_ERR_INVALID, "all ensemble members must use the same arithmetic");
    swe_ensemble* e = new swe_ensemble();
    e->arith = descs[0].arithmetic;
    if (const char* v = std::getenv("SWE_ENSEMBLE_ROWS")) {
        const int r = std::atoi(v);
        if (r > 0) e->rows_per_warp = r;
    }
    for (int m = 0; m < n_members; ++m) {
        swe_domain_t d = nullptr;
        const int rc = swe_domain_create(&descs[m], &d);
        if (rc) {
            free_ensemble(e);
            return rc;
        }
        e->doms.push_back(d);
        e->masked = e->masked || d->masked;
        e->sms = d->sms;
    }
    int rc = ens_rebuild(e);
    if (!rc && !std::getenv("SWE_ENSEMBLE_ROWS")) {
        const int R = ens_auto_rows(e);
        if (R != e->rows_per_warp) {
            e->rows_per_warp = R;
            rc = ens_rebuild(e);
        }
    }
    if (rc) {
        free_ensemble(e);
        return rc;
    }
    *out = e;
    return SWE_OK;
}

int32_t swe_ensemble_rows_per_warp(swe_ensemble_t e) { return e ? e->rows_per_warp : -1; }

int swe_ensemble_destroy(swe_ensemble_t e) {
    if (!e) return SWE_OK;
    cudaDeviceSynchronize();
    free_ensemble(e);
    return SWE_OK;
}

int swe_ensemble_size(swe_ensemble_t e) { return e ? (int)e->doms.size() : -1; }

int swe_ensemble_set_rows_per_warp(swe_ensemble_t e, int32_t rows_per_warp) {
    if (!e || rows_per_warp < 1) return fail(SWE_ERR_INVALID, "rows_per_warp must be >= 1");
    cudaDeviceSynchronize();
    e->rows_per_warp = rows_per_warp;
    return ens_rebuild(e);
}

int swe_ensemble_advance(swe_ensemble_t e, float* const* h, float* const* hu, float* const* hv,
                         const int64_t* pitch, int32_t n_steps, const double* start_s,
                         swe_run_result* results, void* stream) {
    if (!e || !h || !hu || !hv || !pitch || !results) return fail(SWE_ERR_INVALID, "null argument");
    if (n_steps < 0) return fail(SWE_ERR_INVALID, "n_steps must be >= 0");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int n = (int)e->doms.size();
    for (int m = 0; m < n; ++m) {
        swe_domain* d = e->doms[m];
        int rc = check_state_ptrs(h[m], hu[m], hv[m], pitch[m], d->dd.cols);
        if (rc) return rc;
        const double t0 = start_s ? start_s[m] : 0.0;
        const float times[2] = {(float)t0, INFINITY};
        rc = begin_run(d, StateView{h[m], hu[m], hv[m], pitch[m]}, times, 2, t0, 2, n_steps, nullptr,
                       nullptr, nullptr, st);
        if (rc) return rc;
    }
    const int K = 50;
    e->timed_valid = false;
    if (e->timing) {
        if (!e->time_ev[0]) {
            SWE_CK(cudaEventCreate(&e->time_ev[0]));
            SWE_CK(cudaEventCreate(&e->time_ev[1]));
        }
        SWE_CK(cudaEventRecord(e->time_ev[0], st));
    }
    int64_t done_steps = 0;
    if (n_steps >= K) {
        int rc = ens_graph(e, K);
        if (rc) return rc;
        for (; done_steps + K <= n_steps; done_steps += K) SWE_CK(cudaGraphLaunch(e->graph, st));
    }
    for (; done_steps < n_steps; ++done_steps) ens_launch(e, (int)(done_steps & 1), st);
    SWE_CK(cudaGetLastError());
    e->launches = n + n_steps;
    if (e->timing) {
        SWE_CK(cudaEventRecord(e->time_ev[1], st));
        e->timed_steps = n_steps;
        e->timed_valid = true;
    }
    return ens_collect(e, h, hu, hv, pitch, results, st, false);
}

int swe_ensemble_advance_to(swe_ensemble_t e, float* const* h, float* const* hu, float* const* hv,
                            const int64_t* pitch, const double* start_s, double target_s, int32_t max_steps,
                            double* const* dt_logs, swe_run_result* results, void* stream) {
    if (!e || !h || !hu || !hv || !pitch || !results || !start_s) return fail(SWE_ERR_INVALID, "null argument");
    if (max_steps < 0) return fail(SWE_ERR_INVALID, "max_steps must be >= 0");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int n = (int)e->doms.size();
    if (!e->done_counter) {
        SWE_CK(cudaMalloc(&e->done_counter, sizeof(unsigned)));
        SWE_CK(cudaHostAlloc(&e->done_host, 2 * sizeof(unsigned), cudaHostAllocDefault));
        SWE_CK(cudaEventCreateWithFlags(&e->poll_ev[0], cudaEventDisableTiming));
        SWE_CK(cudaEventCreateWithFlags(&e->poll_ev[1], cudaEventDisableTiming));
    }
    SWE_CK(cudaMemsetAsync(e->done_counter, 0, sizeof(unsigned), st));
    for (int m = 0; m < n; ++m) {
        swe_domain* d = e->doms[m];
        int rc = check_state_ptrs(h[m], hu[m], hv[m], pitch[m], d->dd.cols);
        if (rc) return rc;
        if (!(target_s >= start_s[m])) return fail(SWE_ERR_INVALID, "every start time must be <= the target");
        const float times[2] = {(float)start_s[m], (float)target_s};
        const double times64[2] = {start_s[m], target_s};
        d->done_counter = e->done_counter;
        rc = begin_run(d, StateView{h[m], hu[m], hv[m], pitch[m]}, times, 2, start_s[m], 2, max_steps, nullptr,
                       nullptr, nullptr, st, times64, dt_logs ? dt_logs[m] : nullptr);
        d->done_counter = nullptr;
        if (rc) return rc;
    }
    // K-step graphs until every member is done.  The counter is read one
    // graph late so the host never waits on the graph just queued.
    const int K = 50;
    e->timed_valid = false;
    if (e->timing) {
        if (!e->time_ev[0]) {
            SWE_CK(cudaEventCreate(&e->time_ev[0]));
            SWE_CK(cudaEventCreate(&e->time_ev[1]));
        }
        SWE_CK(cudaEventRecord(e->time_ev[0], st));
    }
    int rc = ens_graph(e, K);
    if (rc) return rc;
    const int64_t max_graphs = ((int64_t)max_steps + K - 1) / K;
    int64_t g = 0;
    e->done_host[0] = e->done_host[1] = 0;
    for (; g < max_graphs; ++g) {
        SWE_CK(cudaGraphLaunch(e->graph, st));
        SWE_CK(cudaMemcpyAsync(&e->done_host[g & 1], e->done_counter, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        SWE_CK(cudaEventRecord(e->poll_ev[g & 1], st));
        if (g > 0) {
            SWE_CK(cudaEventSynchronize(e->poll_ev[(g - 1) & 1]));
            if (e->done_host[(g - 1) & 1] >= (unsigned)n) {
                ++g;
                break;
            }
        }
    }
    e->launches = n + g * K;
    if (e->timing) {
        SWE_CK(cudaEventRecord(e->time_ev[1], st));
        e->timed_steps = g * K;
        e->timed_valid = true;
    }
    return ens_collect(e, h, hu, hv, pitch, results, st, true);
}

int swe_ensemble_member(swe_ensemble_t e, int32_t m, swe_domain_t* out) {
    if (!e || !out) return fail(SWE_ERR_INVALID, "null argument");
    if (m < 0 || m >= (int)e->doms.size()) return fail(SWE_ERR_INVALID, "member index out of range");
    *out = e->doms[m];
    return SWE_OK;
}

int swe_ensemble_set_timing(swe_ensemble_t e, int32_t enable) {
    if (!e) return fail(SWE_ERR_INVALID, "null ensemble");
    e->timing = enable != 0;
    return SWE_OK;
}

int swe_ensemble_last_step_time(swe_ensemble_t e, double* ms, int64_t* steps) {
    if (!e || !ms || !steps) return fail(SWE_ERR_INVALID, "null argument");
    if (!e->timed_valid) return fail(SWE_ERR_INVALID, "no timed advance recorded (call swe_ensemble_set_timing first)");
    float f = 0.f;
    SWE_CK(cudaEventElapsedTime(&f, e->time_ev[0], e->time_ev[1]));
    *ms = (double)f;
    *steps = e->timed_steps;
    return SWE_OK;
}

int64_t swe_ensemble_last_launch_count(swe_ensemble_t e) { return e ? e->launches : -1; }

int swe_ensemble_network_features(swe_ensemble_t e, float* const* h, float* const* hu, float* const* hv,
                                  const int64_t* pitch, int32_t layout, const float* mean, const float* stddev,
                                  const float* rain_features, const float* const* terrain,
                                  const float* const* roughness, void* out, int64_t out_member_stride,
                                  int32_t out_bf16, void* stream) {
    if (!e || !h || !hu || !hv || !pitch || !mean || !stddev || !rain_features || !out)
        return fail(SWE_ERR_INVALID, "null argument");
    if (out_member_stride < 0) return fail(SWE_ERR_INVALID, "out_member_stride must be >= 0");
    const size_t esz = out_bf16 ? 2 : 4;
    for (int m = 0; m < (int)e->doms.size(); ++m) {
        void* om = static_cast<char*>(out) + (size_t)m * (size_t)out_member_stride * esz;
        const int rc = swe_network_features(e->doms[m], h[m], hu[m], hv[m], pitch[m], layout, mean + 5 * m,
                                            stddev + 5 * m, rain_features[m], terrain ? terrain[m] : nullptr,
                                            roughness ? roughness[m] : nullptr, om, out_bf16, stream);
        if (rc) return rc;
    }
    return SWE_OK;
}

int swe_ensemble_apply_correction(swe_ensemble_t e, float* const* h, float* const* hu, float* const* hv,
                                  const int64_t* pitch, const void* residual, int32_t residual_bf16,
                                  int64_t res_stride_member, int64_t res_stride_row, int64_t res_stride_col,
                                  int64_t res_stride_channel, int32_t res_channels, const float* clip_limits,
                                  double relaxation, float* const* h_out, float* const* hu_out,
                                  float* const* hv_out, const int64_t* out_pitch, void* stream) {
    if (!e || !h || !hu || !hv || !pitch || !residual || !h_out || !hu_out || !hv_out || !out_pitch)
        return fail(SWE_ERR_INVALID, "null argument");
    if (res_channels != 1 && res_channels != 3) return fail(SWE_ERR_INVALID, "residual must have 1 or 3 channels");
    const size_t esz = residual_bf16 ? 2 : 4;
    for (int m = 0; m < (int)e->doms.size(); ++m) {
        const void* rm = static_cast<const char*>(residual) + (int64_t)m * res_stride_member * (int64_t)esz;
        const int rc = swe_apply_correction(e->doms[m], h[m], hu[m], hv[m], pitch[m], rm, residual_bf16,
                                            res_stride_row, res_stride_col, res_stride_channel, res_channels,
                                            clip_limits ? clip_limits + (size_t)res_channels * m : nullptr,
                                            relaxation, h_out[m], hu_out[m], hv_out[m], out_pitch[m], stream);
        if (rc) return rc;
    }
    return SWE_OK;
}


int swe_max_inverse_dt_noalloc(const float* h, const float* hu, const float* hv, int64_t pitch,
                               const uint8_t* domain_mask, int32_t rows, int32_t cols,
                               double gravity, double dry_tolerance, double dx, double dy,
                               float* max_inverse_dt_out, void* stream) {
    if (!h || !hu || !hv || !domain_mask || !max_inverse_dt_out)
        return fail(SWE_ERR_INVALID, "null argument");
    if (rows < 1 || cols < 1) return fail(SWE_ERR_INVALID, "rows and cols must be >= 1");
    if (pitch < cols) return fail(SWE_ERR_INVALID, "pitch must be >= cols");
    if (!(dx > 0) || !(dy > 0)) return fail(SWE_ERR_INVALID, "dx and dy must be positive");
    const int64_t n = (int64_t)rows * cols;
    if (n > SWE_NOALLOC_MAX_CELLS) {
        char msg[192];
        std::snprintf(msg, sizeof msg,
                      "rows*cols = %lld exceeds the allocation-free limit of %d cells; "
                      "use swe_max_inverse_dt with a domain instead",
                      (long long)n, SWE_NOALLOC_MAX_CELLS);
        return fail(SWE_ERR_INVALID, msg);
    }
    NoAllocScratch* scratch = nullptr;
    const int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    Consts k{};
    k.g = (float)gravity;
    k.half_g = (float)(0.5 * gravity);
    k.dry = (float)dry_tolerance;
    k.dx = (float)dx;
    k.dy = (float)dy;
    k.eps = (float)1.0e-12;
    k.expo = (float)(7.0 / 3.0);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // The ticket must start at zero; clear it in case an earlier launch was cut short.
    SWE_CK(cudaMemsetAsync(&scratch->ticket, 0, sizeof(unsigned), st));
    const int blocks = (int)((n + kNoAllocCellsPerBlock - 1) / kNoAllocCellsPerBlock);
    max_inverse_dt_noalloc_kernel<<<blocks, kNoAllocThreads, 0, st>>>(
        h, hu, hv, pitch, domain_mask, rows, cols, k, scratch, max_inverse_dt_out);
    SWE_CK(cudaGetLastError());
    return SWE_OK;
}


int swe_set_timing(swe_domain_t d, int32_t enable) {
    if (!d) return fail(SWE_ERR_INVALID, "null domain");
    if (enable && !d->time_ev[0]) {
        SWE_CK(cudaEventCreate(&d->time_ev[0]));
        SWE_CK(cudaEventCreate(&d->time_ev[1]));
    }
    d->timing = enable != 0;
    return SWE_OK;
}

int swe_last_step_time(swe_domain_t d, double* ms, int64_t* step_launches) {
    if (!d || !ms || !step_launches) return fail(SWE_ERR_INVALID, "null argument");
    if (!d->timed_valid) return fail(SWE_ERR_INVALID, "no timed run recorded (call swe_set_timing first)");
    float f = 0.f;
    SWE_CK(cudaEventElapsedTime(&f, d->time_ev[0], d->time_ev[1]));
    *ms = (double)f;
    *step_launches = d->timed_steps;
    return SWE_OK;
}


}  // extern "C"

// ---------------------------------------------------------------------------
// Device generators of the synthetic inputs (swe_generate_*)
// ---------------------------------------------------------------------------
namespace {

// Device scratch that frees itself (the generators are set-up calls).
// Scratch of the generators: a stream-ordered memory pool of the library's own
// per device, which keeps freed blocks for the next call (a plain cudaFree
// synchronises the whole device and returns the pages, which cost more than
// the generator's kernels).  Blocks are freed in stream order when the buffer
// goes out of scope, so a call returns without waiting for its kernels.
cudaMemPool_t scratch_pool(int dev) {
    static std::mutex mu;
    static std::vector<cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lock(mu);
    if ((int)pools.size() <= dev) pools.resize((size_t)dev + 1, nullptr);
    if (!pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        pools[dev] = p;
    }
    return pools[dev];
}

template <class T>
struct DevBuf {
    T* p = nullptr;
    cudaStream_t st = nullptr;
    ~DevBuf() {
        if (p) cudaFreeAsync(p, st);
    }
    cudaError_t alloc(size_t n, cudaStream_t s) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaMemPool_t pool = scratch_pool(dev);
        if (!pool) return cudaErrorMemoryAllocation;
        st = s;
        return cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p), sizeof(T) * std::max<size_t>(n, 1), pool, s);
    }
};

int gen_blocks(int64_t work, int sms) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, (int64_t)sms * 8));
}

int device_sms() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

}  // namespace

extern "C" {

int swe_generate_urban(const swe_urban_desc* q, float* bed, float* manning_n, uint8_t* block_mask,
                       int32_t* blocks_used, void* stream) {
    if (!q || !bed || !manning_n) return fail(SWE_ERR_INVALID, "null argument");
    if (q->rows < 1 || q->cols < 1) return fail(SWE_ERR_INVALID, "rows and cols must be >= 1");
    if (!(q->dx > 0)) return fail(SWE_ERR_INVALID, "dx must be positive");
    if (!(q->coverage >= 0.0 && q->coverage <= 1.0)) return fail(SWE_ERR_INVALID, "coverage must lie in [0, 1]");
    if (q->n_rects < 0 || (q->n_rects > 0 && !q->rects)) return fail(SWE_ERR_INVALID, "bad rectangle list");
    if (q->n_rects == 0 && (q->min_side < 1 || q->max_side < q->min_side))
        return fail(SWE_ERR_INVALID, "need 1 <= min_side <= max_side");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int rows = q->rows, cols = q->cols, sms = device_sms();
    const int64_t cells = (int64_t)rows * cols;
    const double target = q->coverage * (double)cells;
    DevBuf<int> first;
    SWE_CK(first.alloc((size_t)cells, st));
    int n_blocks = 0;
    // Drawn rectangles: a first batch about twice the expected need, doubled until it reaches the target.
    const double side = 0.5 * (q->min_side + q->max_side);
    int n = q->n_rects > 0 ? q->n_rects
                           : (int)std::min<double>(1 << 30, 2.0 * -std::log(std::max(1.0 - q->coverage, 1e-6)) *
                                                                (double)cells / (side * side) + 256.0);
    for (;;) {
        DevBuf<Rect> rects;
        DevBuf<int> counts;
        SWE_CK(rects.alloc((size_t)n, st));
        SWE_CK(counts.alloc((size_t)n, st));
        if (q->n_rects > 0) {
            std::vector<Rect> hr((size_t)n);
            for (int i = 0; i < n; ++i) {
                hr[i] = Rect{q->rects[4 * i], q->rects[4 * i + 1], q->rects[4 * i + 2], q->rects[4 * i + 3]};
                if (hr[i].r0 < 0 || hr[i].c0 < 0 || hr[i].h < 0 || hr[i].w < 0)
                    return fail(SWE_ERR_INVALID, "rectangles need non-negative corners and sides");
            }
            SWE_CK(cudaMemcpyAsync(rects.p, hr.data(), sizeof(Rect) * (size_t)n, cudaMemcpyHostToDevice, st));
        } else {
            gen_rects_kernel<<<(n + 255) / 256, 256, 0, st>>>(q->seed, n, rows, cols, q->min_side, q->max_side, rects.p);
        }
        SWE_CK(cudaMemsetAsync(first.p, 0x7f, sizeof(int) * (size_t)cells, st));  // 0x7f7f7f7f: no rectangle yet
        SWE_CK(cudaMemsetAsync(counts.p, 0, sizeof(int) * (size_t)n, st));
        rasterize_rects_kernel<<<std::min(n, sms * 16), 256, 0, st>>>(rects.p, n, rows, cols, first.p);
        first_histogram_kernel<<<gen_blocks(cells, sms), 256, 0, st>>>(first.p, cells, n, counts.p);
        SWE_CK(cudaGetLastError());
        std::vector<int> hc((size_t)n);
        SWE_CK(cudaMemcpyAsync(hc.data(), counts.p, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, st));
        SWE_CK(cudaStreamSynchronize(st));
        // The sequential rule: rectangles are added while the covered cells stay below the target.
        int64_t covered = 0;
        int k = 0;
        while (k < n && (double)covered < target) covered += hc[(size_t)k++];
        if ((double)covered >= target || q->n_rects > 0 || n >= (1 << 29)) {
            n_blocks = k;
            break;
        }
        n *= 2;
    }
    urban_fields_kernel<<<gen_blocks(cells, sms), 256, 0, st>>>(first.p, n_blocks, rows, cols, q->dx, q->slope,
                                                              q->block_raise_m, q->street_offset_m, q->n_block,
                                                              q->n_street, q->n_scale, bed, manning_n, block_mask);
    SWE_CK(cudaGetLastError());
    if (blocks_used) *blocks_used = n_blocks;
    return SWE_OK;
}

int swe_generate_gamma_hyetograph(int32_t n, double step_s, double shape_k, double scale, double to_m_s,
                                  uint64_t seed, float* times, float* rates, void* stream) {
    if (n < 1 || !times || !rates) return fail(SWE_ERR_INVALID, "need n >= 1 and output buffers");
    if (!(shape_k > 0) || !(scale > 0)) return fail(SWE_ERR_INVALID, "Gamma shape and scale must be positive");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    gamma_hyetograph_kernel<<<(n + 127) / 128, 128, 0, st>>>(seed, n, step_s, shape_k, scale, to_m_s, times, rates);
    SWE_CK(cudaGetLastError());
    return SWE_OK;
}

int swe_generate_lognormal_field(int32_t rows, int32_t cols, double median, double sigma_log, int32_t smooth_cells,
                                 uint64_t seed, const double* noise, float* out, void* stream) {
    if (rows < 1 || cols < 1 || !out) return fail(SWE_ERR_INVALID, "bad field arguments");
    if (!(median > 0) || !(sigma_log >= 0)) return fail(SWE_ERR_INVALID, "median must be > 0 and sigma_log >= 0");
    if (smooth_cells < 1) return fail(SWE_ERR_INVALID, "smooth_cells must be >= 1");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t cells = (int64_t)rows * cols;
    const int sms = device_sms();
    const int radius = smooth_cells / 2;
    // Gaussian taps of width smooth_cells (sigma = smooth_cells / 6), normalised to sum 1.
    std::vector<double> taps((size_t)(2 * radius + 1));
    double tsum = 0.0;
    const double sig = smooth_cells / 6.0;
    for (int t = -radius; t <= radius; ++t) {
        const double x = (double)t / sig;
        taps[(size_t)(t + radius)] = std::exp(-0.5 * x * x);
        tsum += taps[(size_t)(t + radius)];
    }
    for (auto& v : taps) v /= tsum;
    DevBuf<double> a, b, dtaps, partials, sums;
    SWE_CK(a.alloc((size_t)cells, st));
    SWE_CK(b.alloc((size_t)cells, st));
    SWE_CK(dtaps.alloc(taps.size(), st));
    SWE_CK(partials.alloc(kGenSumBlocks, st));
    SWE_CK(sums.alloc(2, st));
    SWE_CK(cudaMemcpyAsync(dtaps.p, taps.data(), sizeof(double) * taps.size(), cudaMemcpyHostToDevice, st));
    const double* src = noise;
    if (!src) {
        normal_field_kernel<<<gen_blocks(cells, sms), 256, 0, st>>>(seed, cells, a.p);
        src = a.p;
    }
    const unsigned gx = (unsigned)std::min<int64_t>((cols + 255) / 256, (int64_t)sms * 8);
    const dim3 sgrid(gx, (unsigned)std::max<int64_t>(1, std::min<int64_t>(rows, (int64_t)sms * 8 / gx)));
    smooth_pass_kernel<1><<<sgrid, 256, 0, st>>>(src, b.p, rows, cols, dtaps.p, radius);
    smooth_pass_kernel<0><<<sgrid, 256, 0, st>>>(b.p, a.p, rows, cols, dtaps.p, radius);
    // Two-pass moments: the mean, then the squared deviations from it.
    block_sums_kernel<256><<<kGenSumBlocks, 256, 0, st>>>(a.p, cells, nullptr, partials.p);
    fold_sums_kernel<<<1, 32, 0, st>>>(partials.p, kGenSumBlocks, sums.p);
    block_sums_kernel<256><<<kGenSumBlocks, 256, 0, st>>>(a.p, cells, sums.p, partials.p);
    fold_sums_kernel<<<1, 32, 0, st>>>(partials.p, kGenSumBlocks, sums.p + 1);
    lognormal_finish_kernel<<<gen_blocks(cells, sms), 256, 0, st>>>(a.p, cells, sums.p, median, sigma_log, out);
    SWE_CK(cudaGetLastError());
    return SWE_OK;
}

// ---------------------------------------------------------------------------
// Row strips of one domain (domain decomposition across GPUs)
// ---------------------------------------------------------------------------
// A strip owns global rows [row_begin, row_end) and also holds the row below
// and the row above it when they exist (halo rows, read as ordinary neighbours
// and never updated).  One step of the whole domain is, per strip: the step
// kernel over the owned rows (its warps leave the strip's CFL maximum in the
// stripes), stripe_fold_kernel (that maximum into the control block), the
// maximum over strips (NCCL all-reduce, or a kernel when all strips are in one
// process), which the next step of every strip plans from (the same dt on
// every strip), and the halo exchange of the new state (each strip's first and
// last owned rows to its neighbours).

}  // extern "C"

namespace {

// NCCL, opened at run time so that single-GPU users need no NCCL library.
struct NcclApi {
    ncclResult_t (*GetUniqueId)(ncclUniqueId*);
    ncclResult_t (*CommInitRankConfig)(ncclComm_t*, int, ncclUniqueId, int, ncclConfig_t*);
    ncclResult_t (*CommDestroy)(ncclComm_t);
    ncclResult_t (*CommAbort)(ncclComm_t);
    ncclResult_t (*CommGetAsyncError)(ncclComm_t, ncclResult_t*);
    ncclResult_t (*AllReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t, cudaStream_t);
    ncclResult_t (*Send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
    ncclResult_t (*Recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
    ncclResult_t (*GroupStart)();
    ncclResult_t (*GroupEnd)();
    const char* (*GetErrorString)(ncclResult_t);
};

const NcclApi* nccl_api() {
    static NcclApi api;
    static bool ok = false;
    static std::once_flag once;
    std::call_once(once, [] {
        void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
        if (!h) return;
        auto sym = [&](const char* name) { return dlsym(h, name); };
        api.GetUniqueId = reinterpret_cast<decltype(api.GetUniqueId)>(sym("ncclGetUniqueId"));
        api.CommInitRankConfig = reinterpret_cast<decltype(api.CommInitRankConfig)>(sym("ncclCommInitRankConfig"));
        api.CommDestroy = reinterpret_cast<decltype(api.CommDestroy)>(sym("ncclCommDestroy"));
        api.CommAbort = reinterpret_cast<decltype(api.CommAbort)>(sym("ncclCommAbort"));
        api.CommGetAsyncError = reinterpret_cast<decltype(api.CommGetAsyncError)>(sym("ncclCommGetAsyncError"));
        api.AllReduce = reinterpret_cast<decltype(api.AllReduce)>(sym("ncclAllReduce"));
        api.Send = reinterpret_cast<decltype(api.Send)>(sym("ncclSend"));
        api.Recv = reinterpret_cast<decltype(api.Recv)>(sym("ncclRecv"));
        api.GroupStart = reinterpret_cast<decltype(api.GroupStart)>(sym("ncclGroupStart"));
        api.GroupEnd = reinterpret_cast<decltype(api.GroupEnd)>(sym("ncclGroupEnd"));
        api.GetErrorString = reinterpret_cast<decltype(api.GetErrorString)>(sym("ncclGetErrorString"));
        ok = api.GetUniqueId && api.CommInitRankConfig && api.CommDestroy && api.CommAbort &&
             api.CommGetAsyncError && api.AllReduce && api.Send && api.Recv && api.GroupStart && api.GroupEnd &&
             api.GetErrorString;
    });
    return ok ? &api : nullptr;
}

// Maximum of the strips' CFL maxima into every strip's control block (one
// block).  The control blocks travel as a kernel parameter, so a step needs no
// device table.
constexpr int kMaxLocalStrips = 64;
struct StripCtls {
    Control* c[kMaxLocalStrips];
    int n;
};

__global__ void strips_max_kernel(const StripCtls t) {
    __shared__ float m;
    if (threadIdx.x == 0) {
        float v = 0.f;
        for (int i = 0; i < t.n; ++i) v = fmaxf(v, t.c[i]->maxinv);  // NaN already mapped to +inf
        m = v;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < t.n; i += blockDim.x) t.c[i]->maxinv = m;
}

// Local rows of a strip that take part in the halo exchange: the first and the
// last owned row go to the neighbour below and above, and arrive in local row
// 0 and local row rows-1 (the halo rows).  The one-process exchange and the
// NCCL exchange both use these offsets.
struct HaloRows {
    int send_below, recv_below;  // valid when the strip has a halo row below (upd_lo == 1)
    int send_above, recv_above;  // valid when the strip has a halo row above (upd_hi == rows - 1)
};

HaloRows halo_rows(const swe_domain* d) {
    return HaloRows{d->dd.upd_lo, 0, d->dd.upd_hi - 1, d->dd.rows - 1};
}

float* plane_row(swe_domain* d, int buf, int f, int row) {
    return d->ping[buf][f] + (int64_t)row * d->ppitch;
}

int strip_begin(swe_domain* d, float* h, float* hu, float* hv, int64_t pitch, double t0, int n_steps,
                cudaStream_t st) {
    int rc = check_state_ptrs(h, hu, hv, pitch, d->dd.cols);
    if (rc) return rc;
    rc = ensure_ping(d);
    if (rc) return rc;
    // One partial per CTA of the step kernel as well as of the reduction.
    rc = ensure_parts(d, std::max(make_plan(d, d->run_vec, true).blocks, reduce_blocks(d)));
    if (rc) return rc;
    const float times[2] = {(float)t0, INFINITY};
    return begin_run(d, StateView{h, hu, hv, pitch}, times, 2, t0, 2, n_steps, nullptr, nullptr, nullptr, st,
                     nullptr, nullptr, 1);
}

void strip_step(swe_domain* d, int k, cudaStream_t st) {
    const Plan pl = make_plan(d, d->run_vec, true);
    launch_step(d, pl, run_launch(d, pl, k), true, st);
}

int strip_finish(swe_domain* d, float* h, float* hu, float* hv, int64_t pitch, int n_steps, swe_run_result* r,
                 cudaStream_t st) {
    const int lrc = fold_ledger(d, make_plan(d, d->run_vec, true).blocks, st);
    if (lrc) return lrc;
    const int fb = n_steps & 1;
    float* outs[3] = {h, hu, hv};
    for (int f = 0; f < 3; ++f) {
        const int rc = copy_plane(outs[f], pitch, d->ping[fb][f], d->ppitch, d->dd.rows, d->dd.cols, st);
        if (rc) return rc;
    }
    SWE_CK(cudaMemcpyAsync(&d->ctl_host[0], d->ctl, kControlHead, cudaMemcpyDeviceToHost, st));
    SWE_CK(cudaStreamSynchronize(st));
    const Control& c = d->ctl_host[0];
    r->final_time_s = c.t;
    r->outputs_written = c.idx;
    r->steps_used = c.steps;
    r->status = c.status;
    r->reserved = 0;
    for (int i = 0; i < 6; ++i) r->ledger[i] = c.ledger[i];
    return SWE_OK;
}

// Seconds the host waits for NCCL work before it aborts the communicator
// (SWE_NCCL_TIMEOUT_S, default 120): a rank that never arrives then ends the
// others' collectives with an error instead of leaving them waiting.
double nccl_timeout_s() {
    if (const char* e = std::getenv("SWE_NCCL_TIMEOUT_S")) {
        const double v = std::atof(e);
        if (v > 0) return v;
    }
    return 120.0;
}

double now_s() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

}  // namespace

struct swe_comm {
    ncclComm_t comm = nullptr;
    int world = 1, rank = 0, device = 0;
    int* status_dev = nullptr;     // agreement flag (device int)
    int* status_host = nullptr;    // pinned copy of it
    cudaEvent_t ev = nullptr;      // completion of the enqueued NCCL work
    bool aborted = false;
};

namespace {

// Finishes a non-blocking NCCL call: waits (bounded) while the communicator
// reports ncclInProgress.
ncclResult_t nccl_settle(const NcclApi* api, swe_comm* c, ncclResult_t r) {
    const double deadline = now_s() + nccl_timeout_s();
    while (r == ncclInProgress) {
        if (now_s() > deadline) return ncclSystemError;
        usleep(100);
        if (api->CommGetAsyncError(c->comm, &r) != ncclSuccess) return ncclSystemError;
    }
    return r;
}

int nccl_abort(const NcclApi* api, swe_comm* c, const std::string& why) {
    if (c->comm && !c->aborted) {
        api->CommAbort(c->comm);
        c->aborted = true;
        c->comm = nullptr;
    }
    return fail(SWE_ERR_CUDA, "NCCL: " + why + " (communicator aborted; create a new one)");
}

// Waits for the work enqueued on `st` so far, at most the NCCL timeout; aborts
// the communicator when that runs out or NCCL reports an asynchronous error.
int nccl_wait(const NcclApi* api, swe_comm* c, cudaStream_t st) {
    SWE_CK(cudaEventRecord(c->ev, st));
    const double deadline = now_s() + nccl_timeout_s();
    for (;;) {
        const cudaError_t q = cudaEventQuery(c->ev);
        if (q == cudaSuccess) return SWE_OK;
        if (q != cudaErrorNotReady) return fail(SWE_ERR_CUDA, std::string("strip step: ") + cudaGetErrorString(q));
        ncclResult_t ae = ncclSuccess;
        if (api->CommGetAsyncError(c->comm, &ae) == ncclSuccess && ae != ncclSuccess && ae != ncclInProgress)
            return nccl_abort(api, c, api->GetErrorString(ae));
        if (now_s() > deadline) return nccl_abort(api, c, "timed out waiting for the other ranks");
        usleep(50);
    }
}

}  // namespace

extern "C" {

int swe_comm_unique_id(void* id_out) {
    if (!id_out) return fail(SWE_ERR_INVALID, "null argument");
    const NcclApi* api = nccl_api();
    if (!api) return fail(SWE_ERR_INVALID, "NCCL (libnccl.so.2) could not be loaded");
    ncclUniqueId id;
    const ncclResult_t r = api->GetUniqueId(&id);
    if (r != ncclSuccess) return fail(SWE_ERR_CUDA, std::string("NCCL: ") + api->GetErrorString(r));
    std::memcpy(id_out, &id, sizeof(id));
    return SWE_OK;
}

int swe_comm_create(const void* id, int32_t world, int32_t rank, swe_comm_t* out) {
    if (!id || !out || world < 1 || rank < 0 || rank >= world) return fail(SWE_ERR_INVALID, "bad communicator arguments");
    *out = nullptr;
    const NcclApi* api = nccl_api();
    if (!api) return fail(SWE_ERR_INVALID, "NCCL (libnccl.so.2) could not be loaded");
    ncclUniqueId uid;
    std::memcpy(&uid, id, sizeof(uid));
    auto* c = new swe_comm();
    c->world = world;
    c->rank = rank;
    cudaGetDevice(&c->device);
    auto bail = [&](int code) {
        if (c->ev) cudaEventDestroy(c->ev);
        cudaFree(c->status_dev);
        if (c->status_host) cudaFreeHost(c->status_host);
        delete c;
        return code;
    };
    if (cudaMalloc(&c->status_dev, sizeof(int)) != cudaSuccess ||
        cudaMallocHost(&c->status_host, sizeof(int)) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev, cudaEventDisableTiming) != cudaSuccess)
        return bail(fail(SWE_ERR_CUDA, "communicator scratch allocation failed"));
    // Non-blocking communicator: the host bounds every wait and can abort.
    ncclConfig_t cfg = NCCL_CONFIG_INITIALIZER;
    cfg.blocking = 0;
    ncclResult_t r = api->CommInitRankConfig(&c->comm, world, uid, rank, &cfg);
    if (r == ncclInProgress && c->comm) r = nccl_settle(api, c, r);
    if (r != ncclSuccess) {
        if (c->comm) api->CommAbort(c->comm);
        c->comm = nullptr;
        return bail(fail(SWE_ERR_CUDA, std::string("NCCL: communicator creation failed or timed out: ") +
                                           api->GetErrorString(r)));
    }
    *out = c;
    return SWE_OK;
}

int swe_comm_destroy(swe_comm_t c) {
    if (!c) return SWE_OK;
    const NcclApi* api = nccl_api();
    if (api && c->comm && !c->aborted) api->CommDestroy(c->comm);
    if (c->ev) cudaEventDestroy(c->ev);
    cudaFree(c->status_dev);
    if (c->status_host) cudaFreeHost(c->status_host);
    delete c;
    return SWE_OK;
}

int swe_strip_create(const swe_domain_desc* global, int32_t row_begin, int32_t row_end, swe_domain_t* out) {
    if (!global || !out) return fail(SWE_ERR_INVALID, "null argument");
    *out = nullptr;
    if (row_begin < 0 || row_end <= row_begin || row_end > global->rows)
        return fail(SWE_ERR_INVALID, "need 0 <= row_begin < row_end <= rows");
    const int lo = row_begin > 0 ? row_begin - 1 : 0;
    const int hi = row_end < global->rows ? row_end + 1 : row_end;
    swe_domain_desc q = *global;
    const int64_t off = (int64_t)lo * global->cols;
    q.rows = hi - lo;
    q.bed = global->bed + off;
    q.manning_n = global->manning_n + off;
    q.domain_mask = global->domain_mask + off;
    q.rainfall_multiplier = global->rainfall_multiplier ? global->rainfall_multiplier + off : nullptr;
    swe_domain_t d = nullptr;
    const int rc = swe_domain_create(&q, &d);
    if (rc) return rc;
    d->dd.upd_lo = row_begin - lo;
    d->dd.upd_hi = row_end - lo;
    d->strip_row_begin = row_begin;
    d->strip_row_end = row_end;
    d->strip_total_rows = global->rows;
    *out = d;
    return SWE_OK;
}

int swe_strip_layout(swe_domain_t d, int32_t* local_rows, int32_t* upd_lo, int32_t* upd_hi) {
    if (!d || !local_rows || !upd_lo || !upd_hi) return fail(SWE_ERR_INVALID, "null argument");
    *local_rows = d->dd.rows;
    *upd_lo = d->dd.upd_lo;
    *upd_hi = d->dd.upd_hi;
    return SWE_OK;
}

int swe_strips_advance(const swe_domain_t* strips, int32_t n, float* const* h, float* const* hu, float* const* hv,
                       const int64_t* pitch, int32_t n_steps, double t0, swe_run_result* results, void* stream) {
    if (!strips || n < 1 || !h || !hu || !hv || !pitch || !results || n_steps < 0)
        return fail(SWE_ERR_INVALID, "bad strip arguments");
    if (n > kMaxLocalStrips) return fail(SWE_ERR_INVALID, "at most 64 strips in one process");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int dev = 0;
    SWE_CK(cudaGetDevice(&dev));
    for (int i = 0; i < n; ++i) {
        const swe_domain* s = strips[i];
        if (!s || s->strip_total_rows < 0) return fail(SWE_ERR_INVALID, "every entry must be a strip (swe_strip_create)");
        if (s->device != dev) return fail(SWE_ERR_INVALID, "every strip must live on the current device");
        if (s->dd.cols != strips[0]->dd.cols || s->strip_total_rows != strips[0]->strip_total_rows)
            return fail(SWE_ERR_INVALID, "strips must come from one domain (same rows and cols)");
    }
    // Adjacent slices of the same domain, bottom to top, covering all its rows.
    if (strips[0]->strip_row_begin != 0 || strips[n - 1]->strip_row_end != strips[0]->strip_total_rows)
        return fail(SWE_ERR_INVALID, "strips must cover the domain from its first to its last row");
    for (int i = 0; i + 1 < n; ++i)
        if (strips[i]->strip_row_end != strips[i + 1]->strip_row_begin)
            return fail(SWE_ERR_INVALID, "strips must be given bottom to top, each starting where the previous ends");
    for (int i = 0; i < n; ++i) {
        const int rc = strip_begin(strips[i], h[i], hu[i], hv[i], pitch[i], t0, n_steps, st);
        if (rc) return rc;
    }
    StripCtls table{};
    table.n = n;
    for (int i = 0; i < n; ++i) table.c[i] = strips[i]->ctl;
    // The maximum across strips that the next step of every strip plans from:
    // the start reductions' maxima first, then each step's from its stripes.
    auto max_all = [&](bool fold) {
        if (fold)
            for (int i = 0; i < n; ++i) stripe_fold_kernel<<<1, 32, 0, st>>>(strips[i]->ctl);
        strips_max_kernel<<<1, 32, 0, st>>>(table);
    };
    int rc = SWE_OK;
    max_all(false);
    const int cols = strips[0]->dd.cols;
    for (int k = 0; k < n_steps && !rc; ++k) {
        for (int i = 0; i < n; ++i) strip_step(strips[i], k, st);
        max_all(true);
        const int b = (k + 1) & 1;
        for (int i = 0; i + 1 < n && !rc; ++i) {
            swe_domain* L = strips[i];
            swe_domain* U = strips[i + 1];
            const HaloRows hl = halo_rows(L), hu_ = halo_rows(U);
            for (int f = 0; f < 3 && !rc; ++f) {
                // L's last owned row -> U's halo row below; U's first owned row -> L's halo row above.
                if (cudaMemcpyAsync(plane_row(U, b, f, hu_.recv_below), plane_row(L, b, f, hl.send_above),
                                    sizeof(float) * cols, cudaMemcpyDeviceToDevice, st) ||
                    cudaMemcpyAsync(plane_row(L, b, f, hl.recv_above), plane_row(U, b, f, hu_.send_below),
                                    sizeof(float) * cols, cudaMemcpyDeviceToDevice, st))
                    rc = fail(SWE_ERR_CUDA, "halo copy failed");
            }
        }
    }
    if (!rc && cudaGetLastError() != cudaSuccess) rc = fail(SWE_ERR_CUDA, "strip step launch failed");
    for (int i = 0; i < n && !rc; ++i) rc = strip_finish(strips[i], h[i], hu[i], hv[i], pitch[i], n_steps, &results[i], st);
    cudaStreamSynchronize(st);
    if (rc) return rc;
    for (int i = 0; i < n; ++i)
        if (results[i].status) return fail(results[i].status, "a strip stopped with an error status");
    return SWE_OK;
}

// Every rank takes the same NCCL steps in the same order, error paths
// included: the argument checks and the set-up run first on every rank, then
// one all-reduce of their status decides for all ranks whether to go on; every
// later wait is bounded, and a wait that runs out aborts the communicator.
int swe_strip_advance_nccl(swe_domain_t d, swe_comm_t comm, int32_t rank_below, int32_t rank_above, float* h,
                           float* hu, float* hv, int64_t pitch, int32_t n_steps, double t0, swe_run_result* result,
                           void* stream) {
    const NcclApi* api = nccl_api();
    if (!api) return fail(SWE_ERR_INVALID, "NCCL (libnccl.so.2) could not be loaded");
    if (!comm || !comm->comm) return fail(SWE_ERR_INVALID, "no usable communicator");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // 1. Local checks and set-up, without returning before the agreement.
    int local = SWE_OK;
    std::string local_msg;
    if (!d || !result || n_steps < 0) {
        local = SWE_ERR_INVALID;
        local_msg = "bad strip arguments";
    } else if ((rank_below >= 0) != (d->dd.upd_lo == 1) || (rank_above >= 0) != (d->dd.upd_hi == d->dd.rows - 1)) {
        local = SWE_ERR_INVALID;
        local_msg = "neighbour ranks must match the strip's halo rows";
    } else {
        local = strip_begin(d, h, hu, hv, pitch, t0, n_steps, st);
        if (local) local_msg = g_err;
    }
    // 2. Agreement: the largest status over all ranks.
    *comm->status_host = local;
    SWE_CK(cudaMemcpyAsync(comm->status_dev, comm->status_host, sizeof(int), cudaMemcpyHostToDevice, st));
    ncclResult_t r = nccl_settle(api, comm, api->AllReduce(comm->status_dev, comm->status_dev, 1, ncclInt32, ncclMax,
                                                           comm->comm, st));
    if (r != ncclSuccess) return nccl_abort(api, comm, std::string("status all-reduce: ") + api->GetErrorString(r));
    SWE_CK(cudaMemcpyAsync(comm->status_host, comm->status_dev, sizeof(int), cudaMemcpyDeviceToHost, st));
    int rc = nccl_wait(api, comm, st);
    if (rc) return rc;
    if (local) return fail(local, local_msg);
    if (*comm->status_host) return fail(*comm->status_host, "another rank's strip arguments or set-up failed");
    // 3. The steps.  Each NCCL call is settled; the group is always closed.
    const int cols = d->dd.cols;
    const HaloRows hr = halo_rows(d);
    // The maximum across strips that the next step plans from: the start
    // reduction's maximum first, then each step's from its stripes.
    auto max_all = [&](bool fold) -> int {
        if (fold) stripe_fold_kernel<<<1, 32, 0, st>>>(d->ctl);
        const ncclResult_t e = nccl_settle(api, comm, api->AllReduce(&d->ctl->maxinv, &d->ctl->maxinv, 1, ncclFloat,
                                                                     ncclMax, comm->comm, st));
        if (e != ncclSuccess) return nccl_abort(api, comm, std::string("all-reduce: ") + api->GetErrorString(e));
        return SWE_OK;
    };
    rc = max_all(false);
    for (int k = 0; k < n_steps && !rc; ++k) {
        strip_step(d, k, st);
        rc = max_all(true);
        if (rc) break;
        const int b = (k + 1) & 1;
        ncclResult_t first = api->GroupStart();
        for (int f = 0; f < 3 && first == ncclSuccess; ++f) {
            auto keep = [&](ncclResult_t x) {
                if (first == ncclSuccess && x != ncclSuccess && x != ncclInProgress) first = x;
            };
            if (rank_below >= 0) {
                keep(api->Send(plane_row(d, b, f, hr.send_below), cols, ncclFloat, rank_below, comm->comm, st));
                keep(api->Recv(plane_row(d, b, f, hr.recv_below), cols, ncclFloat, rank_below, comm->comm, st));
            }
            if (rank_above >= 0) {
                keep(api->Send(plane_row(d, b, f, hr.send_above), cols, ncclFloat, rank_above, comm->comm, st));
                keep(api->Recv(plane_row(d, b, f, hr.recv_above), cols, ncclFloat, rank_above, comm->comm, st));
            }
        }
        const ncclResult_t end = nccl_settle(api, comm, api->GroupEnd());
        if (first == ncclSuccess) first = end;
        if (first != ncclSuccess) {
            rc = nccl_abort(api, comm, std::string("halo exchange: ") + api->GetErrorString(first));
            break;
        }
        // Bound the wait on the other ranks every kChunk steps.
        if ((k + 1) % kChunk == 0) rc = nccl_wait(api, comm, st);
    }
    if (!rc && cudaGetLastError() != cudaSuccess) rc = fail(SWE_ERR_CUDA, "strip step launch failed");
    if (!rc) rc = nccl_wait(api, comm, st);
    if (!rc) rc = strip_finish(d, h, hu, hv, pitch, n_steps, result, st);
    if (rc) return rc;
    if (result->status) return fail(result->status, "the strip stopped with an error status");
    return SWE_OK;
}

}  // extern "C"
