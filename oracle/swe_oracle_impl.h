/* Precision-generic body of the C oracle.  Included twice by swe_oracle.c with
 * REAL = float (suffix f32) and REAL = double (suffix f64).
 *
 * TEST INFRASTRUCTURE ONLY: the CPU restatement of the reference step used by
 * tests, smoke() and the CPU-baseline leg of bench.py.
 *
 * Every floating-point operation follows the order of the reference NumPy
 * solver (src/hybrid_flood/numpy_solver/shallow_water_2d.py) so that, compiled
 * with -ffp-contract=off, the float build matches it bit-for-bit except for
 * powf in the friction term (NumPy uses its own vectorised pow, within 1 ulp).
 */

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SUFFIX)

typedef struct {
    REAL f[3];     /* HLL flux (mass, x-momentum, y-momentum), zeroed if irrelevant */
    REAL corr_lo;  /* pressure correction seen by the lower-index cell (normal comp.) */
    REAL corr_hi;  /* ... by the higher-index cell */
} FN(face_t);

typedef struct {
    REAL h, hu, hv, z;
    int act;
} FN(cell_t);

/* shallow_water_2d.py:60-63 */
static inline REAL FN(vel)(REAL m, REAL h, REAL dry) {
    return h > dry ? m / (h > dry ? h : dry) : (REAL)0;
}

static inline REAL FN(rmax)(REAL a, REAL b) { return a > b ? a : b; }
static inline REAL FN(rmin)(REAL a, REAL b) { return a < b ? a : b; }

/* One face between cell `lo` and cell `hi`; axis 1 = x-face (normal momentum
 * hu), axis 0 = y-face (normal momentum hv).  shallow_water_2d.py:66-135 (HLL)
 * and :138-239 (walls, reconstruction, corrections). */
static inline void FN(face)(FN(cell_t) lo, FN(cell_t) hi, int axis, REAL g, REAL half_g,
                            REAL dry, FN(face_t) *out) {
    const int relevant = lo.act || hi.act;
    const int hi_wall = lo.act && !hi.act;
    const int lo_wall = !lo.act && hi.act;
    if (hi_wall) {
        hi = lo;
        if (axis == 1) hi.hu = -lo.hu; else hi.hv = -lo.hv;
        hi.act = 0;
    } else if (lo_wall) {
        lo = hi;
        if (axis == 1) lo.hu = -hi.hu; else lo.hv = -hi.hv;
        lo.act = 0;
    }
    const REAL zf = FN(rmax)(lo.z, hi.z);
    const REAL H0 = FN(rmax)(lo.h + lo.z - zf, (REAL)0);
    const REAL H1 = FN(rmax)(hi.h + hi.z - zf, (REAL)0);
    const REAL X0 = H0 * FN(vel)(lo.hu, lo.h, dry), Y0 = H0 * FN(vel)(lo.hv, lo.h, dry);
    const REAL X1 = H1 * FN(vel)(hi.hu, hi.h, dry), Y1 = H1 * FN(vel)(hi.hv, hi.h, dry);
    const REAL n0 = axis == 1 ? X0 : Y0, n1 = axis == 1 ? X1 : Y1;
    const REAL un0 = FN(vel)(n0, H0, dry), un1 = FN(vel)(n1, H1, dry);
    const REAL c0 = SQRT(g * FN(rmax)(H0, (REAL)0)), c1 = SQRT(g * FN(rmax)(H1, (REAL)0));
    const REAL s0 = FN(rmin)(un0 - c0, un1 - c1);
    const REAL s1 = FN(rmax)(un0 + c0, un1 + c1);
    const REAL p0 = half_g * (H0 * H0), p1 = half_g * (H1 * H1);
    REAL f0[3], f1[3];
    if (axis == 1) {
        f0[0] = X0; f0[1] = X0 * un0 + p0; f0[2] = X0 * FN(vel)(Y0, H0, dry);
        f1[0] = X1; f1[1] = X1 * un1 + p1; f1[2] = X1 * FN(vel)(Y1, H1, dry);
    } else {
        f0[0] = Y0; f0[1] = X0 * un0; f0[2] = Y0 * un0 + p0;
        f1[0] = Y1; f1[1] = X1 * un1; f1[2] = Y1 * un1 + p1;
    }
    const REAL u0[3] = {H0, X0, Y0}, u1[3] = {H1, X1, Y1};
    const REAL spread = s1 - s0;
    const REAL den = spread > (REAL)1.0e-12 ? spread : (REAL)1;
    const REAL s01 = s0 * s1;
    for (int k = 0; k < 3; ++k) {
        const REAL mid = (s1 * f0[k] - s0 * f1[k] + s01 * (u1[k] - u0[k])) / den;
        const REAL f = s0 >= (REAL)0 ? f0[k] : (s1 <= (REAL)0 ? f1[k] : mid);
        out->f[k] = relevant ? f : (REAL)0;
    }
    out->corr_lo = relevant ? half_g * (lo.h * lo.h - H0 * H0) : (REAL)0;
    out->corr_hi = relevant ? half_g * (hi.h * hi.h - H1 * H1) : (REAL)0;
}

/* Cell (r, c) including the ghost ring: edge copy, normal momentum negated on
 * reflective sides (boundary_conditions.py:29-52; bed and mask edge-padded as
 * shallow_water_2d.py:285-286). */
static inline FN(cell_t) FN(cell_at)(const FN(dom_) *d, const REAL *h, const REAL *hu,
                                    const REAL *hv, long r, long c) {
    const long rr = r < 0 ? 0 : (r >= d->rows ? d->rows - 1 : r);
    const long cc = c < 0 ? 0 : (c >= d->cols ? d->cols - 1 : c);
    const long i = rr * d->cols + cc;
    FN(cell_t) x;
    x.h = h[i]; x.hu = hu[i]; x.hv = hv[i];
    x.z = d->bed[i];
    x.act = d->mask[i] != 0;
    if ((c < 0 && d->boundary[0] == 0) || (c >= d->cols && d->boundary[1] == 0)) x.hu = -x.hu;
    if ((r < 0 && d->boundary[2] == 0) || (r >= d->rows && d->boundary[3] == 0)) x.hv = -x.hv;
    return x;
}

/* np.interp(t, times, rates, left=default, right=default) in double
 * (shallow_water_2d.py:254-264). */
static double FN(rain_rate)(const FN(dom_) *d, double t) {
    const int n = d->n_rain;
    if (n <= 0) return d->default_rain;
    const double x0 = (double)d->rain_times[0], xn = (double)d->rain_times[n - 1];
    if (t != t) return t;
    if (t < x0 || t > xn) return d->default_rain;
    if (n == 1 || t == xn) return (double)d->rain_rates[n - 1];
    int lo = 0, hi = n - 1; /* find j with times[j] <= t < times[j+1] */
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if ((double)d->rain_times[mid] <= t) lo = mid; else hi = mid;
    }
    const double xj = (double)d->rain_times[lo], yj = (double)d->rain_rates[lo];
    if (t == xj) return yj;
    const double xj1 = (double)d->rain_times[lo + 1], yj1 = (double)d->rain_rates[lo + 1];
    const double slope = (yj1 - yj) / (xj1 - xj);
    double v = slope * (t - xj) + yj;
    if (v != v) {
        v = slope * (t - xj1) + yj1;
        if (v != v && yj == yj1) v = yj;
    }
    return v;
}

double FN(oracle_rain_rate_)(const FN(dom_) *d, double t) { return FN(rain_rate)(d, t); }

/* Largest (|u|+c)/dx + (|v|+c)/dy over active cells (shallow_water_2d.py:269-273). */
double FN(oracle_max_inverse_dt_)(const FN(dom_) *d, const REAL *h, const REAL *hu,
                                  const REAL *hv) {
    const REAL dry = (REAL)d->dry, g = (REAL)d->g, dx = (REAL)d->dx, dy = (REAL)d->dy;
    const long n = (long)d->rows * d->cols;
    REAL best = 0;
#pragma omp parallel for reduction(max : best) schedule(static)
    for (long i = 0; i < n; ++i) {
        const REAL u = FN(vel)(hu[i], h[i], dry), v = FN(vel)(hv[i], h[i], dry);
        const REAL w = SQRT(g * FN(rmax)(h[i], (REAL)0));
        const REAL inv = (FABS(u) + w) / dx + (FABS(v) + w) / dy;
        const REAL m = d->mask[i] ? inv : (REAL)0;
        if (m > best || m != m) best = m;
    }
    return (double)best;
}

double FN(oracle_cfl_dt_)(const FN(dom_) *d, const REAL *h, const REAL *hu, const REAL *hv) {
    const double m = FN(oracle_max_inverse_dt_)(d, h, hu, hv);
    if (m > 0.0) {
        const double c = d->cfl / m;
        return c < d->max_dt ? c : d->max_dt;
    }
    return d->max_dt;
}

/* One step (shallow_water_2d.py:277-327).  `terms` (may be NULL) receives the
 * FP64 ledger increments in m^3: rain_in, outflow, clip_gain, mask_loss. */
int FN(oracle_step_)(const FN(dom_) *d, const REAL *h, const REAL *hu, const REAL *hv,
                     REAL *ho, REAL *huo, REAL *hvo, double dt, double time_s, double *terms) {
    const long R = d->rows, C = d->cols;
    const REAL g = (REAL)d->g, half_g = (REAL)(0.5 * d->g), dry = (REAL)d->dry;
    const REAL dxr = (REAL)d->dx, dyr = (REAL)d->dy;
    const REAL dtr = (REAL)dt;
    const REAL dt_rain = (REAL)(dt * FN(rain_rate)(d, time_s));
    const REAL dt_g = (REAL)(dt * d->g);
    const REAL expo = (REAL)(7.0 / 3.0);
    double rain_in = 0, outflow = 0, clip_gain = 0, mask_loss = 0;
    int nthreads = 1;
#ifdef _OPENMP
    nthreads = omp_get_max_threads();
#endif
    if (nthreads > R) nthreads = (int)R;
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel num_threads(nthreads) reduction(+ : rain_in, outflow, clip_gain, mask_loss)
    {
        int tid = 0, nt = 1;
#ifdef _OPENMP
        tid = omp_get_thread_num();
        nt = omp_get_num_threads();
#endif
        const long r0 = R * tid / nt, r1 = R * (tid + 1) / nt;
        FN(face_t) *xf = (FN(face_t) *)malloc(sizeof(FN(face_t)) * (size_t)(C + 1));
        FN(face_t) *ybot = (FN(face_t) *)malloc(sizeof(FN(face_t)) * (size_t)C);
        FN(face_t) *ytop = (FN(face_t) *)malloc(sizeof(FN(face_t)) * (size_t)C);
        for (long c = 0; c < C; ++c)
            FN(face)(FN(cell_at)(d, h, hu, hv, r0 - 1, c), FN(cell_at)(d, h, hu, hv, r0, c), 0, g,
                     half_g, dry, &ybot[c]);
        for (long r = r0; r < r1; ++r) {
            for (long c = 0; c <= C; ++c)
                FN(face)(FN(cell_at)(d, h, hu, hv, r, c - 1), FN(cell_at)(d, h, hu, hv, r, c), 1, g,
                         half_g, dry, &xf[c]);
            for (long c = 0; c < C; ++c)
                FN(face)(FN(cell_at)(d, h, hu, hv, r, c), FN(cell_at)(d, h, hu, hv, r + 1, c), 0, g,
                         half_g, dry, &ytop[c]);
            /* outer-face mass fluxes for the ledger */
            outflow += dt * ((double)xf[C].f[0] - (double)xf[0].f[0]) * d->dy;
            if (r == 0)
                for (long c = 0; c < C; ++c) outflow -= dt * (double)ybot[c].f[0] * d->dx;
            if (r == R - 1)
                for (long c = 0; c < C; ++c) outflow += dt * (double)ytop[c].f[0] * d->dx;
            for (long c = 0; c < C; ++c) {
                const long i = r * C + c;
                REAL upd[3];
                const REAL u_in[3] = {h[i], hu[i], hv[i]};
                for (int k = 0; k < 3; ++k) {
                    const REAL xl = xf[c + 1].f[k] + (k == 1 ? xf[c + 1].corr_lo : (REAL)0);
                    const REAL xr = xf[c].f[k] + (k == 1 ? xf[c].corr_hi : (REAL)0);
                    const REAL yb = ytop[c].f[k] + (k == 2 ? ytop[c].corr_lo : (REAL)0);
                    const REAL yt = ybot[c].f[k] + (k == 2 ? ybot[c].corr_hi : (REAL)0);
                    const REAL divx = (xl - xr) / dxr;
                    const REAL divy = (yb - yt) / dyr;
                    upd[k] = u_in[k] - dtr * (divx + divy);
                }
                const REAL rain = dt_rain * d->mult[i];
                upd[0] = upd[0] + rain;
                const REAL hn = FN(rmax)(upd[0], (REAL)0);
                const REAL norm = HYPOT(upd[1], upd[2]);
                const REAL n = d->manning[i];
                const REAL den = (REAL)1 + dt_g * (n * n) * norm / POW(FN(rmax)(hn, dry), expo);
                const REAL qx = upd[1] / den, qy = upd[2] / den;
                const int act = d->mask[i] != 0;
                const int wet = act && hn > dry;
                ho[i] = act ? hn : (REAL)0;
                huo[i] = wet ? qx : (REAL)0;
                hvo[i] = wet ? qy : (REAL)0;
                rain_in += (double)rain;
                if (upd[0] < 0) clip_gain -= (double)upd[0];
                if (!act) mask_loss += (double)hn;
            }
            FN(face_t) *t = ybot; ybot = ytop; ytop = t;
        }
        free(xf); free(ybot); free(ytop);
    }
    if (terms) {
        const double area = d->dx * d->dy;
        terms[0] += rain_in * area;
        terms[1] += outflow;
        terms[2] += clip_gain * area;
        terms[3] += mask_loss * area;
    }
    return 0;
}

double FN(oracle_volume_)(const FN(dom_) *d, const REAL *h) {
    const long n = (long)d->rows * d->cols;
    double s = 0;
    for (long i = 0; i < n; ++i)
        if (d->mask[i]) s += (double)h[i];
    return s * d->dx * d->dy;
}

/* Adaptive run to fixed output times (shallow_water_2d.py:382-424).
 * out: n_out x 3 x rows x cols.  ledger: volume0, volume, rain_in, outflow,
 * clip_gain, mask_loss.  Returns 0, or 1 when max_steps ran out. */
int FN(oracle_run_)(const FN(dom_) *d, const REAL *h0, const REAL *hu0, const REAL *hv0,
                    const float *times, int n_out, int max_steps, REAL *out, double *final_time,
                    int *steps_used, int *written, double *ledger) {
    const long n = (long)d->rows * d->cols;
    REAL *const buf0 = (REAL *)malloc(sizeof(REAL) * (size_t)n * 3);
    REAL *const buf1 = (REAL *)malloc(sizeof(REAL) * (size_t)n * 3);
    REAL *a = buf0, *b = buf1;
    memcpy(a, h0, sizeof(REAL) * (size_t)n);
    memcpy(a + n, hu0, sizeof(REAL) * (size_t)n);
    memcpy(a + 2 * n, hv0, sizeof(REAL) * (size_t)n);
    memcpy(out, a, sizeof(REAL) * (size_t)n * 3);
    double terms[4] = {0, 0, 0, 0};
    ledger[0] = FN(oracle_volume_)(d, a);
    double t = (double)times[0];
    int idx = 1, steps = 0;
    while (idx < n_out && steps < max_steps) {
        const double target = (double)times[idx];
        double dt = FN(oracle_cfl_dt_)(d, a, a + n, a + 2 * n);
        if (target - t < dt) dt = target - t;
        FN(oracle_step_)(d, a, a + n, a + 2 * n, b, b + n, b + 2 * n, dt, t, terms);
        REAL *tmp = a; a = b; b = tmp;
        t += dt;
        ++steps;
        if (t >= target - 1.0e-7) {
            memcpy(out + (size_t)idx * 3 * n, a, sizeof(REAL) * (size_t)n * 3);
            ++idx;
        }
    }
    ledger[1] = FN(oracle_volume_)(d, a);
    ledger[2] = terms[0]; ledger[3] = terms[1]; ledger[4] = terms[2]; ledger[5] = terms[3];
    *final_time = t;
    *steps_used = steps;
    *written = idx;
    free(buf0); free(buf1);
    return idx == n_out ? 0 : 1;
}

#undef FN
#undef CAT
#undef CAT_
