/* C restatement of the reference shallow-water step (test oracle).
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py (as the checker or the timed CPU baseline),
 * never by the product path.
 *
 * Restates src/hybrid_flood/numpy_solver/shallow_water_2d.py:60-424 with the
 * per-side boundary codes of src/hybrid_flood/jax_solver/boundary_conditions.py:29-52
 * and an FP64 mass ledger.  Build: see oracle/build.py (gcc -O3 -fopenmp
 * -ffp-contract=off, so float arithmetic is rounded operation by operation
 * exactly as NumPy does).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Layout shared with oracle/cport.py (ctypes).  Pointers are host arrays of
 * the build's precision except `mask` (uint8, nonzero = active). */
#define DOMAIN_FIELDS(REAL)                                                        \
    int64_t rows, cols;                                                            \
    double dx, dy, g, cfl, dry, max_dt, default_rain;                              \
    int32_t boundary[4]; /* left, right, bottom, top: 0 reflective, 1 open */      \
    int32_t n_rain, pad_;                                                          \
    const REAL *rain_times, *rain_rates, *bed, *manning;                          \
    const uint8_t *mask;                                                           \
    const REAL *mult;

typedef struct { DOMAIN_FIELDS(float) } dom_f32;
typedef struct { DOMAIN_FIELDS(double) } dom_f64;

void oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

#define REAL float
#define SUFFIX f32
#define SQRT sqrtf
#define FABS fabsf
#define HYPOT hypotf
#define POW powf
#include "swe_oracle_impl.h"
#undef REAL
#undef SUFFIX
#undef SQRT
#undef FABS
#undef HYPOT
#undef POW

#define REAL double
#define SUFFIX f64
#define SQRT sqrt
#define FABS fabs
#define HYPOT hypot
#define POW pow
#include "swe_oracle_impl.h"
