/*
 * penta_oracle.c -- CPU restatement of the reference pentadiagonal solver.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle that the CUDA library is
 * checked against.  Only tests, the smoke check and the CPU-baseline leg of
 * bench.py load it; the product library never links or calls it.
 *
 * It restates the scalar solver of SidhantKrAgrawal/pentadiagonal-solver,
 * src/cpu/singlenode/pentad_orig_cpu.cpp, in plain C:
 *
 *   penta_oracle_line_*     pentadsolver_x           (:9-56) and
 *                           pentadsolver_strided     (:73-122): one system,
 *                           elimination with normalised rows, then backward
 *                           substitution.  One routine covers both because the
 *                           x solve is the strided solve with stride 1.
 *   penta_oracle_batch_*    pentadsolver_gpsv_batch  (:197-216) routing to
 *                           pentadsolver_gpsv_batch_x / _outermost / _middle
 *                           (:158-195) and the batch loops (:58-156).
 *
 * Arithmetic order is the reference's, operation for operation, so that with
 * -ffp-contract=off the results are bit-identical to the reference compiled
 * with g++ -std=c++17 (which does not contract either).  Unlike the reference
 * there is no N_MAX=1024 limit: the per-system scratch is allocated.
 *
 * Row i of a system reads ds[i] x[i-2] + dl[i] x[i-1] + d[i] x[i]
 *                      + du[i] x[i+1] + dw[i] x[i+2] = b[i].
 * Row 0 never reads ds[0], dl[0]; row 1 never reads ds[1]; du[n-1], dw[n-2]
 * and dw[n-1] only feed scratch values that the backward sweep never reads.
 */
#include <stddef.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define DEFINE_ORACLE(SUF, REAL)                                               \
  /* pentad_orig_cpu.cpp:73-122 (stride 1 gives :9-56) */                      \
  void penta_oracle_line_##SUF(const REAL *ds, const REAL *dl, const REAL *d, \
                               const REAL *du, const REAL *dw, REAL *x,       \
                               size_t n, size_t stride, REAL *scratch) {      \
    REAL *du2 = scratch, *dw2 = scratch + n, *x2 = scratch + 2 * n;           \
    du2[0] = du[0] / d[0];                                                     \
    dw2[0] = dw[0] / d[0];                                                     \
    x2[0] = x[0] / d[0];                                                       \
    REAL ddl = dl[1 * stride];                                                 \
    REAL dd = d[1 * stride] - ddl * du2[0];                                    \
    du2[1] = (du[1 * stride] - ddl * dw2[0]) / dd;                             \
    dw2[1] = dw[1 * stride] / dd;                                              \
    x2[1] = (x[1 * stride] - ddl * x2[0]) / dd;                                \
    for (size_t i = 2; i < n; ++i) {                                           \
      REAL dds = ds[i * stride];                                               \
      ddl = dl[i * stride] - dds * du2[i - 2];                                 \
      dd = d[i * stride] - dds * dw2[i - 2] - ddl * du2[i - 1];                \
      du2[i] = (du[i * stride] - ddl * dw2[i - 1]) / dd;                       \
      dw2[i] = dw[i * stride] / dd;                                            \
      x2[i] = (x[i * stride] - dds * x2[i - 2] - ddl * x2[i - 1]) / dd;        \
    }                                                                          \
    x[(n - 1) * stride] = x2[n - 1];                                           \
    REAL ddu = du2[n - 2];                                                     \
    x[(n - 2) * stride] = x2[n - 2] - ddu * x[(n - 1) * stride];               \
    for (long i = (long)n - 3; i >= 0; --i) {                                  \
      REAL ddw = dw2[i];                                                       \
      ddu = du2[i];                                                            \
      x[i * stride] = x2[i] - ddw * x[(i + 2) * stride] -                      \
                      ddu * x[(i + 1) * stride];                               \
    }                                                                          \
  }                                                                            \
                                                                               \
  /* pentad_orig_cpu.cpp:158-216: returns 0, or -1 for an invalid shape.      \
   * Lines are indexed (outer o, inner j): start o*inner*n + j, stride inner. \
   * solvedim 0 has inner = 1; the outermost dimension has outer = 1. */      \
  int penta_oracle_batch_##SUF(const REAL *ds, const REAL *dl, const REAL *d, \
                               const REAL *du, const REAL *dw, REAL *x,       \
                               const int *dims, int ndim, int solvedim) {     \
    if (ndim < 1 || solvedim < 0 || solvedim >= ndim) return -1;              \
    size_t inner = 1, outer = 1;                                               \
    for (int k = 0; k < solvedim; ++k) inner *= (size_t)dims[k];              \
    for (int k = solvedim + 1; k < ndim; ++k) outer *= (size_t)dims[k];       \
    size_t n = (size_t)dims[solvedim];                                         \
    if (n < 2) return -1;                                                      \
    long total = (long)(inner * outer);                                        \
    int failed = 0;                                                            \
    _Pragma("omp parallel")                                                    \
    {                                                                          \
      REAL *scratch = (REAL *)malloc(3 * n * sizeof(REAL));                    \
      if (!scratch) {                                                          \
        _Pragma("omp atomic write") failed = 1;                                \
      } else {                                                                 \
        _Pragma("omp for schedule(static)")                                    \
        for (long s = 0; s < total; ++s) {                                     \
          size_t o = (size_t)s / inner, j = (size_t)s % inner;                 \
          size_t start = o * inner * n + j;                                    \
          penta_oracle_line_##SUF(ds + start, dl + start, d + start,          \
                                  du + start, dw + start, x + start, n,       \
                                  inner, scratch);                             \
        }                                                                      \
        free(scratch);                                                         \
      }                                                                        \
    }                                                                          \
    return failed ? -2 : 0;                                                    \
  }                                                                            \
                                                                               \
  /* Backward residual max_i |(A x - b)_i| over every line along solvedim.    \
   * Out-of-range couplings are skipped, as in the solve. */                  \
  double penta_oracle_residual_##SUF(                                          \
      const REAL *ds, const REAL *dl, const REAL *d, const REAL *du,          \
      const REAL *dw, const REAL *x, const REAL *b, const int *dims,          \
      int ndim, int solvedim) {                                                \
    size_t inner = 1, outer = 1;                                               \
    for (int k = 0; k < solvedim; ++k) inner *= (size_t)dims[k];              \
    for (int k = solvedim + 1; k < ndim; ++k) outer *= (size_t)dims[k];       \
    long n = dims[solvedim];                                                   \
    long total = (long)(inner * outer);                                        \
    double worst = 0.0;                                                        \
    _Pragma("omp parallel for reduction(max : worst) schedule(static)")        \
    for (long s = 0; s < total; ++s) {                                         \
      size_t o = (size_t)s / inner, j = (size_t)s % inner;                     \
      size_t st = o * inner * (size_t)n + j;                                   \
      for (long i = 0; i < n; ++i) {                                           \
        size_t g = st + (size_t)i * inner;                                     \
        double r = (double)d[g] * (double)x[g] - (double)b[g];                 \
        if (i >= 2) r += (double)ds[g] * (double)x[g - 2 * inner];             \
        if (i >= 1) r += (double)dl[g] * (double)x[g - inner];                 \
        if (i + 1 < n) r += (double)du[g] * (double)x[g + inner];              \
        if (i + 2 < n) r += (double)dw[g] * (double)x[g + 2 * inner];          \
        r = fabs(r);                                                           \
        if (r > worst) worst = r;                                              \
      }                                                                        \
    }                                                                          \
    return worst;                                                              \
  }

DEFINE_ORACLE(d, double)
DEFINE_ORACLE(s, float)

/* Forward error max_i |x_i - ref_i| / max_i |ref_i|, the definition used by
 * the reference's apps/fp32_accuracy_cuda.cu. */
double penta_oracle_fwd_err_d(const double *x, const double *ref, size_t n) {
  double num = 0.0, den = 0.0;
  for (size_t i = 0; i < n; ++i) {
    double e = fabs(x[i] - ref[i]);
    double m = fabs(ref[i]);
    if (e > num || e != e) num = e;
    if (m > den) den = m;
  }
  return den > 0.0 ? num / den : num;
}

int penta_oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
