/*
 * mesh_oracle.c -- CPU restatement of the reference's random test mesh.
 *
 * TEST INFRASTRUCTURE ONLY.  The device generator of the library is checked
 * against this file; the product library never links or calls it.
 *
 * It restates Mesh<Float>::Mesh(solve_dim, dims) of
 * SidhantKrAgrawal/pentadiagonal-solver, include/util/mesh.hpp:85-124, the
 * random grid its benchmarks solve (benchmarks/cuda/my_bm.cu:7,
 * benchmarks/cpu/my_bm.cpp:8):
 *
 *   - an OpenMP parallel region; thread t seeds its own std::mt19937_64 with t
 *     and draws from std::uniform_real_distribution<Float> (mesh.hpp:103-104);
 *   - `omp for collapse(2)` over (outer i, inner j) systems with the default
 *     (static) schedule: the n_sys_out * n_sys_in systems, in collapsed order
 *     c = i * n_sys_in + j, are cut into nthreads contiguous chunks, the first
 *     (count % nthreads) of them one system longer (libgomp's static split);
 *   - per system, rows in order, per row the draws of ds (n > 1), dl (n > 0),
 *     d, du (n < N-1), dw (n < N-2) and x in that order (mesh.hpp:112-119):
 *     ds, dl, du, dw = -u, d = 6u, x = u; entries without a draw are 0.  N is
 *     unsigned there, so a system of one row (N - 2 wraps) draws dw too.
 *
 * The generator is MT19937-64 (Matsumoto and Nishimura; Nishimura, ACM TOMACS
 * 10(4), 2000) with the parameters the C++ standard fixes for mt19937_64
 * ([rand.predef]), its seeding recurrence x[i] = f (x[i-1] ^ (x[i-1] >> 62)) + i,
 * and the canonical conversion of libstdc++ (generate_canonical with one 64-bit
 * draw): u = (Float)v / 2^64, rounded to nearest, and the largest Float below
 * 1 when that rounds up to 1.  The output depends on nthreads, as the
 * reference's does.
 */
#include <stddef.h>
#include <stdint.h>

#define MT_N 312
#define MT_M 156

typedef struct {
  uint64_t x[MT_N];
  int i;
} penta_mt64;

static void mt64_seed(penta_mt64 *g, uint64_t seed) {
  g->x[0] = seed;
  for (int i = 1; i < MT_N; ++i)
    g->x[i] = 6364136223846793005ULL * (g->x[i - 1] ^ (g->x[i - 1] >> 62)) + (uint64_t)i;
  g->i = MT_N;
}

static uint64_t mt64_mix(uint64_t hi, uint64_t lo, uint64_t far) {
  uint64_t y = (hi & 0xFFFFFFFF80000000ULL) | (lo & 0x7FFFFFFFULL);
  return far ^ (y >> 1) ^ ((y & 1) ? 0xB5026F5AA96619E9ULL : 0);
}

static uint64_t mt64_next(penta_mt64 *g) {
  if (g->i >= MT_N) {
    int k = 0;
    for (; k < MT_N - MT_M; ++k) g->x[k] = mt64_mix(g->x[k], g->x[k + 1], g->x[k + MT_M]);
    for (; k < MT_N - 1; ++k) g->x[k] = mt64_mix(g->x[k], g->x[k + 1], g->x[k + MT_M - MT_N]);
    g->x[MT_N - 1] = mt64_mix(g->x[MT_N - 1], g->x[0], g->x[MT_M - 1]);
    g->i = 0;
  }
  uint64_t y = g->x[g->i++];
  y ^= (y >> 29) & 0x5555555555555555ULL;
  y ^= (y << 17) & 0x71D67FFFEDA60000ULL;
  y ^= (y << 37) & 0xFFF7EEE000000000ULL;
  y ^= y >> 43;
  return y;
}

/* The n-th (1-based) output of a generator seeded with `seed`. */
uint64_t penta_oracle_mt64_nth(uint64_t seed, long long n) {
  penta_mt64 g;
  mt64_seed(&g, seed);
  uint64_t v = 0;
  for (long long k = 0; k < n; ++k) v = mt64_next(&g);
  return v;
}

static double canon_d(uint64_t v) {
  double u = (double)v / 18446744073709551616.0;
  return u >= 1.0 ? 0x1.fffffffffffffp-1 : u;
}

static float canon_s(uint64_t v) {
  float u = (float)v / 18446744073709551616.0f;
  return u >= 1.0f ? 0x1.fffffep-1f : u;
}

#define DEFINE_MESH(SUF, REAL, CANON)                                              \
  int penta_oracle_mesh_random_##SUF(const int *dims, int ndims, int solvedim,     \
                                     int nthreads, REAL *ds, REAL *dl, REAL *d,    \
                                     REAL *du, REAL *dw, REAL *x) {                \
    if (ndims < 1 || solvedim < 0 || solvedim >= ndims || nthreads < 1) return -1; \
    long long inner = 1, outer = 1;                                                \
    for (int k = 0; k < solvedim; ++k) inner *= dims[k];                           \
    for (int k = solvedim + 1; k < ndims; ++k) outer *= dims[k];                   \
    const long long n = dims[solvedim];                                            \
    const long long count = inner * outer;                                         \
    const long long q = count / nthreads, rem = count % nthreads;                  \
    for (int t = 0; t < nthreads; ++t) {                                           \
      const long long lo = q * t + (t < rem ? t : rem);                            \
      const long long hi = lo + q + (t < rem ? 1 : 0);                             \
      penta_mt64 g;                                                                \
      mt64_seed(&g, (uint64_t)t);                                                  \
      for (long long c = lo; c < hi; ++c) {                                        \
        const long long i = c / inner, j = c % inner;                              \
        const long long start = i * inner * n + j;                                 \
        for (long long r = 0; r < n; ++r) {                                        \
          const long long idx = start + r * inner;                                 \
          ds[idx] = r > 1 ? -CANON(mt64_next(&g)) : (REAL)0;                       \
          dl[idx] = r > 0 ? -CANON(mt64_next(&g)) : (REAL)0;                       \
          d[idx] = (REAL)6 * CANON(mt64_next(&g));                                 \
          du[idx] = r < n - 1 ? -CANON(mt64_next(&g)) : (REAL)0;                   \
          dw[idx] = (uint64_t)r < (uint64_t)n - 2 ? -CANON(mt64_next(&g)) : (REAL)0; \
          x[idx] = CANON(mt64_next(&g));                                           \
        }                                                                          \
      }                                                                            \
    }                                                                              \
    return 0;                                                                      \
  }

DEFINE_MESH(d, double, canon_d)
DEFINE_MESH(s, float, canon_s)
