// refine_kernels.cu -- the FP64 steps of mixed-precision iterative refinement.
//
// A pentadiagonal system with FP64 coefficients A and right-hand side b is
// solved with FP32 sweeps and refined:
//     r0 = fl32(b);  x = solve32(A32, r0)            (FP32 sweep)
//     repeat: r = fl32(b - A x)                       (FP64 residual)
//             d = solve32(A32, r)                     (FP32 sweep)
//             x = x + d                               (FP64 correction)
// The residual and the correction are the only FP64 arithmetic; the sweeps
// are the library's FP32 kernels.  With one refinement step (or none) the
// first iterate stays in FP32 (x0 in r) and b stays in the caller's x until
// the correction writes the result: q = fl32(b - A x0) goes to a second FP32
// array, the second sweep solves it in place, and x = x0 + d -- the same
// values as the general form without its FP64 copies of x0 and b (140
// instead of 168 bytes per point with cached FP32 coefficients).  Each kernel here walks the points of one
// or many grids (a grid table; one CTA handles a chunk of one grid), so a
// batch of uneven grids is one launch per step.
//
// The residual uses the same masking as the solvers: the couplings that leave
// a line (ds at rows 0,1; dl at row 0; du at row n-1; dw at rows n-2,n-1) are
// ignored whatever they hold.
//
// The correction step also records, per grid, max|d| and max|x| (non-negative
// doubles compared as integers with atomicMax), whose ratio estimates the
// forward error of the iterate before the step.
#include <cstdint>

#include "penta_internal.hpp"

namespace penta {
namespace {

constexpr int kChunk = 4096;   // points per CTA
constexpr int kThreads = 256;

// The grid CTA `block` works on: `one` when there is no table.
__device__ __forceinline__ const RefineGrid &grid_of(const RefineGrid &one,
                                                     const RefineGrid *table, int count,
                                                     int block, long long &first) {
  if (table == nullptr) {
    first = (long long)block * kChunk;
    return one;
  }
  int lo = 0, hi = count - 1;  // last grid whose chunk_base <= block
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (table[mid].chunk_base <= block) lo = mid; else hi = mid - 1;
  }
  first = (long long)(block - table[lo].chunk_base) * kChunk;
  return table[lo];
}

// Whether points [first, end) of an array can be walked in pairs: an even
// start and end, and an array aligned for the pair's width.
__device__ __forceinline__ bool pairs_ok(long long first, long long end, const void *a,
                                         int width) {
  return ((first | end) & 1) == 0 && (reinterpret_cast<uintptr_t>(a) & (width - 1)) == 0;
}

__device__ __forceinline__ void cast_pair(const double *src, float *dst, long long i) {
  const double2 v = *reinterpret_cast<const double2 *>(src + i);
  *reinterpret_cast<float2 *>(dst + i) = make_float2((float)v.x, (float)v.y);
}

__device__ __forceinline__ bool cast_pairs_ok(const RefineGrid &g, long long first,
                                              long long end) {
  return pairs_ok(first, end, g.ds, 16) && pairs_ok(first, end, g.dl, 16) &&
         pairs_ok(first, end, g.d, 16) && pairs_ok(first, end, g.du, 16) &&
         pairs_ok(first, end, g.dw, 16) && pairs_ok(first, end, g.s_ds, 8) &&
         pairs_ok(first, end, g.s_dl, 8) && pairs_ok(first, end, g.s_d, 8) &&
         pairs_ok(first, end, g.s_du, 8) && pairs_ok(first, end, g.s_dw, 8);
}

__global__ void __launch_bounds__(kThreads)
rf_prepare_kernel(const __grid_constant__ RefineGrid one, const RefineGrid *__restrict__ table, int count, int cast_coefficients, int save_b) {
  long long first;
  const RefineGrid &g = grid_of(one, table, count, blockIdx.x, first);
  const long long end = min(first + kChunk, g.n_points);
  if (!save_b && pairs_ok(first, end, g.x, 16) && pairs_ok(first, end, g.r, 8) &&
      (!cast_coefficients || cast_pairs_ok(g, first, end))) {  // the one-step form: pairs
    for (long long i = first + 2 * threadIdx.x; i < end; i += 2 * kThreads) {
      if (cast_coefficients) {
        cast_pair(g.ds, g.s_ds, i);
        cast_pair(g.dl, g.s_dl, i);
        cast_pair(g.d, g.s_d, i);
        cast_pair(g.du, g.s_du, i);
        cast_pair(g.dw, g.s_dw, i);
      }
      cast_pair(g.x, g.r, i);
    }
    return;
  }
  for (long long i = first + threadIdx.x; i < end; i += kThreads) {
    if (cast_coefficients) {
      g.s_ds[i] = (float)g.ds[i];
      g.s_dl[i] = (float)g.dl[i];
      g.s_d[i] = (float)g.d[i];
      g.s_du[i] = (float)g.du[i];
      g.s_dw[i] = (float)g.dw[i];
    }
    const double b = g.x[i];
    if (save_b) g.b[i] = b;
    g.r[i] = (float)b;
  }
}

// x = fl64(r) after the first FP32 sweep.
__global__ void __launch_bounds__(kThreads)
rf_lift_kernel(const __grid_constant__ RefineGrid one, const RefineGrid *__restrict__ table, int count) {
  long long first;
  const RefineGrid &g = grid_of(one, table, count, blockIdx.x, first);
  const long long end = min(first + kChunk, g.n_points);
  for (long long i = first + threadIdx.x; i < end; i += kThreads) g.x[i] = (double)g.r[i];
}

// r = fl32(b - A x), FP64 arithmetic.
__global__ void __launch_bounds__(kThreads)
rf_residual_kernel(const __grid_constant__ RefineGrid one, const RefineGrid *__restrict__ table, int count) {
  long long first;
  const RefineGrid &g = grid_of(one, table, count, blockIdx.x, first);
  const long long end = min(first + kChunk, g.n_points);
  const long long s = g.inner;
  const int n = g.n;
  for (long long i = first + threadIdx.x; i < end; i += kThreads) {
    const int k = (int)((i / s) % n);  // row within its line
    double ax = g.d[i] * g.x[i];
    if (k >= 2) ax = fma(g.ds[i], g.x[i - 2 * s], ax);
    if (k >= 1) ax = fma(g.dl[i], g.x[i - s], ax);
    if (k <= n - 2) ax = fma(g.du[i], g.x[i + s], ax);
    if (k <= n - 3) ax = fma(g.dw[i], g.x[i + 2 * s], ax);
    g.r[i] = (float)(g.b[i] - ax);
  }
}

// q = fl32(b - A x0) with b still in the caller's x and x0 the FP32 iterate in
// r, FP64 arithmetic: the same values as Lift followed by Residual.
__global__ void __launch_bounds__(kThreads)
rf_residual1_kernel(const __grid_constant__ RefineGrid one, const RefineGrid *__restrict__ table, int count) {
  long long first;
  const RefineGrid &g = grid_of(one, table, count, blockIdx.x, first);
  const long long end = min(first + kChunk, g.n_points);
  const long long s = g.inner;
  const int n = g.n;
  for (long long i = first + threadIdx.x; i < end; i += kThreads) {
    const int k = (int)((i / s) % n);  // row within its line
    double ax = g.d[i] * (double)g.r[i];
    if (k >= 2) ax = fma(g.ds[i], (double)g.r[i - 2 * s], ax);
    if (k >= 1) ax = fma(g.dl[i], (double)g.r[i - s], ax);
    if (k <= n - 2) ax = fma(g.du[i], (double)g.r[i + s], ax);
    if (k <= n - 3) ax = fma(g.dw[i], (double)g.r[i + 2 * s], ax);
    g.q[i] = (float)(g.x[i] - ax);
  }
}

__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v) {
  // non-negative doubles order like their bit patterns
  atomicMax(reinterpret_cast<unsigned long long *>(addr),
            (unsigned long long)__double_as_longlong(v));
}

// est = max(est, (md, mx)) for the whole CTA: one warp-level and one
// CTA-level reduction, then at most two atomics, skipped when the stored
// maxima are already at least as large (a stale read of them only costs an
// atomic: the maxima never decrease).  Every thread of the CTA calls it.
__device__ __forceinline__ void cta_max_into(double *est, double md, double mx) {
  __shared__ double part[2][kThreads / 32];
  for (int o = 16; o > 0; o /= 2) {
    md = fmax(md, __shfl_xor_sync(0xffffffffu, md, o));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  const int w = threadIdx.x / 32;
  if ((threadIdx.x & 31) == 0) {
    part[0][w] = md;
    part[1][w] = mx;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    double v = part[threadIdx.x][0];
    for (int k = 1; k < kThreads / 32; ++k) v = fmax(v, part[threadIdx.x][k]);
    double *const slot = est + threadIdx.x;
    if (v > *reinterpret_cast<volatile double *>(slot)) atomic_max_nonneg(slot, v);
  }
}

// x += fl64(d); est = (max|d|, max|x|) over the grid.
__global__ void __launch_bounds__(kThreads)
rf_correct_kernel(const __grid_constant__ RefineGrid one, const RefineGrid *__restrict__ table, int count) {
  long long first;
  const RefineGrid &g = grid_of(one, table, count, blockIdx.x, first);
  const long long end = min(first + kChunk, g.n_points);
  double md = 0.0, mx = 0.0;
  for (long long i = first + threadIdx.x; i < end; i += kThreads) {
    const double dd = (double)g.r[i];
    const double xn = g.x[i] + dd;
    g.x[i] = xn;
    md = fmax(md, fabs(dd));
    mx = fmax(mx, fabs(xn));
  }
  cta_max_into(g.est, md, mx);
}

// x = fl64(x0) + fl64(d) with x0 in r and d in q; est as rf_correct_kernel.
__global__ void __launch_bounds__(kThreads)
rf_correct1_kernel(const __grid_constant__ RefineGrid one, const RefineGrid *__restrict__ table, int count) {
  long long first;
  const RefineGrid &g = grid_of(one, table, count, blockIdx.x, first);
  const long long end = min(first + kChunk, g.n_points);
  double md = 0.0, mx = 0.0;
  if (pairs_ok(first, end, g.x, 16) && pairs_ok(first, end, g.r, 8) &&
      pairs_ok(first, end, g.q, 8)) {
    for (long long i = first + 2 * threadIdx.x; i < end; i += 2 * kThreads) {
      const float2 d2 = *reinterpret_cast<const float2 *>(g.q + i);
      const float2 x2 = *reinterpret_cast<const float2 *>(g.r + i);
      const double d0 = (double)d2.x, d1 = (double)d2.y;
      const double2 xn = make_double2((double)x2.x + d0, (double)x2.y + d1);
      *reinterpret_cast<double2 *>(g.x + i) = xn;
      md = fmax(md, fmax(fabs(d0), fabs(d1)));
      mx = fmax(mx, fmax(fabs(xn.x), fabs(xn.y)));
    }
  } else {
    for (long long i = first + threadIdx.x; i < end; i += kThreads) {
      const double dd = (double)g.q[i];
      const double xn = (double)g.r[i] + dd;
      g.x[i] = xn;
      md = fmax(md, fabs(dd));
      mx = fmax(mx, fabs(xn));
    }
  }
  cta_max_into(g.est, md, mx);
}

// Clear the estimate before a correction step.
__global__ void rf_clear_kernel(const __grid_constant__ RefineGrid one,
                                const RefineGrid *__restrict__ table, int count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) {
    double *est = table ? table[i].est : one.est;
    est[0] = 0.0;
    est[1] = 0.0;
  }
}

}  // namespace

int refine_chunks(long long n_points) { return (int)((n_points + kChunk - 1) / kChunk); }

cudaError_t launch_refine_step(RefineStep step, const RefineGrid &one, const RefineGrid *table,
                               int count, int total_chunks, cudaStream_t stream) {
  if (total_chunks <= 0) return cudaSuccess;
  switch (step) {
    case RefineStep::PrepareCast:
      rf_prepare_kernel<<<total_chunks, kThreads, 0, stream>>>(one, table, count, 1, 1);
      break;
    case RefineStep::Prepare:
      rf_prepare_kernel<<<total_chunks, kThreads, 0, stream>>>(one, table, count, 0, 1);
      break;
    case RefineStep::FirstCast:
      rf_prepare_kernel<<<total_chunks, kThreads, 0, stream>>>(one, table, count, 1, 0);
      break;
    case RefineStep::First:
      rf_prepare_kernel<<<total_chunks, kThreads, 0, stream>>>(one, table, count, 0, 0);
      break;
    case RefineStep::Residual1:
      rf_residual1_kernel<<<total_chunks, kThreads, 0, stream>>>(one, table, count);
      break;
    case RefineStep::Correct1:
      rf_clear_kernel<<<(count + 127) / 128, 128, 0, stream>>>(one, table, count);
      rf_correct1_kernel<<<total_chunks, kThreads, 0, stream>>>(one, table, count);
      break;
    case RefineStep::Lift:  // no correction yet: the estimate reads zero
      rf_clear_kernel<<<(count + 127) / 128, 128, 0, stream>>>(one, table, count);
      rf_lift_kernel<<<total_chunks, kThreads, 0, stream>>>(one, table, count);
      break;
    case RefineStep::Residual:
      rf_residual_kernel<<<total_chunks, kThreads, 0, stream>>>(one, table, count);
      break;
    case RefineStep::Correct:
      rf_clear_kernel<<<(count + 127) / 128, 128, 0, stream>>>(one, table, count);
      rf_correct_kernel<<<total_chunks, kThreads, 0, stream>>>(one, table, count);
      break;
  }
  return cudaGetLastError();
}

}  // namespace penta
