// penta_device.cuh -- device-side building blocks shared by every kernel.
//
// Row i of a system is  ds[i] x[i-2] + dl[i] x[i-1] + d[i] x[i] + du[i] x[i+1]
// + dw[i] x[i+2] = b[i]  (reference include/pentadsolver.hpp:88-131).  Entries
// that couple to rows outside the system (ds at rows 0,1; dl at row 0; du at
// row n-1; dw at rows n-2,n-1) are never read by the reference
// (src/cpu/singlenode/pentad_orig_cpu.cpp:17-56), so every kernel here masks
// them to zero on load: any value there, NaN included, leaves the result
// unchanged.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "penta_lines.h"

namespace penta {

template <typename F> __device__ __forceinline__ F rcp(F v);
template <> __device__ __forceinline__ double rcp<double>(double v) {
  return __drcp_rn(v);
}
template <> __device__ __forceinline__ float rcp<float>(float v) {
  return __frcp_rn(v);
}

template <typename F> __device__ __forceinline__ bool bad_pivot(F dd) {
  return !(dd != F(0)) || !isfinite(dd);
}

template <typename F> struct Carry {
  F u1, u2, w1, w2, y1, y2;
  __device__ __forceinline__ void zero() {
    u1 = u2 = w1 = w2 = y1 = y2 = F(0);
  }
};

// Reciprocal by Newton-Raphson refinement of the hardware approximation:
// r <- r + r (1 - d r) doubles the number of correct bits per step, so two
// steps take the ~20-bit rcp.approx.ftz.f64 seed past double precision (the
// result is within an ulp or two of 1/d, not necessarily correctly rounded).
// One step suffices from the single-precision seed.  A zero, infinite or NaN
// pivot gives a non-finite result, which the kernels report.
__device__ __forceinline__ double rcp_nr(double d) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
  double e = fma(-d, r, 1.0);
  r = fma(r, e, r);
  e = fma(-d, r, 1.0);
  return fma(r, e, r);
}
__device__ __forceinline__ float rcp_nr(float d) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(d));
  const float e = fmaf(-d, r, 1.0f);
  return fmaf(r, e, r);
}

// Forward elimination of one row whose couplings are already masked; carries
// as for fwd_row below.  `bad` collects non-finite reciprocals (zero pivots).
template <typename F>
__device__ __forceinline__ void fwd_row_fast(F ds, F dl, F d, F du, F dw, F b,
                                             Carry<F> &c, F &du2, F &dw2,
                                             F &x2, bool &bad) {
  const F ddl = dl - ds * c.u2;
  const F dd = d - ds * c.w2 - ddl * c.u1;
  const F inv = rcp_nr(dd);
  bad |= !isfinite(inv);
  du2 = (du - ddl * c.w1) * inv;
  dw2 = dw * inv;
  x2 = (b - ds * c.y2 - ddl * c.y1) * inv;
  c.u2 = c.u1; c.u1 = du2;
  c.w2 = c.w1; c.w1 = dw2;
  c.y2 = c.y1; c.y1 = x2;
}

// One row of forward elimination (couplings already masked); as fwd_row_fast
// without the per-row pivot check -- a zero pivot turns the carries into NaN,
// which the kernel checks once per tile.
template <typename F>
__device__ __forceinline__ void fwd_row_lean(F ds, F dl, F d, F du, F dw, F b,
                                             Carry<F> &c, F &du2, F &dw2, F &x2) {
  const F ddl = dl - ds * c.u2;
  const F dd = d - ds * c.w2 - ddl * c.u1;
  const F inv = rcp_nr(dd);
  du2 = (du - ddl * c.w1) * inv;
  dw2 = dw * inv;
  x2 = (b - ds * c.y2 - ddl * c.y1) * inv;
  c.u2 = c.u1; c.u1 = du2;
  c.w2 = c.w1; c.w1 = dw2;
  c.y2 = c.y1; c.y1 = x2;
}

// Zero the out-of-range couplings of row i of an n-row system.
template <typename F>
__device__ __forceinline__ void mask_row(long long i, long long n, F &ds,
                                         F &dl, F &du, F &dw) {
  ds = (i < 2) ? F(0) : ds;
  dl = (i < 1) ? F(0) : dl;
  du = (i > n - 2) ? F(0) : du;
  dw = (i > n - 3) ? F(0) : dw;
}

// One row of forward elimination with the carries of the two previous rows
// (zero before row 0).  This is the recurrence of pentad_orig_cpu.cpp:30-40
// with the division replaced by one reciprocal; with zero carries and masked
// couplings it also reproduces the reference's special first two rows.
//   in : ds dl d du dw b  of row i,  carries (u1,u2) = du2[i-1], du2[i-2],
//        (w1,w2) = dw2[i-1], dw2[i-2], (y1,y2) = x2[i-1], x2[i-2]
//   out: du2[i], dw2[i], x2[i] (also shifted into the carries)
template <typename F>
__device__ __forceinline__ void fwd_row(F ds, F dl, F d, F du, F dw, F b,
                                        Carry<F> &c, F &du2, F &dw2, F &x2,
                                        int &status) {
  const F ddl = dl - ds * c.u2;
  const F dd = d - ds * c.w2 - ddl * c.u1;
  if (bad_pivot(dd)) status |= STATUS_ZERO_PIVOT_BIT;
  const F inv = rcp(dd);
  du2 = (du - ddl * c.w1) * inv;
  dw2 = dw * inv;
  x2 = (b - ds * c.y2 - ddl * c.y1) * inv;
  c.u2 = c.u1; c.u1 = du2;
  c.w2 = c.w1; c.w1 = dw2;
  c.y2 = c.y1; c.y1 = x2;
}

// Solve the 4x4 interface of a line split into a top part (rows < m, in upper
// form x_i + du2_i x_{i+1} + dw2_i x_{i+2} = x2_i) and a bottom part (rows >= m,
// eliminated upwards into lower form x_i + e_i x_{i-1} + c_i x_{i-2} = y_i).
//   T1 (row m-2): u0 + a1 u1 + b1 u2      = r0
//   T2 (row m-1):      u1 + a2 u2 + b2 u3 = r1
//   B1 (row m)  : c1 u0 + e1 u1 + u2      = r2
//   B2 (row m+1):      c2 u1 + e2 u2 + u3 = r3
// with (u0,u1,u2,u3) = (x_{m-2}, x_{m-1}, x_m, x_{m+1}).  Eliminating u0 and
// u3 leaves a 2x2 system in (u1,u2), solved by Cramer's rule.
template <typename F>
__device__ __forceinline__ void solve_interface(F a1, F b1, F r0, F a2, F b2,
                                                F r1, F e1, F c1, F r2, F e2,
                                                F c2, F r3, F &u0, F &u1,
                                                F &u2, F &u3) {
  const F p11 = F(1) - b2 * c2, p12 = a2 - b2 * e2, q1 = r1 - b2 * r3;
  const F p21 = e1 - c1 * a1, p22 = F(1) - c1 * b1, q2 = r2 - c1 * r0;
  const F inv_det = rcp(p11 * p22 - p12 * p21);
  u1 = (q1 * p22 - p12 * q2) * inv_det;
  u2 = (p11 * q2 - p21 * q1) * inv_det;
  u0 = r0 - a1 * u1 - b1 * u2;
  u3 = r3 - c2 * u1 - e2 * u2;
}

// ---------------------------------------------------------------------------
// Asynchronous global -> shared copies (sm_80+ cp.async; no TMA descriptors
// needed, so any n, stride or alignment works).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
template <int BYTES>
__device__ __forceinline__ void cp_async_ca(void *dst_smem, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(
                   smem_u32(dst_smem)),
               "l"(src), "n"(BYTES)
               : "memory");
}
template <int BYTES>
__device__ __forceinline__ void cp_async_cg(void *dst_smem, const void *src) {
  static_assert(BYTES == 16, "cp.async.cg copies 16 bytes");
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(
                   smem_u32(dst_smem)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

}  // namespace penta
