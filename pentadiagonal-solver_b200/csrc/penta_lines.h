// penta_lines.h -- the line-set descriptor shared by host and device code.
//
// For a grid dims[0..ndim) (dims[0] contiguous) solved along `solvedim`:
//   n     = dims[solvedim]                       rows per system
//   inner = prod(dims[0..solvedim))              element stride between rows
//   n_sys = inner * prod(dims[solvedim+1..ndim)) number of systems
// System s starts at base(s) = (s / inner) * inner * n + (s % inner) and its
// row i sits at base(s) + i * inner.  solvedim 0 gives inner = 1 (contiguous
// lines, the reference's pentadsolver_gpsv_batch_x); the last dimension gives
// one run of `inner` adjacent systems (the reference's "outermost" z solve);
// any other dimension gives runs of `inner` adjacent systems (the reference's
// "middle" y solve) -- src/cuda/singlenode/pentad_cuda.cu:1420-1445.
#pragma once

#if defined(__CUDACC__)
#define PENTA_HD __host__ __device__ __forceinline__
#else
#define PENTA_HD inline
#endif

namespace penta {

// Status bits kernels OR into the per-device status word.
enum : int {
  STATUS_ZERO_PIVOT_BIT = 1,  // a pivot was exactly zero or not finite
  STATUS_TIMEOUT_BIT = 2,     // a bounded wait inside a kernel ran out
};

struct Lines {
  long long n;      // rows per system
  long long inner;  // row stride in elements
  long long n_sys;  // systems
};

PENTA_HD long long line_base(const Lines &L, long long s) {
  return (s / L.inner) * L.inner * L.n + (s % L.inner);
}

}  // namespace penta
