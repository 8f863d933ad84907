// thomas_kernels.cu -- the global-scratch Thomas kernel ("naive").
//
//  * thomas_global: one thread per system, the factorisation
//    (du2, dw2, x2) kept in the caller's scratch buffer, element-major
//    [row][system] so a warp touches consecutive addresses at every row.  The
//    any-shape fallback; 13 array passes (6 in, 3+3 scratch, 1 out).  It plays
//    the role of the reference's Algorithm 1
//    (src/cuda/singlenode/pentad_cuda.cu:1219-1314).
//    The on-chip kernels of tiled_kernels.cu serve every shape they fit;
//    this one serves the rest (lines too long for shared memory, grids of
//    2^31 elements or more) and the explicit "naive" selection.
#include "penta_device.cuh"
#include "penta_internal.hpp"

namespace penta {

// ---------------------------------------------------------------------------
// thomas_global
// ---------------------------------------------------------------------------
template <typename F>
__global__ void __launch_bounds__(128)
thomas_global_kernel(const F *__restrict__ ds, const F *__restrict__ dl,
                     const F *__restrict__ d, const F *__restrict__ du,
                     const F *__restrict__ dw, F *__restrict__ x, Lines L,
                     F *__restrict__ scratch, int *__restrict__ status_word) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= L.n_sys) return;
  const long long n = L.n, ns = L.n_sys, st = L.inner;
  const long long base = line_base(L, s);
  F *du2 = scratch + s;
  F *dw2 = du2 + n * ns;
  F *x2 = dw2 + n * ns;
  int status = 0;
  Carry<F> c;
  c.zero();
  for (long long i = 0; i < n; ++i) {
    const long long g = base + i * st;
    F a = ds[g], b = dl[g], e = du[g], w = dw[g];
    mask_row(i, n, a, b, e, w);
    F u, v, y;
    fwd_row(a, b, d[g], e, w, x[g], c, u, v, y, status);
    du2[i * ns] = u;
    dw2[i * ns] = v;
    x2[i * ns] = y;
  }
  F xa = F(0), xb = F(0);  // x[i+1], x[i+2]
  for (long long i = n - 1; i >= 0; --i) {
    const F xi = x2[i * ns] - du2[i * ns] * xa - dw2[i * ns] * xb;
    x[base + i * st] = xi;
    xb = xa;
    xa = xi;
  }
  if (status) atomicOr(status_word, status);
}

template <typename F>
cudaError_t launch_thomas_global(const SolveArgs<F> &a, cudaStream_t stream) {
  const long long ns = a.L.n_sys;
  const int block = 128;
  const long long grid = (ns + block - 1) / block;
  if (grid > 0x7fffffffLL) return cudaErrorInvalidValue;
  thomas_global_kernel<F><<<(unsigned)grid, block, 0, stream>>>(
      a.ds, a.dl, a.d, a.du, a.dw, a.x, a.L, static_cast<F *>(a.scratch),
      a.status);
  return cudaGetLastError();
}

template cudaError_t launch_thomas_global<double>(const SolveArgs<double> &,
                                                  cudaStream_t);
template cudaError_t launch_thomas_global<float>(const SolveArgs<float> &,
                                                 cudaStream_t);

}  // namespace penta
