// noalloc.cu -- a solve entry point that allocates nothing and needs no
// caller scratch buffer.
//
// Who it is for: callers that cannot call cudaMalloc around a solve.  Some
// applications hand all device memory to their own pool at start-up and
// forbid raw cudaMalloc afterwards; in others cudaMalloc/cudaFree are not an
// option in the solve loop because they can synchronise the whole device; and
// code ported from the reference's CPU interface passes no scratch buffer at
// all (t_buffer = NULL).  The regular entry points need a caller-allocated
// t_buffer for the global-scratch kernel; this one runs that same kernel
// (thomas_global, thomas_kernels.cu) with its scratch placed in a fixed
// device array that is part of the library image.
//
// The array: PENTADSOLVER_NOALLOC_MAX_BYTES (16 MiB) of file-scope __device__
// memory.  Every GPU that loads the library holds it until the process exits.
// A solve needs 3 * n_total * 8 bytes of it (n_total = product of t_dims), so
// grids up to 699,050 points (e.g. 88^3) fit; larger ones are rejected with
// PENTAD_STATUS_INVALID_VALUE before anything runs on the device.
//
// Sharing: all calls on a device use the same array, and it keeps whatever
// the last call left there.  The kernel writes every scratch element before
// reading it, so nothing has to be cleared between calls.  Calls that can
// overlap on the GPU (issued on different streams without ordering, or from
// several threads) race on the array and corrupt each other's results: issue
// them on one stream, or order them.
//
// Set-up: the device address of the array is taken with cudaGetSymbolAddress
// the first time the entry point runs on each device, with that device
// current.  (In host code the array's name only stands in for the device
// symbol; it is not a device address.)  That first call should therefore come
// before any stream capture on the device.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "pentad_common.hpp"
#include "pentadsolver_ext.h"
#include "penta_internal.hpp"

namespace {

constexpr size_t kNoallocBytes = PENTADSOLVER_NOALLOC_MAX_BYTES;
static __device__ __align__(256) double g_noalloc_scratch[kNoallocBytes / sizeof(double)];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double *g_scratch_addr[kMaxDevices] = {};

// Device address of the array on the current device (taken once per device).
cudaError_t scratch_address(double **out) {
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return err;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_mu);
  if (g_scratch_addr[dev] == nullptr) {
    void *p = nullptr;
    err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (err != cudaSuccess) return err;
    g_scratch_addr[dev] = static_cast<double *>(p);
  }
  *out = g_scratch_addr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" PENTAD_API pentadStatus_t pentadsolver_D_gpsv_batch_noalloc(
    pentadsolver_handle_t handle, const double *ds, const double *dl,
    const double *d, const double *du, const double *dw, double *x,
    const int *t_dims, int t_ndim, int t_solvedim, void *stream) {
  // Shape checks first (the same rules as every other entry point):
  // nothing touches the device for a rejected call.
  penta::Lines L{};
  const char *why = "";
  pentadStatus_t st = penta::check_shape(t_dims, t_ndim, t_solvedim, L, &why);
  if (st != PENTAD_STATUS_SUCCESS) return st;
  if (!ds || !dl || !d || !du || !dw || !x) return PENTAD_STATUS_INVALID_VALUE;
  const size_t need = penta::thomas_global_scratch<double>(L);
  if (need > kNoallocBytes) {
    std::fprintf(stderr,
                 "[penta] pentadsolver_D_gpsv_batch_noalloc: this grid needs %zu "
                 "bytes of scratch; the built-in array holds %zu "
                 "(at most %zu grid points) -- use pentadsolver_D_gpsv_batch_ex "
                 "with a caller buffer\n",
                 need, kNoallocBytes, kNoallocBytes / (3 * sizeof(double)));
    return PENTAD_STATUS_INVALID_VALUE;
  }

  // the handle (NULL: the current device's default context) gives the status
  // word, as for pentadsolver_D_gpsv_batch_ex
  int *status_word = nullptr;
  st = penta::bind_handle(handle, &status_word, &why);
  if (st != PENTAD_STATUS_SUCCESS) return st;
  double *scratch = nullptr;
  if (scratch_address(&scratch) != cudaSuccess) {
    cudaGetLastError();
    return PENTAD_STATUS_NOT_INITIALIZED;
  }

  penta::SolveArgs<double> a{ds, dl, d, du, dw, x, L, scratch, kNoallocBytes,
                             status_word};
  if (penta::launch_thomas_global<double>(a, static_cast<cudaStream_t>(stream)) !=
      cudaSuccess) {
    cudaGetLastError();
    return PENTAD_STATUS_EXECUTION_FAILED;
  }
  return PENTAD_STATUS_SUCCESS;
}
