// penta_adi.cpp -- ADI iterations captured once into a CUDA graph (C ABI).
//
// An ADI time step solves one grid in place along x, then y, then z, with
// coefficient arrays that do not change between steps: the loop of the
// reference's application (apps/adi_cuda.cu:167-176), one
// pentadsolver_gpsv_batch call per direction.  pentadsolver_adi_create records
// `iterations` such steps (3 x iterations solves through
// pentadsolver_{D,S}_gpsv_batch_ex with the caller's handle, so its algorithm
// choices hold -- with shared factorisation the factor tables stay cached in
// the buffer for every step) into one CUDA graph; pentadsolver_adi_replay
// launches them all with one call and none of the host work between launches.
//
// What a solve sets up on the host the first time (kernel attributes,
// occupancy queries, tensor-map encoding, status-word addresses) happens in an
// eager warm-up pass before capture.  The warm-up solves a copy of x kept in
// the tail of the caller's buffer -- the reference-sized buffer of the x
// direction holds 9 values per point, and no kernel uses more than 3 -- so x
// is untouched until the first replay and nothing is allocated.
#include <cuda_runtime_api.h>

#include <cstdint>

#include "pentad_common.hpp"
#include "pentadsolver_ext.h"

struct pentadsolver_adi_s {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int launches = 0;
};

namespace {

pentadStatus_t solve_ex(int elem, pentadsolver_handle_t h, const void *const *a, void *x,
                        const int *dims, int ndim, int solvedim, void *buf, size_t bytes,
                        cudaStream_t s) {
  if (elem == 8)
    return pentadsolver_D_gpsv_batch_ex(h, static_cast<const double *>(a[0]),
                                        static_cast<const double *>(a[1]),
                                        static_cast<const double *>(a[2]),
                                        static_cast<const double *>(a[3]),
                                        static_cast<const double *>(a[4]),
                                        static_cast<double *>(x), dims, ndim, solvedim, buf,
                                        bytes, s);
  return pentadsolver_S_gpsv_batch_ex(h, static_cast<const float *>(a[0]),
                                      static_cast<const float *>(a[1]),
                                      static_cast<const float *>(a[2]),
                                      static_cast<const float *>(a[3]),
                                      static_cast<const float *>(a[4]), static_cast<float *>(x),
                                      dims, ndim, solvedim, buf, bytes, s);
}

}  // namespace

extern "C" PENTAD_API pentadStatus_t pentadsolver_adi_create(
    pentadsolver_handle_t handle, int elem_bytes, const void *ds, const void *dl, const void *d,
    const void *du, const void *dw, void *x, const int *t_dims, int t_ndim, int iterations,
    void *t_buffer, size_t t_buffer_bytes, pentadsolver_adi_t *adi) {
  if (adi == nullptr) return PENTAD_STATUS_INVALID_VALUE;
  *adi = nullptr;
  if ((elem_bytes != 4 && elem_bytes != 8) || !ds || !dl || !d || !du || !dw || !x ||
      t_buffer == nullptr || iterations < 1 || iterations > 100000)
    return PENTAD_STATUS_INVALID_VALUE;
  size_t need = 0, points = 1;
  pentadStatus_t st = pentadsolver_buffer_size_ex(handle, elem_bytes, t_dims, t_ndim, 0, &need);
  if (st != PENTAD_STATUS_SUCCESS) return st;
  for (int k = 0; k < t_ndim; ++k) points *= (size_t)t_dims[k];
  const size_t xbytes = points * (size_t)elem_bytes;
  if (t_buffer_bytes < need || need < 4 * xbytes) return PENTAD_STATUS_INVALID_VALUE;
  // the warm-up copy of x: the buffer's last x-sized, 256-byte aligned block
  unsigned char *base = static_cast<unsigned char *>(t_buffer);
  const uintptr_t end = reinterpret_cast<uintptr_t>(base) + t_buffer_bytes;
  unsigned char *copy = reinterpret_cast<unsigned char *>((end - xbytes) & ~uintptr_t(255));
  const size_t scratch_bytes = (size_t)(copy - base);
  const void *arrays[5] = {ds, dl, d, du, dw};
  // work queued on any stream may still use the buffer or write x: creation
  // waits for the device first (creation is set-up, not the solve path)
  if (cudaDeviceSynchronize() != cudaSuccess) {
    cudaGetLastError();
    return PENTAD_STATUS_EXECUTION_FAILED;
  }
  cudaStream_t s = nullptr;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    return PENTAD_STATUS_NOT_INITIALIZED;
  }
  auto fail = [&](pentadStatus_t e) {
    cudaStreamDestroy(s);
    cudaGetLastError();
    return e;
  };
  if (cudaMemcpyAsync(copy, x, xbytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return fail(PENTAD_STATUS_EXECUTION_FAILED);
  for (int axis = 0; axis < t_ndim; ++axis)
    if ((st = solve_ex(elem_bytes, handle, arrays, copy, t_dims, t_ndim, axis, base,
                       scratch_bytes, s)) != PENTAD_STATUS_SUCCESS)
      return fail(st);
  if (cudaStreamSynchronize(s) != cudaSuccess) return fail(PENTAD_STATUS_EXECUTION_FAILED);

  auto *a = new pentadsolver_adi_s();
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    delete a;
    return fail(PENTAD_STATUS_EXECUTION_FAILED);
  }
  for (int it = 0; it < iterations && st == PENTAD_STATUS_SUCCESS; ++it)
    for (int axis = 0; axis < t_ndim && st == PENTAD_STATUS_SUCCESS; ++axis)
      st = solve_ex(elem_bytes, handle, arrays, x, t_dims, t_ndim, axis, base, scratch_bytes, s);
  const cudaError_t ce = cudaStreamEndCapture(s, &a->graph);
  if (st == PENTAD_STATUS_SUCCESS &&
      (ce != cudaSuccess || cudaGraphInstantiate(&a->exec, a->graph, 0) != cudaSuccess))
    st = PENTAD_STATUS_EXECUTION_FAILED;
  if (st != PENTAD_STATUS_SUCCESS) {
    if (a->graph) cudaGraphDestroy(a->graph);
    delete a;
    return fail(st);
  }
  cudaStreamDestroy(s);
  a->launches = iterations * t_ndim;
  *adi = a;
  return PENTAD_STATUS_SUCCESS;
}

extern "C" PENTAD_API pentadStatus_t pentadsolver_adi_replay(pentadsolver_adi_t adi,
                                                             void *stream) {
  if (adi == nullptr || adi->exec == nullptr) return PENTAD_STATUS_INVALID_VALUE;
  if (cudaGraphLaunch(adi->exec, static_cast<cudaStream_t>(stream)) != cudaSuccess) {
    cudaGetLastError();
    return PENTAD_STATUS_EXECUTION_FAILED;
  }
  return PENTAD_STATUS_SUCCESS;
}

extern "C" PENTAD_API int pentadsolver_adi_launches(pentadsolver_adi_t adi) {
  return adi == nullptr ? 0 : adi->launches;
}

extern "C" PENTAD_API pentadStatus_t pentadsolver_adi_destroy(pentadsolver_adi_t adi) {
  if (adi == nullptr) return PENTAD_STATUS_INVALID_VALUE;
  if (adi->exec) cudaGraphExecDestroy(adi->exec);
  if (adi->graph) cudaGraphDestroy(adi->graph);
  cudaGetLastError();
  delete adi;
  return PENTAD_STATUS_SUCCESS;
}
