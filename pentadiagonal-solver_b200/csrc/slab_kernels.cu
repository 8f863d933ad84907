// slab_kernels.cu -- the data movement of the slab-decomposed multi-GPU ADI.
//
// A grid of nx x ny x nz points (x contiguous) is split over `parts` ranks
// into slabs along z: rank k holds z in [k nzl, (k+1) nzl), all x and y, as
// A_k[zl][y][x].  x and y lines lie inside a slab and are solved where they
// are.  z lines cross every slab, so before the z solve the grid is
// transposed to slabs along y: rank r holds y in [r nyp, (r+1) nyp), all z,
// as B_r[z][yl][x] (nyp = ny / parts), and z lines are local again.
//
// One all-to-all of equal blocks does that transposition when each rank
// sends rank r the block  send[r][zl][yl][x] = A_k[zl][r nyp + yl][x]:  rank
// r then receives from rank k exactly B_r[k nzl + zl][yl][x], contiguous, so
// the receive buffer is B_r itself.  The way back sends B_r's contiguous
// blocks as they are and scatters what arrives with the inverse map.  Both
// maps copy parts * nzl segments of nyp * nx consecutive elements each:
// segment s = (r, zl) sits at (zl ny + r nyp) nx in A_k and at s nyp nx in
// the packed buffer.
//
// The kernels are plain bandwidth-bound copies: each CTA walks whole segments
// with 16-byte vectors when the segment length and both bases allow it (the
// usual case: nx a multiple of 2 in FP64, 4 in FP32), element copies
// otherwise.  Grid: one CTA per segment, at most 8 per SM.
#include <cuda_runtime.h>

#include <cstdint>

#include "pentad_common.hpp"
#include "pentadsolver_ext.h"
#include "penta_internal.hpp"

namespace penta {
namespace {

// One CTA per segment at a time (grid-stride over segments); its threads walk
// the segment's units.  Units are T: a 16-byte vector or one element.
template <typename T>
__global__ void __launch_bounds__(256)
slab_copy_kernel(const T *__restrict__ src, T *__restrict__ dst, long long seg_len, int nzl,
                 int parts, long long row_stride, int to_packed) {
  const long long n_seg = (long long)parts * nzl;
  for (long long s = blockIdx.x; s < n_seg; s += gridDim.x) {
    const long long r = s / nzl, zl = s - (s / nzl) * nzl;
    const long long a0 = zl * row_stride + r * seg_len;  // (zl ny + r nyp) nx
    const long long p0 = s * seg_len;                     // s nyp nx
    if (to_packed)
      for (long long j = threadIdx.x; j < seg_len; j += blockDim.x) dst[p0 + j] = src[a0 + j];
    else
      for (long long j = threadIdx.x; j < seg_len; j += blockDim.x) dst[a0 + j] = src[p0 + j];
  }
}

}  // namespace

cudaError_t launch_slab_copy(int elem_bytes, const void *src, void *dst, int nx, int ny,
                             int nz_local, int parts, bool to_packed, int sm_count,
                             cudaStream_t stream) {
  const long long nyp = ny / parts;
  const long long seg = nyp * nx;                   // elements per segment
  const long long row = (long long)ny * nx;         // elements per z plane
  const long long total = seg * parts * nz_local;   // elements moved
  if (total == 0) return cudaSuccess;
  const bool vec = (seg * elem_bytes) % 16 == 0 && (row * elem_bytes) % 16 == 0 &&
                   reinterpret_cast<uintptr_t>(src) % 16 == 0 &&
                   reinterpret_cast<uintptr_t>(dst) % 16 == 0;
  const int unit = vec ? 16 : elem_bytes;
  const long long seg_u = seg * elem_bytes / unit, row_u = row * elem_bytes / unit;
  const int threads = 256;
  long long blocks = (long long)parts * nz_local;     // one segment per CTA
  const long long cap = (long long)sm_count * 8;    // 8 CTAs of 256 threads per SM
  if (blocks > cap) blocks = cap;
  const int tp = to_packed ? 1 : 0;
  if (unit == 16)
    slab_copy_kernel<int4><<<(unsigned)blocks, threads, 0, stream>>>(
        static_cast<const int4 *>(src), static_cast<int4 *>(dst), seg_u, nz_local, parts, row_u,
        tp);
  else if (unit == 8)
    slab_copy_kernel<long long><<<(unsigned)blocks, threads, 0, stream>>>(
        static_cast<const long long *>(src), static_cast<long long *>(dst), seg_u, nz_local,
        parts, row_u, tp);
  else
    slab_copy_kernel<int><<<(unsigned)blocks, threads, 0, stream>>>(
        static_cast<const int *>(src), static_cast<int *>(dst), seg_u, nz_local, parts, row_u,
        tp);
  return cudaGetLastError();
}

}  // namespace penta

// ---------------------------------------------------------------------------
// C ABI (pentadsolver_ext.h)
// ---------------------------------------------------------------------------
namespace {
pentadStatus_t slab_entry(int elem_bytes, const void *src, void *dst, int nx, int ny,
                          int nz_local, int parts, bool to_packed, void *stream) {
  if ((elem_bytes != 4 && elem_bytes != 8) || src == nullptr || dst == nullptr || src == dst ||
      nx < 1 || ny < 1 || nz_local < 1 || parts < 1 || ny % parts != 0)
    return PENTAD_STATUS_INVALID_VALUE;
  if ((long long)nx * ny > (1LL << 40) / nz_local) return PENTAD_STATUS_INVALID_VALUE;
  if (reinterpret_cast<uintptr_t>(src) % elem_bytes || reinterpret_cast<uintptr_t>(dst) % elem_bytes)
    return PENTAD_STATUS_INVALID_VALUE;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return PENTAD_STATUS_NOT_INITIALIZED;
  }
  if (penta::launch_slab_copy(elem_bytes, src, dst, nx, ny, nz_local, parts, to_packed, sms,
                              static_cast<cudaStream_t>(stream)) != cudaSuccess) {
    cudaGetLastError();
    return PENTAD_STATUS_EXECUTION_FAILED;
  }
  return PENTAD_STATUS_SUCCESS;
}
}  // namespace

extern "C" PENTAD_API pentadStatus_t pentadsolver_slab_pack(int elem_bytes, const void *zslab,
                                                            void *send, int nx, int ny,
                                                            int nz_local, int parts,
                                                            void *stream) {
  return slab_entry(elem_bytes, zslab, send, nx, ny, nz_local, parts, true, stream);
}

extern "C" PENTAD_API pentadStatus_t pentadsolver_slab_unpack(int elem_bytes, const void *recv,
                                                              void *zslab, int nx, int ny,
                                                              int nz_local, int parts,
                                                              void *stream) {
  return slab_entry(elem_bytes, recv, zslab, nx, ny, nz_local, parts, false, stream);
}
