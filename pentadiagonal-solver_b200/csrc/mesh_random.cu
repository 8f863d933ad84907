// mesh_random.cu -- the reference's random test mesh, generated on the device.
//
// The reference's benchmarks (benchmarks/cuda/my_bm.cu:7-13) solve the grid
// that Mesh<Float>(solve_dim, dims) builds on the host (include/util/mesh.hpp:
// 85-124) and DeviceMesh copies to the GPU (include/util/device_mesh.hpp:52-65):
//
//   - every OpenMP thread t runs its own std::mt19937_64 seeded with t and
//     draws std::uniform_real_distribution<Float> values;
//   - the systems, in collapsed (outer i, inner j) order c = i * inner + j, are
//     split by the static schedule into nthreads contiguous chunks (the first
//     count % nthreads one system longer); thread t fills chunk t in order;
//   - per system, rows in order, per row the draws of ds (row > 1), dl
//     (row > 0), d, du (row < N-1), dw (row < N-2, with N unsigned, so a
//     one-row system draws it too) and x; ds, dl, du, dw = -u, d = 6u, x = u;
//     entries without a draw are 0.
//
// So the grid depends on the host's thread count; the entry points here take
// it as `n_threads` and write, straight into device arrays, the grid the
// reference builds with that many threads -- bit for bit, in FP64 and FP32.
//
// Device design: one CTA per host thread replays that thread's generator.
// MT19937-64 (Matsumoto and Nishimura; the parameters the C++ standard fixes
// for mt19937_64) keeps 312 words; a refill computes word k from words k,
// k+1 and k+156, so 156 lanes produce all 312 new words in one step: lane k
// makes word k from old words and word k+156 from its own new word k (and, for
// the last word, from a second copy of new word 0).  Each lane then tempers
// its two words, turns them into the two draws they are (draw index ->
// system, row, array) and stores them.  A stream is sequential, so a CTA
// emits 312 draws per step; the grid's time is set by draws per host thread.
// The canonical conversion is libstdc++'s generate_canonical with one 64-bit
// draw: u = (Float)v * 2^-64 rounded to nearest (an exact scaling), and the
// largest Float below 1 when the conversion rounds up to 2^64.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>

#include "pentad_common.hpp"
#include "pentadsolver_mesh.h"

namespace {

constexpr int kMtN = 312;
constexpr int kMtHalf = 156;
constexpr int kMeshThreads = 160;  // 156 working lanes, five warps

struct MeshShape {
  long long inner;   // product of dims below solvedim (row stride)
  long long n;       // rows per system
  long long count;   // systems
  long long per_sys; // draws per system
  int threads;       // host threads being replayed
};

__device__ __forceinline__ uint64_t mt_mix(uint64_t hi, uint64_t lo, uint64_t far) {
  const uint64_t y = (hi & 0xFFFFFFFF80000000ull) | (lo & 0x7FFFFFFFull);
  return far ^ (y >> 1) ^ ((y & 1ull) ? 0xB5026F5AA96619E9ull : 0ull);
}

__device__ __forceinline__ uint64_t mt_temper(uint64_t y) {
  y ^= (y >> 29) & 0x5555555555555555ull;
  y ^= (y << 17) & 0x71D67FFFEDA60000ull;
  y ^= (y << 37) & 0xFFF7EEE000000000ull;
  return y ^ (y >> 43);
}

template <typename F> __device__ __forceinline__ F canonical(uint64_t v);
template <> __device__ __forceinline__ double canonical<double>(uint64_t v) {
  const double u = __ull2double_rn(v) * 0x1p-64;
  return u >= 1.0 ? 0x1.fffffffffffffp-1 : u;
}
template <> __device__ __forceinline__ float canonical<float>(uint64_t v) {
  const float u = __ull2float_rn(v) * 0x1p-64f;
  return u >= 1.0f ? 0x1.fffffep-1f : u;
}

// Draws in rows [0, r) of a system of n rows.
__device__ __forceinline__ long long draws_before(long long r, long long n) {
  const long long ds = r > 2 ? r - 2 : 0;
  const long long dl = r > 1 ? r - 1 : 0;
  const long long du = r < n - 1 ? r : n - 1;
  const long long dw = n >= 2 ? (r < n - 2 ? r : n - 2) : r;
  return 2 * r + ds + dl + du + dw;
}

template <typename F> struct MeshOut {
  F *a[6];  // ds, dl, d, du, dw, x
  // selected with constant indices only, so the pointers stay in registers
  __device__ __forceinline__ F *pick(int slot) const {
    F *p = a[0];
#pragma unroll
    for (int q = 1; q < 6; ++q) p = slot == q ? a[q] : p;
    return p;
  }
};

// Stores draw number g (0-based) of host thread t's stream: value v.
template <typename F>
__device__ __forceinline__ void place(const MeshShape &s, long long lo, long long g, F v,
                                      const MeshOut<F> &out) {
  const long long sys = lo + g / s.per_sys;
  const long long e = g % s.per_sys;
  // row: the largest r with draws_before(r) <= e (each row draws at least twice)
  long long a = 0, b = s.n;
  while (b - a > 1) {
    const long long mid = (a + b) >> 1;
    if (draws_before(mid, s.n) <= e) a = mid; else b = mid;
  }
  const long long r = a;
  const int k = static_cast<int>(e - draws_before(r, s.n));
  const bool has[6] = {r > 1, r > 0, true, r < s.n - 1,
                       s.n >= 2 ? r < s.n - 2 : true, true};
  int slot = 0;
  for (int seen = -1; slot < 6; ++slot) {
    seen += has[slot] ? 1 : 0;
    if (seen == k) break;
  }
  const long long i = sys / s.inner, j = sys - i * s.inner;
  const long long idx = i * s.inner * s.n + j + r * s.inner;
  out.pick(slot)[idx] = slot == 2 ? F(6) * v : (slot == 5 ? v : -v);
  if (slot == 2) {
    // the row's entries that take no draw, written once per row
#pragma unroll
    for (int q = 0; q < 5; ++q)
      if (q != 2 && !has[q]) out.a[q][idx] = F(0);
  }
}

template <typename F>
__global__ void __launch_bounds__(kMeshThreads)
mesh_random_kernel(MeshShape s, F *ds, F *dl, F *d, F *du, F *dw, F *x) {
  __shared__ uint64_t mt[kMtN];
  const MeshOut<F> out{{ds, dl, d, du, dw, x}};
  const long long t = blockIdx.x;
  const long long q = s.count / s.threads, rem = s.count % s.threads;
  const long long lo = q * t + (t < rem ? t : rem);
  const long long total = (q + (t < rem ? 1 : 0)) * s.per_sys;
  if (total == 0) return;
  const int k = threadIdx.x;

  if (k == 0) {
    uint64_t w = static_cast<uint64_t>(t);
    mt[0] = w;
    for (int i = 1; i < kMtN; ++i) {
      w = 6364136223846793005ull * (w ^ (w >> 62)) + static_cast<uint64_t>(i);
      mt[i] = w;
    }
  }
  __syncthreads();

  for (long long base = 0; base < total; base += kMtN) {
    uint64_t lo_new = 0, hi_new = 0;
    if (k < kMtHalf) {
      const uint64_t a0 = mt[k], a1 = mt[k + 1], b0 = mt[k + kMtHalf];
      // word k + 157 is old, except after the last word, where it is new word 0
      const uint64_t b1 = k + 1 < kMtHalf ? mt[k + kMtHalf + 1]
                                          : mt_mix(mt[0], mt[1], mt[kMtHalf]);
      lo_new = mt_mix(a0, a1, b0);
      hi_new = mt_mix(b0, b1, lo_new);
    }
    __syncthreads();  // every old word read before any is replaced
    if (k < kMtHalf) {
      mt[k] = lo_new;
      mt[k + kMtHalf] = hi_new;
      const long long g0 = base + k, g1 = base + kMtHalf + k;
      if (g0 < total) place<F>(s, lo, g0, canonical<F>(mt_temper(lo_new)), out);
      if (g1 < total) place<F>(s, lo, g1, canonical<F>(mt_temper(hi_new)), out);
    }
    __syncthreads();  // the new words are in place before the next refill
  }
}

template <typename F>
pentadStatus_t mesh_random(const int *dims, int ndims, int solvedim, int n_threads, F *ds,
                           F *dl, F *d, F *du, F *dw, F *x, void *stream) {
  if (dims == nullptr || ndims < 1 || ndims > PENTAD_MAXDIM || solvedim < 0 ||
      solvedim >= ndims || n_threads < 1 || n_threads > PENTADSOLVER_MESH_MAX_THREADS)
    return PENTAD_STATUS_INVALID_VALUE;
  if (!ds || !dl || !d || !du || !dw || !x) return PENTAD_STATUS_INVALID_VALUE;
  MeshShape s{1, dims[solvedim], 1, 0, n_threads};
  for (int k = 0; k < ndims; ++k) {
    if (dims[k] < 1) return PENTAD_STATUS_INVALID_VALUE;
    if (k < solvedim) s.inner *= dims[k];
    if (k != solvedim) s.count *= dims[k];
  }
  // draws per system: rows 0..n-1 in full
  {
    const long long n = s.n, r = n;
    const long long dsn = r > 2 ? r - 2 : 0, dln = r > 1 ? r - 1 : 0;
    const long long dun = r < n - 1 ? r : n - 1;
    const long long dwn = n >= 2 ? (r < n - 2 ? r : n - 2) : r;
    s.per_sys = 2 * r + dsn + dln + dun + dwn;
  }
  mesh_random_kernel<F><<<n_threads, kMeshThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      s, ds, dl, d, du, dw, x);
  if (cudaGetLastError() != cudaSuccess) return PENTAD_STATUS_EXECUTION_FAILED;
  return PENTAD_STATUS_SUCCESS;
}

}  // namespace

extern "C" PENTAD_API pentadStatus_t pentadsolver_D_mesh_random(
    const int *dims, int ndims, int solvedim, int n_threads, double *ds, double *dl,
    double *d, double *du, double *dw, double *x, void *stream) {
  return mesh_random<double>(dims, ndims, solvedim, n_threads, ds, dl, d, du, dw, x, stream);
}

extern "C" PENTAD_API pentadStatus_t pentadsolver_S_mesh_random(
    const int *dims, int ndims, int solvedim, int n_threads, float *ds, float *dl, float *d,
    float *du, float *dw, float *x, void *stream) {
  return mesh_random<float>(dims, ndims, solvedim, n_threads, ds, dl, d, du, dw, x, stream);
}
