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
// the last word, from a second copy of new word 0).  A batch refills 8 steps
// into a ring in shared memory (one barrier per step, little work), then 624
// threads temper and place its 2496 draws with no barrier between them: each
// keeps a cursor (system, draw within the system, first element) that moves
// 624 draws at a time without a division, and finds the row in closed form.
// A stream is sequential, so the grid's time is set by draws per host thread.
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
constexpr int kSteps = 8;           // generator steps refilled per batch
constexpr int kPerWord = 2;         // placing threads per word position
constexpr int kPlacers = kPerWord * kMtN;
constexpr int kMeshThreads = 640;   // 624 placing threads, 156 of them also refill
static_assert(kSteps % kPerWord == 0, "each placing thread takes every kPerWord-th step");

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

// Where draw e of a system falls: its row r and k, the draw's rank in the row.
// For n >= 4 the rows have 4, 5, 6, ..., 6, 5, 4 draws (row r >= 2 starts at
// draw 6r - 3 up to row n-2); shorter systems search the prefix counts.
__device__ __forceinline__ void row_of(long long e, long long n, long long &r, int &k) {
  if (n >= 4) {
    if (e < 4) {
      r = 0;
      k = static_cast<int>(e);
    } else if (e < 9) {
      r = 1;
      k = static_cast<int>(e - 4);
    } else if (e < 6 * n - 15) {
      const unsigned long long q = static_cast<unsigned long long>(e + 3) / 6ull;
      r = static_cast<long long>(q);
      k = static_cast<int>(e + 3 - 6 * r);
    } else if (e < 6 * n - 10) {
      r = n - 2;
      k = static_cast<int>(e - (6 * n - 15));
    } else {
      r = n - 1;
      k = static_cast<int>(e - (6 * n - 10));
    }
    return;
  }
  long long a = 0, b = n;  // the largest a with draws_before(a) <= e
  while (b - a > 1) {
    const long long mid = (a + b) >> 1;
    if (draws_before(mid, n) <= e) a = mid; else b = mid;
  }
  r = a;
  k = static_cast<int>(e - draws_before(a, n));
}

// A lane's position in its host thread's stream: draw e of system `sys`, whose
// first element is `start` (= i * inner * n + j for sys = i * inner + j).
struct Cursor {
  long long sys, e, j, start;
};

__device__ __forceinline__ void cursor_set(Cursor &c, const MeshShape &s, long long sys,
                                           long long e) {
  const long long i = sys / s.inner;
  c.sys = sys;
  c.e = e;
  c.j = sys - i * s.inner;
  c.start = i * s.inner * s.n + c.j;
}

// Moves the cursor `step` draws on; one system ahead at most without a division.
__device__ __forceinline__ void cursor_advance(Cursor &c, const MeshShape &s, long long step) {
  c.e += step;
  if (c.e < s.per_sys) return;
  if (c.e - s.per_sys < s.per_sys) {
    c.e -= s.per_sys;
    ++c.sys;
    ++c.start;
    if (++c.j == s.inner) {
      c.j = 0;
      c.start += s.inner * (s.n - 1);
    }
    return;
  }
  const long long w = c.e / s.per_sys;
  cursor_set(c, s, c.sys + w, c.e - w * s.per_sys);
}

// Stores the draw under cursor c, value v.
template <typename F>
__device__ __forceinline__ void place(const MeshShape &s, const Cursor &c, F v,
                                      const MeshOut<F> &out) {
  long long r;
  int k;
  row_of(c.e, s.n, r, k);
  const bool has[6] = {r > 1, r > 0, true, r < s.n - 1,
                       s.n >= 2 ? r < s.n - 2 : true, true};
  int slot = 0;
  for (int seen = -1; slot < 6; ++slot) {
    seen += has[slot] ? 1 : 0;
    if (seen == k) break;
  }
  const long long idx = c.start + r * s.inner;
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
  // the untempered words of the batch's steps; before the first batch the last
  // slot holds the seeded state
  __shared__ uint64_t ring[kSteps][kMtN];
  const MeshOut<F> out{{ds, dl, d, du, dw, x}};
  const long long t = blockIdx.x;
  const long long q = s.count / s.threads, rem = s.count % s.threads;
  const long long lo = q * t + (t < rem ? t : rem);
  const long long total = (q + (t < rem ? 1 : 0)) * s.per_sys;
  if (total == 0) return;
  const int k = threadIdx.x;

  if (k == 0) {
    uint64_t w = static_cast<uint64_t>(t);
    ring[kSteps - 1][0] = w;
    for (int i = 1; i < kMtN; ++i) {
      w = 6364136223846793005ull * (w ^ (w >> 62)) + static_cast<uint64_t>(i);
      ring[kSteps - 1][i] = w;
    }
  }
  // Thread k < 624 places word `word` of steps half, half + 2, ... of every
  // batch: draws half * 312 + word + 624 j of the stream.
  const int word = k % kMtN, half = k / kMtN;
  Cursor c;
  {
    const long long g = static_cast<long long>(half) * kMtN + word;
    cursor_set(c, s, lo + g / s.per_sys, g % s.per_sys);
  }
  __syncthreads();

  for (long long base = 0; base < total; base += kSteps * kMtN) {
    // Refill: step st from step st - 1 (the previous batch's last for st = 0).
    // Lane k makes word k and word k + 156; word k + 157 is old, except after
    // the last word, where it is new word 0 (made again here from old words).
#pragma unroll 1
    for (int st = 0; st < kSteps; ++st) {
      const uint64_t *prev = ring[(st + kSteps - 1) % kSteps];
      if (k < kMtHalf) {
        const uint64_t a0 = prev[k], a1 = prev[k + 1], b0 = prev[k + kMtHalf];
        const uint64_t b1 = k + 1 < kMtHalf ? prev[k + kMtHalf + 1]
                                            : mt_mix(prev[0], prev[1], prev[kMtHalf]);
        const uint64_t lo_new = mt_mix(a0, a1, b0);
        ring[st][k] = lo_new;
        ring[st][k + kMtHalf] = mt_mix(b0, b1, lo_new);
      }
      __syncthreads();
    }
    if (k < kPlacers) {
#pragma unroll
      for (int st = 0; st < kSteps; st += kPerWord) {
        const long long g = base + static_cast<long long>(st + half) * kMtN + word;
        if (g < total) place<F>(s, c, canonical<F>(mt_temper(ring[st + half][word])), out);
        cursor_advance(c, s, kPlacers);
      }
    }
    __syncthreads();  // the batch is placed before its slots are refilled
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
