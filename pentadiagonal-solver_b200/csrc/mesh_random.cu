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
// Device design: a cluster of up to 8 CTAs per host thread replays that
// thread's generator.  MT19937-64 (Matsumoto and Nishimura; the parameters the
// C++ standard fixes for mt19937_64) keeps 312 words; a refill computes word k
// from words k, k+1 and k+156, so 156 lanes produce all 312 new words in one
// step: lane k makes word k from old words and word k+156 from its own new
// word k (and, for the last word, from a second copy of new word 0).  Five
// warps of the cluster's first CTA refill 32 steps (9,984 draws) at a time
// into a double-buffered ring in its shared memory, one batch ahead, with a
// named barrier between steps; meanwhile 624 threads of every CTA of the
// cluster temper and place the current batch, reading the ring through
// distributed shared memory.  Each placing thread keeps a cursor (system, draw
// within the system, first element) that moves a fixed number of draws at a
// time without a division, and finds the row in closed form.  One cluster
// barrier per batch.  A stream is sequential: the time is set by the refill
// chain of one host thread.  The cluster width is the widest of which the
// device holds one per host thread at once (cudaOccupancyMaxActiveClusters):
// a second wave of clusters would double the time.
// The canonical conversion is libstdc++'s generate_canonical with one 64-bit
// draw: u = (Float)v * 2^-64 rounded to nearest (an exact scaling), and the
// largest Float below 1 when the conversion rounds up to 2^64.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>
#include <type_traits>

#include "pentad_common.hpp"
#include "pentadsolver_mesh.h"

namespace {

constexpr int kMtN = 312;
constexpr int kMtHalf = 156;
constexpr int kSteps = 32;                  // generator steps per batch
constexpr int kBatch = kSteps * kMtN;       // draws per batch (9984)
constexpr int kPlacers = 624;               // placing threads per CTA
constexpr int kPlaceWarps = 20;             // warps 0-19 place (624 of their 640 lanes)
constexpr int kRefillWarps = 5;             // warps 20-24 refill (156 of 160 lanes)
constexpr int kMeshThreads = 32 * (kPlaceWarps + kRefillWarps);
constexpr int kMaxCluster = 8;
constexpr size_t kRingBytes = 2ull * kBatch * sizeof(uint64_t);  // two batches
static_assert(kBatch % (kPlacers * kMaxCluster) == 0, "placers of a cluster tile a batch");

// I is the index type of everything within the grid: int when the grid has
// fewer than 2^31 points and a system fewer than 2^31 draws, else long long.
template <typename I> struct MeshShape {
  I inner;     // product of dims below solvedim (row stride)
  I n;         // rows per system
  I count;     // systems
  I per_sys;   // draws per system
  I lim_mid;   // 6 n - 15: first draw of row n - 2 (n >= 4)
  I lim_last;  // 6 n - 10: first draw of row n - 1 (n >= 4)
  int threads; // host threads being replayed
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
template <typename I> __device__ __forceinline__ I draws_before(I r, I n) {
  const I ds = r > 2 ? r - 2 : 0;
  const I dl = r > 1 ? r - 1 : 0;
  const I du = r < n - 1 ? r : n - 1;
  const I dw = n >= 2 ? (r < n - 2 ? r : n - 2) : r;
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
template <typename I>
__device__ __forceinline__ void row_of(const MeshShape<I> &s, I e, I &r, int &k) {
  using U = typename std::make_unsigned<I>::type;
  if (s.n >= 4) {
    if (e < 4) {
      r = 0;
      k = static_cast<int>(e);
    } else if (e < 9) {
      r = 1;
      k = static_cast<int>(e - 4);
    } else if (e < s.lim_mid) {
      r = static_cast<I>(static_cast<U>(e + 3) / U(6));
      k = static_cast<int>(e + 3 - 6 * r);
    } else if (e < s.lim_last) {
      r = s.n - 2;
      k = static_cast<int>(e - s.lim_mid);
    } else {
      r = s.n - 1;
      k = static_cast<int>(e - s.lim_last);
    }
    return;
  }
  I a = 0, b = s.n;  // the largest a with draws_before(a) <= e
  while (b - a > 1) {
    const I mid = (a + b) >> 1;
    if (draws_before<I>(mid, s.n) <= e) a = mid; else b = mid;
  }
  r = a;
  k = static_cast<int>(e - draws_before<I>(a, s.n));
}

// A lane's position in its host thread's stream: draw e of system `sys`, whose
// first element is `start` (= i * inner * n + j for sys = i * inner + j).
template <typename I> struct Cursor {
  I sys, e, j, start;
};

template <typename I>
__device__ __forceinline__ void cursor_set(Cursor<I> &c, const MeshShape<I> &s, I sys, I e) {
  const I i = sys / s.inner;
  c.sys = sys;
  c.e = e;
  c.j = sys - i * s.inner;
  c.start = i * s.inner * s.n + c.j;
}

// Moves the cursor `step` draws on; one system ahead at most without a division.
template <typename I>
__device__ __forceinline__ void cursor_advance(Cursor<I> &c, const MeshShape<I> &s, I step) {
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
  const I w = c.e / s.per_sys;
  cursor_set<I>(c, s, c.sys + w, c.e - w * s.per_sys);
}

// Stores the draw under cursor c, value v.
template <typename F, typename I>
__device__ __forceinline__ void place(const MeshShape<I> &s, const Cursor<I> &c, F v,
                                      const MeshOut<F> &out) {
  I r;
  int k;
  row_of<I>(s, c.e, r, k);
  const bool has[6] = {r > 1, r > 0, true, r < s.n - 1,
                       s.n >= 2 ? r < s.n - 2 : true, true};
  int slot = 0;
  for (int seen = -1; slot < 6; ++slot) {
    seen += has[slot] ? 1 : 0;
    if (seen == k) break;
  }
  const I idx = c.start + r * s.inner;
  out.pick(slot)[idx] = slot == 2 ? F(6) * v : (slot == 5 ? v : -v);
  if (slot == 2) {
    // the row's entries that take no draw, written once per row
#pragma unroll
    for (int q = 0; q < 5; ++q)
      if (q != 2 && !has[q]) out.a[q][idx] = F(0);
  }
}

__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ unsigned cluster_size() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}
// Every thread of every CTA of the cluster.  `release`: this thread's writes
// before it (the ring's shared memory) are visible to the cluster's reads after
// it.  Without it the arrive orders nothing -- the placing threads' loads are
// consumed before it anyway, and their scattered global stores need not drain
// at every batch.
__device__ __forceinline__ void cluster_sync_all(bool release) {
  __syncwarp();  // the .aligned forms want the whole warp converged
  if (release)
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
  else
    asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
__device__ __forceinline__ uint64_t ld_cluster_u64(uint32_t addr) {
  uint64_t v;
  asm volatile("ld.shared::cluster.u64 %0, [%1];" : "=l"(v) : "r"(addr) : "memory");
  return v;
}
__device__ __forceinline__ void refill_sync() {  // the five refilling warps only
  asm volatile("bar.sync 1, %0;" ::"n"(32 * kRefillWarps) : "memory");
}

// Steps 0 .. kSteps-1 of one batch into `cur`; step 0 follows `prev_last`.
// Lane k makes word k from old words and word k + 156 from its own new word k;
// word k + 157 is old except after the last word, where it is new word 0 (made
// again here from old words).
__device__ __forceinline__ void refill(uint64_t *cur, const uint64_t *prev_last, int k) {
#pragma unroll 1
  for (int st = 0; st < kSteps; ++st) {
    const uint64_t *prev = st == 0 ? prev_last : cur + (st - 1) * kMtN;
    uint64_t *out = cur + st * kMtN;
    if (k < kMtHalf) {
      const uint64_t a0 = prev[k], a1 = prev[k + 1], b0 = prev[k + kMtHalf];
      const uint64_t b1 = k + 1 < kMtHalf ? prev[k + kMtHalf + 1]
                                          : mt_mix(prev[0], prev[1], prev[kMtHalf]);
      const uint64_t lo_new = mt_mix(a0, a1, b0);
      out[k] = lo_new;
      out[k + kMtHalf] = mt_mix(b0, b1, lo_new);
    }
    refill_sync();
  }
}

// One host thread's stream per cluster of C CTAs (C = 1, 2, 4 or 8; blocks
// [t C, t C + C) replay thread t).  Warps 20-24 of the cluster's first CTA
// refill a double-buffered ring of batches in its shared memory, one batch
// ahead; warps 0-19 of every CTA place the current batch, reading the ring
// over distributed shared memory: placing thread p = rank * 624 + lane takes
// batch draws p, p + 624 C, ... (16 / C of them), so its draws in the stream
// are 624 C apart.  One cluster barrier per batch.
template <typename F, typename I>
__global__ void __launch_bounds__(kMeshThreads, 1)
mesh_random_kernel(MeshShape<I> s, F *ds, F *dl, F *d, F *du, F *dw, F *x) {
  extern __shared__ __align__(16) uint64_t ring[];  // [2][kSteps][312], first CTA only
  const MeshOut<F> out{{ds, dl, d, du, dw, x}};
  const unsigned rank = cluster_rank(), csize = cluster_size();
  const long long t = blockIdx.x / csize;
  const long long q = (long long)s.count / s.threads, rem = (long long)s.count % s.threads;
  const long long lo = q * t + (t < rem ? t : rem);
  const long long total = (q + (t < rem ? 1 : 0)) * (long long)s.per_sys;
  if (total == 0) return;  // the whole cluster (same t) leaves
  const int warp = threadIdx.x / 32;
  const bool refiller = rank == 0 && warp >= kPlaceWarps;
  const int rk = threadIdx.x - 32 * kPlaceWarps;  // lane within the refilling warps
  const int p_local = threadIdx.x;                // placing thread within the CTA
  const int stride = kPlacers * (int)csize;
  const int per_batch = kBatch / stride;          // draws per placing thread per batch
  const int p = (int)rank * kPlacers + p_local;

  if (refiller) {
    // seed into the last step of buffer 1, then batch 0 into buffer 0
    uint64_t *seed = ring + kBatch + (kSteps - 1) * kMtN;
    if (rk == 0) {
      uint64_t w = static_cast<uint64_t>(t);
      seed[0] = w;
      for (int i = 1; i < kMtN; ++i) {
        w = 6364136223846793005ull * (w ^ (w >> 62)) + static_cast<uint64_t>(i);
        seed[i] = w;
      }
    }
    refill_sync();
    refill(ring, seed, rk);
  }
  Cursor<I> c;
  if (p_local < kPlacers) cursor_set<I>(c, s, (I)lo + (I)p / s.per_sys, (I)p % s.per_sys);
  uint32_t ring0;  // the ring in the first CTA's shared memory
  asm volatile("mapa.shared::cluster.u32 %0, %1, 0;"
               : "=r"(ring0) : "r"((uint32_t)__cvta_generic_to_shared(ring)));
  cluster_sync_all(refiller);

  long long b = 0;
  for (long long base = 0; base < total; base += kBatch, ++b) {
    const int buf = (int)(b & 1);
    if (refiller && base + kBatch < total)
      refill(ring + (buf ^ 1) * kBatch, ring + buf * kBatch + (kSteps - 1) * kMtN, rk);
    if (p_local < kPlacers) {
      for (int i = 0; i < per_batch; ++i) {
        const int j = p + stride * i;  // draw within the batch
        if (base + j < total) {
          const uint64_t w = ld_cluster_u64(ring0 + (uint32_t)((buf * kBatch + j) * 8));
          place<F, I>(s, c, canonical<F>(mt_temper(w)), out);
        }
        cursor_advance<I>(c, s, (I)stride);
      }
    }
    cluster_sync_all(refiller);  // batch placed and the next one refilled
  }
}

constexpr int kMaxDevices = 64;
std::mutex g_mu;
// [FP32, FP64][32-bit, 64-bit indices][device][cluster width 1, 2, 4, 8]:
// clusters the device can hold at once (0 = not yet known, -1 = cannot launch)
int g_active[2][2][kMaxDevices][4] = {};

// How many clusters of `width` CTAs the device runs at once, found once per
// device, precision and width (clusters of 8 CTAs need 8 free SMs of one GPC,
// so fewer fit than SMs / 8).
template <typename F, typename I> int active_clusters(int dev, int width) {
  std::lock_guard<std::mutex> lock(g_mu);
  int &a = g_active[sizeof(F) == 8][sizeof(I) == 8][dev][width == 8 ? 3 : width / 2];
  if (a != 0) return a;
  a = -1;
  auto kern = mesh_random_kernel<F, I>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)kRingBytes) != cudaSuccess) {
    cudaGetLastError();
    return a;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)width);
  cfg.blockDim = dim3(kMeshThreads);
  cfg.dynamicSmemBytes = kRingBytes;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)width;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) == cudaSuccess && clusters > 0)
    a = clusters;
  cudaGetLastError();
  return a;
}

template <typename F, typename I>
pentadStatus_t launch_mesh(const MeshShape<I> &s, int n_threads, F *ds, F *dl, F *d, F *du,
                           F *dw, F *x, void *stream) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return PENTAD_STATUS_NOT_INITIALIZED;
  }
  auto kern = mesh_random_kernel<F, I>;
  // CTAs per host thread: the widest cluster (8, 4, 2) of which the device
  // holds one per host thread at once; else one CTA per host thread
  int csize = 1;
  for (int w = kMaxCluster; w > 1; w /= 2)
    if (active_clusters<F, I>(dev, w) >= n_threads) {
      csize = w;
      break;
    }
  if (csize == 1 && active_clusters<F, I>(dev, 1) < 1) return PENTAD_STATUS_EXECUTION_FAILED;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(n_threads * csize));
  cfg.blockDim = dim3(kMeshThreads);
  cfg.dynamicSmemBytes = kRingBytes;
  cfg.stream = static_cast<cudaStream_t>(stream);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)csize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (cudaLaunchKernelEx(&cfg, kern, s, ds, dl, d, du, dw, x) != cudaSuccess ||
      cudaGetLastError() != cudaSuccess) {
    cudaGetLastError();
    return PENTAD_STATUS_EXECUTION_FAILED;
  }
  return PENTAD_STATUS_SUCCESS;
}

template <typename F>
pentadStatus_t mesh_random(const int *dims, int ndims, int solvedim, int n_threads, F *ds,
                           F *dl, F *d, F *du, F *dw, F *x, void *stream) {
  if (dims == nullptr || ndims < 1 || ndims > PENTAD_MAXDIM || solvedim < 0 ||
      solvedim >= ndims || n_threads < 1 || n_threads > PENTADSOLVER_MESH_MAX_THREADS)
    return PENTAD_STATUS_INVALID_VALUE;
  if (!ds || !dl || !d || !du || !dw || !x) return PENTAD_STATUS_INVALID_VALUE;
  long long inner = 1, count = 1, points = 1;
  const long long n = dims[solvedim];
  for (int k = 0; k < ndims; ++k) {
    if (dims[k] < 1) return PENTAD_STATUS_INVALID_VALUE;
    if (k < solvedim) inner *= dims[k];
    if (k != solvedim) count *= dims[k];
    points *= dims[k];
  }
  // draws per system: rows 0..n-1 in full
  const long long per_sys = 2 * n + (n > 2 ? n - 2 : 0) + (n > 1 ? n - 1 : 0) + (n - 1) +
                            (n >= 2 ? n - 2 : n);
  if (points < (1LL << 31) && per_sys < (1LL << 31)) {
    const MeshShape<int> s{(int)inner, (int)n, (int)count, (int)per_sys,
                           (int)(6 * n - 15), (int)(6 * n - 10), n_threads};
    return launch_mesh<F, int>(s, n_threads, ds, dl, d, du, dw, x, stream);
  }
  const MeshShape<long long> s{inner, n, count, per_sys, 6 * n - 15, 6 * n - 10, n_threads};
  return launch_mesh<F, long long>(s, n_threads, ds, dl, d, du, dw, x, stream);
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
