// thomas_kernels.cu -- Thomas-elimination kernels for one batch of lines.
//
// Two families:
//
//  * thomas_global ("naive"): one thread per system, the factorisation
//    (du2, dw2, x2) kept in the caller's scratch buffer, element-major
//    [row][system] so a warp touches consecutive addresses at every row.  The
//    any-shape fallback; 13 array passes (6 in, 3+3 scratch, 1 out).  It plays
//    the role of the reference's Algorithm 1
//    (src/cuda/singlenode/pentad_cuda.cu:1219-1314).
//
//  * thomas_tiled ("thomas-pcr" with P partitions per system, P = 1 or 2):
//    a CTA owns S systems.  Their rows stream through a shared-memory ring
//    filled by cp.async, the factorisation stays on chip in shared memory,
//    and the solution leaves through a coalesced copy-out, so HBM sees the
//    7 array passes the problem needs.  With P = 2 each system is split at
//    row m: one thread eliminates rows 0..m-1 downwards, a second eliminates
//    rows n-1..m upwards on the mirrored coefficients, a 4x4 interface solve
//    joins them, and each back-substitutes its half (a two-partition
//    Thomas/SPIKE hybrid that halves the serial recurrence per thread).
//    CONTIG selects the contiguous x layout, where the ring is filled by a
//    cooperative, transposing copy (consecutive threads read consecutive rows
//    of one system) instead of each thread fetching its own row.
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

// ---------------------------------------------------------------------------
// thomas_tiled
// ---------------------------------------------------------------------------
template <typename F, int S, int P, bool CONTIG, int R, int STAGES>
struct TiledShape {
  static constexpr int T = S * P;                       // threads
  static constexpr int STAGE_ELEMS = R * 6 * P * S;     // one ring slot
  static size_t smem_bytes(long long n) {
    return (size_t)(3 * n * S + (long long)STAGES * STAGE_ELEMS + P * S * 6) *
           sizeof(F);
  }
};

template <typename F, int S, int P, bool CONTIG, int R, int STAGES>
__global__ void __launch_bounds__(S *P)
thomas_tiled_kernel(const F *__restrict__ ds, const F *__restrict__ dl,
                    const F *__restrict__ d, const F *__restrict__ du,
                    const F *__restrict__ dw, F *__restrict__ x, Lines L,
                    long long n_tiles, int *__restrict__ status_word) {
  using Shape = TiledShape<F, S, P, CONTIG, R, STAGES>;
  constexpr int T = Shape::T;
  constexpr int SE = Shape::STAGE_ELEMS;
  static_assert(P == 1 || P == 2, "one or two partitions per system");

  extern __shared__ __align__(16) unsigned char smem_raw[];
  const long long n = L.n;
  F *scr = reinterpret_cast<F *>(smem_raw);  // [3][n][S]: du2, dw2, x2/x
  F *ring = scr + 3 * n * S;                 // [STAGES][R][6][P][S]
  F *ifc = ring + (long long)STAGES * SE;    // [P][S][6]

  const int t = threadIdx.x;
  const int sys = t % S;
  const int part = t / S;  // 0: rows 0..mt-1 downwards; 1: rows n-1..mt upwards
  const long long mt = (P == 2) ? (n + 1) / 2 : n;
  const long long mb = n - mt;
  const long long my_rows = (part == 0) ? mt : mb;
  const long long n_stages = (mt + R - 1) / R;
  const F *arr[6] = {ds, dl, d, du, dw, x};
  int status = 0;

  for (long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const long long s0 = tile * S;
    const bool active = (s0 + sys) < L.n_sys;
    const long long base = active ? line_base(L, s0 + sys) : 0;

    // Fill ring slot stg % STAGES with rows [stg*R, stg*R + R) of every part.
    auto issue = [&](long long stg) {
      if (stg < n_stages) {
        F *buf = ring + (stg % STAGES) * SE;
        if constexpr (!CONTIG) {
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const long long k = stg * R + r;
            if (active && k < my_rows) {
              const long long row = (part == 0) ? k : n - 1 - k;
              const long long g = base + row * L.inner;
#pragma unroll
              for (int q = 0; q < 6; ++q)
                cp_async_ca<sizeof(F)>(&buf[((r * 6 + q) * P + part) * S + sys],
                                       arr[q] + g);
            }
          }
        } else {
          // Item (q, pt, sy, r), r fastest: consecutive threads read
          // consecutive rows of one system (contiguous in memory).
#pragma unroll
          for (int q = 0; q < 6; ++q) {
#pragma unroll
            for (int j = 0; j < R; ++j) {
              const int it = t + j * T;  // in [0, P*S*R)
              const int r = it % R;
              const int sy = (it / R) % S;
              const int pt = it / (R * S);
              const long long k = stg * R + r;
              const long long rows_pt = (pt == 0) ? mt : mb;
              if (s0 + sy < L.n_sys && k < rows_pt) {
                const long long row = (pt == 0) ? k : n - 1 - k;
                const long long g = (s0 + sy) * n + row;  // inner == 1
                cp_async_ca<sizeof(F)>(&buf[((r * 6 + q) * P + pt) * S + sy],
                                       arr[q] + g);
              }
            }
          }
        }
      }
      cp_async_commit();
    };

#pragma unroll
    for (int q = 0; q < STAGES - 1; ++q) issue(q);

    Carry<F> c;
    c.zero();
    for (long long stg = 0; stg < n_stages; ++stg) {
      issue(stg + STAGES - 1);
      cp_async_wait<STAGES - 1>();
      if constexpr (CONTIG) __syncthreads();
      const F *buf = ring + (stg % STAGES) * SE;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const long long k = stg * R + r;
        if (active && k < my_rows) {
          const long long row = (part == 0) ? k : n - 1 - k;
          const F *v = buf + (r * 6 * P + part) * S + sys;
          F a = v[0 * P * S], b = v[1 * P * S], dd = v[2 * P * S];
          F e = v[3 * P * S], w = v[4 * P * S], rhs = v[5 * P * S];
          mask_row(row, n, a, b, e, w);
          if (part == 1) {  // eliminate upwards: mirror the band
            F tmp = a; a = w; w = tmp;
            tmp = b; b = e; e = tmp;
          }
          F u, vv, y;
          fwd_row(a, b, dd, e, w, rhs, c, u, vv, y, status);
          scr[(0 * n + row) * S + sys] = u;
          scr[(1 * n + row) * S + sys] = vv;
          scr[(2 * n + row) * S + sys] = y;
        }
      }
      if constexpr (CONTIG) __syncthreads();
    }
    cp_async_wait<0>();

    F xa, xb;  // the two solution values next to the part's first unsolved row
    if constexpr (P == 2) {
      F *mine = ifc + (part * S + sys) * 6;
      mine[0] = c.u1; mine[1] = c.u2; mine[2] = c.w1;
      mine[3] = c.w2; mine[4] = c.y1; mine[5] = c.y2;
      __syncthreads();
      const F *tp = ifc + (0 * S + sys) * 6;
      const F *bt = ifc + (1 * S + sys) * 6;
      F u0, u1, u2, u3;
      solve_interface(tp[1], tp[3], tp[5], tp[0], tp[2], tp[4],  // T1, T2
                      bt[0], bt[2], bt[4], bt[1], bt[3], bt[5],  // B1, B2
                      u0, u1, u2, u3);
      if (part == 0) {
        scr[(2 * n + (mt - 1)) * S + sys] = u1;
        scr[(2 * n + (mt - 2)) * S + sys] = u0;
        xa = u0; xb = u1;
        for (long long i = mt - 3; i >= 0; --i) {
          const F xi = scr[(2 * n + i) * S + sys] -
                       scr[(0 * n + i) * S + sys] * xa -
                       scr[(1 * n + i) * S + sys] * xb;
          scr[(2 * n + i) * S + sys] = xi;
          xb = xa; xa = xi;
        }
      } else {
        scr[(2 * n + mt) * S + sys] = u2;
        scr[(2 * n + mt + 1) * S + sys] = u3;
        xa = u3; xb = u2;
        for (long long i = mt + 2; i < n; ++i) {
          const F xi = scr[(2 * n + i) * S + sys] -
                       scr[(0 * n + i) * S + sys] * xa -
                       scr[(1 * n + i) * S + sys] * xb;
          scr[(2 * n + i) * S + sys] = xi;
          xb = xa; xa = xi;
        }
      }
    } else {
      xa = F(0); xb = F(0);
      for (long long i = n - 1; i >= 0; --i) {
        const F xi = scr[(2 * n + i) * S + sys] -
                     scr[(0 * n + i) * S + sys] * xa -
                     scr[(1 * n + i) * S + sys] * xb;
        scr[(2 * n + i) * S + sys] = xi;
        xb = xa; xa = xi;
      }
    }
    __syncthreads();

    // Coalesced copy-out of the tile's solution.
    const long long total = n * S;
    const F *sol = scr + 2 * n * S;
    if constexpr (!CONTIG) {
      // thread (sys, part) writes rows part, part+P, ...: a warp's lanes
      // cover consecutive systems of one row, i.e. consecutive addresses
      if (active)
        for (long long row = part; row < n; row += P)
          x[base + row * L.inner] = sol[row * S + sys];
    } else {
      const int ni = (int)n;
      for (int f = t; f < (int)total; f += T) {
        const int sy = f / ni;
        const int row = f - sy * ni;
        if (s0 + sy < L.n_sys) x[(s0 + sy) * n + row] = sol[row * S + sy];
      }
    }
    __syncthreads();
  }
  if (status) atomicOr(status_word, status);
}

template <typename F, int S, int P, bool CONTIG, int R, int STAGES>
static cudaError_t launch_tiled_impl(const SolveArgs<F> &a, int max_ctas,
                                     cudaStream_t stream) {
  using Shape = TiledShape<F, S, P, CONTIG, R, STAGES>;
  auto kern = thomas_tiled_kernel<F, S, P, CONTIG, R, STAGES>;
  const size_t smem = Shape::smem_bytes(a.L.n);
  cudaError_t err = cudaFuncSetAttribute(
      kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  const long long n_tiles = (a.L.n_sys + S - 1) / S;
  long long grid = n_tiles;
  if (max_ctas > 0 && grid > max_ctas) grid = max_ctas;
  if (grid > 0x7fffffffLL) grid = 0x7fffffffLL;
  kern<<<(unsigned)grid, Shape::T, smem, stream>>>(a.ds, a.dl, a.d, a.du, a.dw,
                                                   a.x, a.L, n_tiles, a.status);
  return cudaGetLastError();
}

template <typename F>
size_t tiled_smem_bytes(const TiledConfig &cfg, long long n) {
  const int S = cfg.S, P = cfg.P, R = cfg.R, ST = cfg.stages;
  return (size_t)(3 * n * S + (long long)ST * R * 6 * P * S + P * S * 6) *
         sizeof(F);
}

// The instantiated configurations.  (S, P, R, STAGES) per layout and
// precision; the dispatcher and the autotuner choose among them.
#define PENTA_TILED_CONFIGS(X)       \
  X(double, 16, 2, false, 1, 8)      \
  X(double, 16, 2, false, 2, 4)      \
  X(double, 32, 1, false, 1, 6)      \
  X(double, 8, 2, false, 1, 8)       \
  X(double, 16, 2, true, 4, 2)       \
  X(double, 16, 2, true, 2, 4)       \
  X(double, 8, 2, true, 8, 2)        \
  X(double, 16, 1, true, 4, 2)       \
  X(float, 16, 2, false, 1, 8)       \
  X(float, 32, 2, false, 1, 8)       \
  X(float, 32, 1, false, 1, 8)       \
  X(float, 16, 2, true, 8, 2)        \
  X(float, 16, 2, true, 4, 4)        \
  X(float, 32, 2, true, 4, 2)        \
  X(float, 32, 1, true, 4, 2)

template <typename F> const std::vector<TiledConfig> &tiled_configs() {
  static const std::vector<TiledConfig> v = [] {
    std::vector<TiledConfig> out;
#define PENTA_X(FT_, S_, P_, C_, R_, ST_) \
  if (std::is_same<F, FT_>::value) out.push_back(TiledConfig{S_, P_, C_, R_, ST_});
    PENTA_TILED_CONFIGS(PENTA_X)
#undef PENTA_X
    return out;
  }();
  return v;
}

template <typename F>
cudaError_t launch_thomas_tiled(const SolveArgs<F> &a, const TiledConfig &cfg,
                                int max_ctas, cudaStream_t stream) {
#define PENTA_X(FT_, S_, P_, C_, R_, ST_)                                   \
  if (std::is_same<F, FT_>::value && cfg.S == S_ && cfg.P == P_ &&          \
      cfg.contig == C_ && cfg.R == R_ && cfg.stages == ST_)                 \
    return launch_tiled_impl<FT_, S_, P_, C_, R_, ST_>(                     \
        reinterpret_cast<const SolveArgs<FT_> &>(a), max_ctas, stream);
  PENTA_TILED_CONFIGS(PENTA_X)
#undef PENTA_X
  return cudaErrorInvalidConfiguration;
}

template <typename F>
int tiled_occupancy(const TiledConfig &cfg, long long n) {
  int blocks = 0;
  const size_t smem = tiled_smem_bytes<F>(cfg, n);
#define PENTA_X(FT_, S_, P_, C_, R_, ST_)                                      \
  if (std::is_same<F, FT_>::value && cfg.S == S_ && cfg.P == P_ &&             \
      cfg.contig == C_ && cfg.R == R_ && cfg.stages == ST_) {                  \
    auto kern = thomas_tiled_kernel<FT_, S_, P_, C_, R_, ST_>;                 \
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                             (int)smem) != cudaSuccess) {                      \
      cudaGetLastError();                                                      \
      return 0;                                                                \
    }                                                                          \
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, S_ * P_,  \
                                                      smem) != cudaSuccess) {  \
      cudaGetLastError();                                                      \
      return 0;                                                                \
    }                                                                          \
    return blocks;                                                             \
  }
  PENTA_TILED_CONFIGS(PENTA_X)
#undef PENTA_X
  return 0;
}

template cudaError_t launch_thomas_global<double>(const SolveArgs<double> &,
                                                  cudaStream_t);
template cudaError_t launch_thomas_global<float>(const SolveArgs<float> &,
                                                 cudaStream_t);
template cudaError_t launch_thomas_tiled<double>(const SolveArgs<double> &,
                                                 const TiledConfig &, int,
                                                 cudaStream_t);
template cudaError_t launch_thomas_tiled<float>(const SolveArgs<float> &,
                                                const TiledConfig &, int,
                                                cudaStream_t);
template size_t tiled_smem_bytes<double>(const TiledConfig &, long long);
template size_t tiled_smem_bytes<float>(const TiledConfig &, long long);
template int tiled_occupancy<double>(const TiledConfig &, long long);
template int tiled_occupancy<float>(const TiledConfig &, long long);
template const std::vector<TiledConfig> &tiled_configs<double>();
template const std::vector<TiledConfig> &tiled_configs<float>();

}  // namespace penta
