// tiled_kernels.cu -- the on-chip Thomas kernels ("thomas-pcr", P = 1 or 2
// partitions per system; "transpose" is the P = 1 contiguous variant).
//
// One warp owns S = 32 / P systems.  Their rows stream HBM -> shared memory
// through a ring of cp.async stages; the factorisation (du2, dw2, x2 -- three
// values per row, 24 B/row in FP64) stays in shared memory; the solution is
// written once.  HBM therefore sees the 7 array passes the problem needs
// (5 coefficient arrays + RHS in, solution out) instead of the 13 of a
// factorisation kept in global scratch.
//
// P = 2 splits every system at row m = ceil(n/2): lanes 0..S-1 eliminate rows
// 0..m-1 downwards, lanes S..2S-1 eliminate rows n-1..m upwards on the
// mirrored band (ds<->dw, dl<->du), the two halves meet in a 4x4 interface
// solve exchanged by warp shuffles, and each half back-substitutes away from
// the cut.  That halves the serial recurrence each lane walks, which is what
// bounds a warp's throughput here (the dependent chain pivot -> reciprocal ->
// next pivot), at no extra storage.
//
// CTAs are persistent: each walks tiles b, b + gridDim, ...  Ring stages are
// numbered across the CTA's whole tile sequence, so while one tile runs its
// interface solve and backward sweep the first stages of the next tile are
// already in flight.
//
// Layouts (elements of F):
//   ring    [STAGES][R][6][32]          lane = part * S + sys, so a warp reads
//                                       256 contiguous bytes per array/row
//   strided scratch [3][n][S]           row-major, rows of S systems
//   contig  scratch [3][S][n + 1]       system-major with an odd row pitch: the
//                                       compute lanes (one row, 16 systems) and
//                                       the copy-out (one system, 32 rows) are
//                                       both free of bank conflicts
// All in-tile arithmetic is 32-bit; the host only selects these kernels when
// the grid has fewer than 2^31 elements.
#include "penta_device.cuh"
#include "penta_internal.hpp"

namespace penta {
namespace {

template <typename F, int P, bool CONTIG, int R, int STAGES>
struct TileGeom {
  static constexpr int S = 32 / P;
  static constexpr int SLOT = R * 6 * 32;
  static long long scratch_elems(long long n) {
    return CONTIG ? 3LL * S * (n + 1) : 3LL * n * S;
  }
  static size_t smem_bytes(long long n) {
    return (size_t)(scratch_elems(n) + (long long)STAGES * SLOT) * sizeof(F);
  }
};

// Where the tile's systems live.
struct TileCtx {
  int base;   // element offset of (system 0 of the tile, row 0)
  int count;  // systems of the tile that exist (<= S)
};

template <int S, bool CONTIG>
__device__ __forceinline__ TileCtx tile_ctx(int tile, int n, int inner,
                                            int tiles_per_run, int n_sys) {
  TileCtx c;
  if constexpr (CONTIG) {
    const int s0 = tile * S;
    c.base = s0 * n;
    c.count = min(S, n_sys - s0);
  } else {
    const int run = tile / tiles_per_run;
    const int j0 = (tile - run * tiles_per_run) * S;
    c.base = run * inner * n + j0;
    c.count = min(S, inner - j0);
  }
  return c;
}

template <typename F, int P, bool CONTIG, int R, int STAGES>
__global__ void __launch_bounds__(32)
tiled_kernel(const F *__restrict__ ds, const F *__restrict__ dl,
             const F *__restrict__ d, const F *__restrict__ du,
             const F *__restrict__ dw, F *__restrict__ x, int n, int inner,
             int n_sys, int tiles_per_run, int n_tiles,
             int *__restrict__ status_word) {
  using G = TileGeom<F, P, CONTIG, R, STAGES>;
  constexpr int S = G::S;
  constexpr int SLOT = G::SLOT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  F *const scr = reinterpret_cast<F *>(smem_raw);
  const int sc_pitch = CONTIG ? S * (n + 1) : n * S;  // one scratch array
  F *const ring = scr + 3 * sc_pitch;

  const int lane = threadIdx.x;
  const int sys = lane % S;
  const int part = lane / S;
  const int mt = (P == 2) ? (n + 1) / 2 : n;
  const int mb = n - mt;
  const int my_rows = part ? mb : mt;
  const int n_stages = (mt + R - 1) / R;
  // Ring slot q holds, for a lane of the lower part, the band mirrored
  // (ds<->dw, dl<->du) so that every lane runs the same downward recurrence.
  const F *const band_dn[6] = {ds, dl, d, du, dw, x};
  const F *const band_up[6] = {dw, du, d, dl, ds, x};
  const int sc_sys = CONTIG ? sys * (n + 1) : sys;
  const int sc_row = CONTIG ? 1 : S;

  const int my_first = blockIdx.x;
  const int my_tiles = (my_first < n_tiles)
                           ? (n_tiles - 1 - my_first) / (int)gridDim.x + 1
                           : 0;

  // ---- producer: the next stage to issue (tile p_ti, stage p_g, slot) ----
  // In elimination order a lane's k-th row is k (upper part) or n-1-k
  // (lower part).  Ring entries that fall outside the line (k < 2 for slot
  // 0 = ds', k < 1 for slot 1 = dl') are written as zeros instead of loaded,
  // so the consumer needs no masking.
  int p_ti = 0, p_g = 0, p_slot = 0;
  const F *p_src[CONTIG ? R : 1][6];
  int p_dst[CONTIG ? R : 1];
  int p_lim[CONTIG ? R : 1];
  int p_dir[CONTIG ? R : 1];
  int p_off = 0, p_step = 0;
  bool p_ok = false;
  auto setup_tile = [&](int ti) {
    const TileCtx t = tile_ctx<S, CONTIG>(my_first + ti * (int)gridDim.x, n,
                                          inner, tiles_per_run, n_sys);
    if constexpr (!CONTIG) {
      p_ok = sys < t.count;
      const int o = t.base + sys + (part ? (n - 1) * inner : 0);
#pragma unroll
      for (int q = 0; q < 6; ++q) p_src[0][q] = (part ? band_up[q] : band_dn[q]) + o;
      p_off = 0;
      p_step = part ? -inner : inner;
    } else {
#pragma unroll
      for (int j = 0; j < R; ++j) {  // item: r fastest, then system, then part
        const int it = lane + 32 * j;
        const int r = it % R, sy = (it / R) % S, pt = it / (R * S);
        const int o = t.base + sy * n + (pt ? n - 1 - r : r);
#pragma unroll
        for (int q = 0; q < 6; ++q) p_src[j][q] = (pt ? band_up[q] : band_dn[q]) + o;
        p_dst[j] = (r * 6) * 32 + pt * S + sy;
        p_lim[j] = (sy < t.count) ? (pt ? mb : mt) - r : 0;  // rows left
        p_dir[j] = pt ? -1 : 1;
      }
    }
  };
  if (my_tiles > 0) setup_tile(0);

  auto issue_next = [&]() {
    if (p_ti < my_tiles) {
      F *slot = ring + p_slot * SLOT;
      const int k0 = p_g * R;
      if constexpr (!CONTIG) {
        if (p_ok) {
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int k = k0 + r;
            if (k < my_rows) {
#pragma unroll
              for (int q = 0; q < 6; ++q) {
                F *dst = slot + (r * 6 + q) * 32 + lane;
                if (q < 2 && k < 2 - q)
                  *dst = F(0);
                else
                  cp_async_ca<sizeof(F)>(dst, p_src[0][q] + p_off);
              }
            }
            p_off += p_step;
          }
        }
      } else {
#pragma unroll
        for (int j = 0; j < R; ++j) {
          const int r = (lane + 32 * j) % R;
          const int k = k0 + r;
          if (k0 < p_lim[j]) {
            const int koff = p_dir[j] * k0;
#pragma unroll
            for (int q = 0; q < 6; ++q) {
              F *dst = slot + p_dst[j] + q * 32;
              if (q < 2 && k < 2 - q)
                *dst = F(0);
              else
                cp_async_ca<sizeof(F)>(dst, p_src[j][q] + koff);
            }
          }
        }
      }
      if (++p_g == n_stages) {
        p_g = 0;
        if (++p_ti < my_tiles) setup_tile(p_ti);
      }
    }
    cp_async_commit();
    p_slot = (p_slot + 1 == STAGES) ? 0 : p_slot + 1;
  };

#pragma unroll
  for (int q = 0; q < STAGES - 1; ++q) issue_next();

  bool bad = false;
  int c_slot = 0;
  for (int ti = 0; ti < my_tiles; ++ti) {
    const TileCtx tc = tile_ctx<S, CONTIG>(my_first + ti * (int)gridDim.x, n,
                                           inner, tiles_per_run, n_sys);
    const bool active = sys < tc.count;

    // ---------------- forward elimination into shared scratch -------------
    Carry<F> c;
    c.zero();
    F *sp = scr + sc_sys + (part ? (n - 1) : 0) * sc_row;
    const int sp_step = part ? -sc_row : sc_row;
#pragma unroll 2
    for (int g = 0; g < n_stages; ++g) {
      issue_next();
      cp_async_wait<STAGES - 1>();
      if constexpr (CONTIG) __syncwarp();
      const F *v = ring + c_slot * SLOT + lane;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int k = g * R + r;
        if (active && k < my_rows) {
          F u, vv, y;
          fwd_row_fast(v[(r * 6 + 0) * 32], v[(r * 6 + 1) * 32],
                       v[(r * 6 + 2) * 32], v[(r * 6 + 3) * 32],
                       v[(r * 6 + 4) * 32], v[(r * 6 + 5) * 32], c, u, vv, y,
                       bad);
          sp[0] = u;
          sp[sc_pitch] = vv;
          sp[2 * sc_pitch] = y;
          sp += sp_step;
        }
      }
      if constexpr (CONTIG) __syncwarp();
      c_slot = (c_slot + 1 == STAGES) ? 0 : c_slot + 1;
    }

    // ---------------- join and backward substitution ----------------------
    // x(k) is the solution at this lane's k-th row (k = 0 is its first row
    // in elimination order, K = my_rows - 1 its last).  x(K) and x(K-1) come
    // from the cut (P = 2) or the line's end (P = 1); the sweep then runs
    // k = K-2 .. 0 with xa = x(k+1), xb = x(k+2).
    F xa, xb;
    int k0;
    if constexpr (P == 2) {
      const F pu1 = __shfl_xor_sync(0xffffffffu, c.u1, S);
      const F pu2 = __shfl_xor_sync(0xffffffffu, c.u2, S);
      const F pw1 = __shfl_xor_sync(0xffffffffu, c.w1, S);
      const F pw2 = __shfl_xor_sync(0xffffffffu, c.w2, S);
      const F py1 = __shfl_xor_sync(0xffffffffu, c.y1, S);
      const F py2 = __shfl_xor_sync(0xffffffffu, c.y2, S);
      // upper carries: rows m-1 (u1,w1,y1) and m-2 (u2,w2,y2);
      // lower carries: rows m (u1,w1,y1) and m+1 (u2,w2,y2)
      F u0, u1, u2, u3;
      if (part == 0)
        solve_interface(c.u2, c.w2, c.y2, c.u1, c.w1, c.y1, pu1, pw1, py1,
                        pu2, pw2, py2, u0, u1, u2, u3);
      else
        solve_interface(pu2, pw2, py2, pu1, pw1, py1, c.u1, c.w1, c.y1, c.u2,
                        c.w2, c.y2, u0, u1, u2, u3);
      xb = part ? u2 : u1;  // x(K): row m (lower part) / m-1 (upper part)
      xa = part ? u3 : u0;  // x(K-1): row m+1 / m-2
      k0 = my_rows - 3;
    } else {
      const int ib = sc_sys + (n - 1) * sc_row, ia = ib - sc_row;
      xb = scr[2 * sc_pitch + ib];
      xa = scr[2 * sc_pitch + ia] - scr[ia] * xb;
      k0 = n - 3;
    }
    const int row_K = part ? n - my_rows : my_rows - 1;  // row of x(K)
    const int rstep = part ? 1 : -1;                      // row(k) - row(k+1)

    if constexpr (!CONTIG) {
      // rows go straight to HBM: per part, lanes cover S adjacent systems
      if (active) {
        F *xo = x + (tc.base + sys + row_K * inner);
        const int ostep = rstep * inner;
        xo[0] = xb;
        xo += ostep;
        xo[0] = xa;
        const F *s2 = scr + sc_sys + (row_K + 2 * rstep) * sc_row;
        const int s2_step = rstep * sc_row;
#pragma unroll 2
        for (int k = k0; k >= 0; --k) {
          xo += ostep;
          const F xk = s2[2 * sc_pitch] - s2[0] * xa - s2[sc_pitch] * xb;
          xo[0] = xk;
          xb = xa;
          xa = xk;
          s2 += s2_step;
        }
      }
    } else {
      // solution into the x2 slot, then a coalesced copy-out per system
      if (active) {
        F *s2 = scr + sc_sys + row_K;
        s2[2 * sc_pitch] = xb;
        s2 += rstep;
        s2[2 * sc_pitch] = xa;
#pragma unroll 2
        for (int k = k0; k >= 0; --k) {
          s2 += rstep;
          const F xk = s2[2 * sc_pitch] - s2[0] * xa - s2[sc_pitch] * xb;
          s2[2 * sc_pitch] = xk;
          xb = xa;
          xa = xk;
        }
      }
      __syncwarp();
      const F *sol = scr + 2 * sc_pitch;
      for (int sy = 0; sy < tc.count; ++sy) {
        F *dst = x + (tc.base + sy * n);
        const F *src = sol + sy * (n + 1);
        for (int row = lane; row < n; row += 32) dst[row] = src[row];
      }
      __syncwarp();
    }
  }
  cp_async_wait<0>();
  if (__any_sync(0xffffffffu, bad) && lane == 0)
    atomicOr(status_word, STATUS_ZERO_PIVOT_BIT);
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side: the instantiated variants and their launch.
// ---------------------------------------------------------------------------
#define PENTA_TILED2_CONFIGS(X) \
  X(double, 2, false, 1, 11)    \
  X(double, 2, false, 1, 8)     \
  X(double, 2, false, 2, 5)     \
  X(double, 1, false, 1, 20)    \
  X(double, 2, true, 2, 5)      \
  X(double, 2, true, 4, 2)      \
  X(double, 2, true, 1, 10)     \
  X(double, 1, true, 2, 8)      \
  X(float, 2, false, 1, 9)      \
  X(float, 2, false, 2, 8)      \
  X(float, 1, false, 1, 16)     \
  X(float, 2, true, 2, 4)       \
  X(float, 2, true, 4, 4)       \
  X(float, 1, true, 2, 8)

template <typename F, int P, bool C, int R, int ST>
static cudaError_t tiled_launch(const SolveArgs<F> &a, int grid,
                                cudaStream_t stream) {
  using G = TileGeom<F, P, C, R, ST>;
  auto kern = tiled_kernel<F, P, C, R, ST>;
  const size_t smem = G::smem_bytes(a.L.n);
  cudaError_t err = cudaFuncSetAttribute(
      kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  const int n = (int)a.L.n, inner = (int)a.L.inner, n_sys = (int)a.L.n_sys;
  const int S = G::S;
  int tiles_per_run = 1, n_tiles;
  if (C) {
    n_tiles = (n_sys + S - 1) / S;
  } else {
    tiles_per_run = (inner + S - 1) / S;
    n_tiles = (n_sys / inner) * tiles_per_run;
  }
  if (grid <= 0 || grid > n_tiles) grid = n_tiles;
  kern<<<grid, 32, smem, stream>>>(a.ds, a.dl, a.d, a.du, a.dw, a.x, n, inner,
                                   n_sys, tiles_per_run, n_tiles, a.status);
  return cudaGetLastError();
}

template <typename F, int P, bool C, int R, int ST>
static int tiled_occ(long long n) {
  using G = TileGeom<F, P, C, R, ST>;
  auto kern = tiled_kernel<F, P, C, R, ST>;
  const size_t smem = G::smem_bytes(n);
  int blocks = 0;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, 32, smem) !=
          cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return blocks;
}

template <typename F> const std::vector<TiledConfig> &tiled2_configs() {
  static const std::vector<TiledConfig> v = [] {
    std::vector<TiledConfig> out;
#define PENTA_X(FT_, P_, C_, R_, ST_)   \
  if (std::is_same<F, FT_>::value)      \
    out.push_back(TiledConfig{32 / P_, P_, C_, R_, ST_});
    PENTA_TILED2_CONFIGS(PENTA_X)
#undef PENTA_X
    return out;
  }();
  return v;
}

template <typename F>
size_t tiled2_smem_bytes(const TiledConfig &c, long long n) {
  const long long S = c.S;
  const long long sc = c.contig ? 3 * S * (n + 1) : 3 * n * S;
  return (size_t)(sc + (long long)c.stages * c.R * 6 * 32) * sizeof(F);
}

template <typename F> int tiled2_occupancy(const TiledConfig &cfg, long long n) {
#define PENTA_X(FT_, P_, C_, R_, ST_)                                      \
  if (std::is_same<F, FT_>::value && cfg.P == P_ && cfg.contig == C_ &&    \
      cfg.R == R_ && cfg.stages == ST_)                                    \
    return tiled_occ<FT_, P_, C_, R_, ST_>(n);
  PENTA_TILED2_CONFIGS(PENTA_X)
#undef PENTA_X
  return 0;
}

template <typename F>
cudaError_t launch_tiled2(const SolveArgs<F> &a, const TiledConfig &cfg,
                          int grid, cudaStream_t stream) {
#define PENTA_X(FT_, P_, C_, R_, ST_)                                      \
  if (std::is_same<F, FT_>::value && cfg.P == P_ && cfg.contig == C_ &&    \
      cfg.R == R_ && cfg.stages == ST_)                                    \
    return tiled_launch<FT_, P_, C_, R_, ST_>(                             \
        reinterpret_cast<const SolveArgs<FT_> &>(a), grid, stream);
  PENTA_TILED2_CONFIGS(PENTA_X)
#undef PENTA_X
  return cudaErrorInvalidConfiguration;
}

template const std::vector<TiledConfig> &tiled2_configs<double>();
template const std::vector<TiledConfig> &tiled2_configs<float>();
template size_t tiled2_smem_bytes<double>(const TiledConfig &, long long);
template size_t tiled2_smem_bytes<float>(const TiledConfig &, long long);
template int tiled2_occupancy<double>(const TiledConfig &, long long);
template int tiled2_occupancy<float>(const TiledConfig &, long long);
template cudaError_t launch_tiled2<double>(const SolveArgs<double> &,
                                           const TiledConfig &, int,
                                           cudaStream_t);
template cudaError_t launch_tiled2<float>(const SolveArgs<float> &,
                                          const TiledConfig &, int,
                                          cudaStream_t);

}  // namespace penta
