// shared_fact_kernels.cu -- shared factorisation: every line of the batch has
// the same coefficients (those of line 0), so the factorisation is computed
// once and only the right-hand sides move.
//
// Semantics follow the reference's Algorithm 4
// (src/cuda/singlenode/pentad_cuda.cu:957-1127): the table
// [ds | ddl | 1/dd | du2 | dw2] is built from line 0's coefficients, and the
// caller guarantees that every other line shares them (not checked).  Unlike
// the reference, out-of-range couplings (ds rows 0,1; dl row 0; du row n-1;
// dw rows n-2, n-1) are masked explicitly, so any value there -- NaN included
// -- is ignored, as on every other path.
//
// The Tensor-Memory kernel (n <= 256 in FP64, n <= 512 in FP32):
//  * one CTA per SM: for each TMEM lane quarter c, warp c runs the forward
//    substitution and warp 4 + c the back substitution of the same tiles, one
//    tile behind; warp 8 builds the table.  A tile is 32 lines (one per
//    lane).  The forward warp streams their right-hand sides through a ring
//    of TMA tiles {R rows x 32 lines} (along x: 128-byte rows, 128-byte
//    swizzle) that it refills itself and keeps x2 of every row in its TMEM
//    lane quarter (one tcgen05.st of 32 columns per stage); the back
//    substitution reads it back and writes x (directly along y/z, through a
//    swizzled shared tile and TMA stores along x).  Consecutive tiles fill
//    TMEM blocks in opposite orders and a progress word hands blocks over, as
//    in tmem_kernels.cu.  HBM traffic is the algorithmic 2 x sizeof(F) per
//    point; loads and stores carry an evict-first L2 policy.
//  * The builder warp loads line 0's coefficients, masks them and runs the
//    serial recurrence into a shared-memory table, publishing it R rows at a
//    time; consumers on their first tile follow it row block by row block.
//  * The table is cached at the end of the caller's buffer together with the
//    coefficients it came from.  When a later call finds its line-0
//    coefficients identical, bit for bit, to the cached ones, the builder
//    copies the table instead of recomputing it (e.g. the 50 iterations of an
//    ADI run); otherwise it recomputes and refreshes the cache.  The result is
//    the same either way.
//
// Other shapes use a one-thread-per-line kernel with x2 in the caller's buffer
// and a table built by a single-thread kernel, as in the reference.
#include <cstdlib>
#include <type_traits>

#include "penta_internal.hpp"
#include "tma_device.cuh"

namespace penta {
namespace {

constexpr int SL = 32;              // lines per consumer tile (one per lane)
constexpr int NCONS = 4;            // consumer warps: one per TMEM lane quarter
constexpr uint32_t kTmemCols = 512;
constexpr int kCacheMagic = 0x5f4a4355;  // table layout [e | a | inv | du2 | dw2]

// A stage is R = 16 (FP64) / 32 (FP32) rows, 128 bytes of a line along x
// (one TMA tile {R rows, 32 lines}, 128-byte swizzle), 32 TMEM columns.
template <typename F> constexpr int sf_rows_per_stage() { return 128 / (int)sizeof(F); }

// TMEM holds x2 for n_pad = R ceil(n / R) rows: 2 columns per FP64 row.
template <typename F> constexpr int sf_max_rows() {
  return (int)kTmemCols / ((int)sizeof(F) / 4);
}

template <typename F, bool CONTIG, int ST> struct SfGeom {
  static constexpr int R = sf_rows_per_stage<F>();
  static constexpr int SE = R * SL;                       // elements per stage
  static constexpr int OBE = CONTIG ? 2 * SE : 0;         // output tiles (2 buffers)
  static constexpr size_t kData = (size_t)(ST * SE + OBE) * sizeof(F);
  static constexpr size_t kCons = (kData + (ST + 2) * 8 + 1023) / 1024 * 1024;
  static constexpr int kTabRows = sf_max_rows<F>();
  // table [e | a | inv | du2 | dw2], line-0 inputs, cached inputs: 3 x 5 rows
  static constexpr size_t kTable = (size_t)15 * kTabRows * sizeof(F);
  static constexpr size_t kUsed = NCONS * kCons + kTable + 128 + 1024;
  // at least 116 KB, so that one CTA holds an SM (and all of its TMEM)
  static constexpr size_t kSmem = kUsed > 118784 ? kUsed : 118784;
  static constexpr int kCols = R * (int)sizeof(F) / 4;    // TMEM columns per stage (32)
  static constexpr int NB = (int)kTmemCols / kCols;       // TMEM blocks of one stage each
  static_assert(kCols == 32, "32 TMEM columns per stage");
  static_assert(kSmem <= 232448, "shared memory per CTA");
};

// The cache at the end of the caller's buffer:
// [header 128 B][inputs 5 x n_pad][table 5 x n_pad], one component after another.
struct SfCacheHeader {
  int magic;
  int n;
  int elem;
};

template <typename F>
__device__ __forceinline__ F sf_mask(int q, int i, int n, F v) {
  // q: 0 ds, 1 dl, 2 d, 3 du, 4 dw
  const bool out = (q == 0 && i < 2) || (q == 1 && i < 1) || (q == 3 && i >= n - 1) ||
                   (q == 4 && i >= n - 2) || i >= n;
  return out ? (q == 2 && i < n ? v : F(0)) : v;
}

template <typename F> __device__ __forceinline__ void put_x2(uint32_t (&tv)[32], int r, F v);
template <> __device__ __forceinline__ void put_x2<double>(uint32_t (&tv)[32], int r, double v) {
  tv[2 * r] = (uint32_t)__double2loint(v);
  tv[2 * r + 1] = (uint32_t)__double2hiint(v);
}
template <> __device__ __forceinline__ void put_x2<float>(uint32_t (&tv)[32], int r, float v) {
  tv[r] = __float_as_uint(v);
}
template <typename F> __device__ __forceinline__ F get_x2(const uint32_t (&tv)[32], int r);
template <> __device__ __forceinline__ double get_x2<double>(const uint32_t (&tv)[32], int r) {
  return __hiloint2double((int)tv[2 * r + 1], (int)tv[2 * r]);
}
template <> __device__ __forceinline__ float get_x2<float>(const uint32_t (&tv)[32], int r) {
  return __uint_as_float(tv[r]);
}

__device__ __forceinline__ bool same_bits(double a, double b) {
  return __double_as_longlong(a) == __double_as_longlong(b);
}
__device__ __forceinline__ bool same_bits(float a, float b) {
  return __float_as_int(a) == __float_as_int(b);
}

// Bounded wait for the builder to publish `rows` table rows.
__device__ __forceinline__ bool wait_table(volatile int *ready, int rows) {
  if (*ready >= rows) return true;
  const unsigned long long t0 = global_ns();
  while (*ready < rows)
    if (global_ns() - t0 > 2000000000ull) return false;
  return true;
}

template <typename F, bool CONTIG, int ST>
__global__ void __launch_bounds__(32 * (2 * NCONS + 1), 1)
sf_tmem_kernel(const __grid_constant__ CUtensorMap xmap, const F *__restrict__ ds,
               const F *__restrict__ dl, const F *__restrict__ d, const F *__restrict__ du,
               const F *__restrict__ dw, F *__restrict__ x, unsigned char *__restrict__ cache,
               int n, int n_pad, int inner, int tpr, int n_sys, int n_tiles,
               int *__restrict__ status_word) {
  using G = SfGeom<F, CONTIG, ST>;
  using V2 = typename Vec2<F>::T;
  constexpr int R = G::R, SE = G::SE, NB = G::NB;
  constexpr int EPC = 16 / (int)sizeof(F);
  constexpr int TR = G::kTabRows;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *const base =
      smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const int warp = threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  F *const tab = reinterpret_cast<F *>(base + NCONS * G::kCons);  // [5][TR]
  F *const coef = tab + 5 * TR;                                    // line-0 inputs [5][TR]
  F *const cin = coef + 5 * TR;                                    // cached inputs [5][TR]
  unsigned char *const tail = base + NCONS * G::kCons + G::kTable;
  uint32_t *const tmem_slot = reinterpret_cast<uint32_t *>(tail);
  volatile int *const ready = reinterpret_cast<volatile int *>(tail + 16);
  volatile int *const stop = reinterpret_cast<volatile int *>(tail + 32);  // [NCONS]
  uint64_t *const cbar = reinterpret_cast<uint64_t *>(tail + 64);
  int *const prog = reinterpret_cast<int *>(tail + 96);                    // [NCONS]

  // The builder warp starts first: the table cache's bulk copies and the
  // gather of line 0's coefficients (every load of a lane issued before any
  // is used; rows lane + 32 j of each array) go out before the solving
  // warps' ring loads, which they would otherwise queue behind.
  constexpr int PL = (TR + 31) / 32;
  const bool builder = warp == 2 * NCONS;
  const long long stride = CONTIG ? 1 : inner;  // line 0's row stride
  SfCacheHeader *const hdr = reinterpret_cast<SfCacheHeader *>(cache);
  F *const c_in = cache ? reinterpret_cast<F *>(cache + 128) : nullptr;
  F *const c_tab = c_in ? c_in + 5 * (long long)n_pad : nullptr;
  F v[5][PL];
  bool same = false;
  if (builder) {
    if (cache != nullptr && lane == 0) {
      const unsigned comp = (unsigned)(n_pad * sizeof(F));
      mbar_init(cbar, 1);
      mbar_init_fence();
      mbar_expect_tx(cbar, 10u * comp);
      for (int q = 0; q < 5; ++q) {
        bulk_load(cin + q * TR, c_in + (long long)q * n_pad, comp, cbar);
        bulk_load(tab + q * TR, c_tab + (long long)q * n_pad, comp, cbar);
      }
    }
    const F *const src[5] = {ds, dl, d, du, dw};
#pragma unroll
    for (int q = 0; q < 5; ++q)
#pragma unroll
      for (int j = 0; j < PL; ++j) {
        const int i = lane + 32 * j;
        v[q][j] = i < n ? src[q][(long long)i * stride] : F(0);
      }
    if (cache != nullptr) {
      const volatile SfCacheHeader *vh = hdr;
      same = vh->magic == kCacheMagic && vh->n == n && vh->elem == (int)sizeof(F);
    }
  }

  if (threadIdx.x == 0) {
    for (int c = 0; c < NCONS; ++c) {
      uint64_t *f = reinterpret_cast<uint64_t *>(base + c * G::kCons + G::kData);
      for (int s = 0; s < ST + 2; ++s) mbar_init(&f[s], 1);
      stop[c] = 0;
      prog[c] = 0;
    }
    *ready = 0;
    mbar_init_fence();
  }
  if (warp == 0) tmem_alloc(tmem_slot, kTmemCols);
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  const uint32_t tmem_base = *tmem_slot;

  // ================================ builder =================================
  if (builder) {
    const int total = 5 * n_pad;
#pragma unroll
    for (int q = 0; q < 5; ++q)
#pragma unroll
      for (int j = 0; j < PL; ++j) {
        const int i = lane + 32 * j;
        if (i < n_pad) coef[q * TR + i] = sf_mask<F>(q, i, n, v[q][j]);
      }
    bool copies_done = true;
    if (cache != nullptr) copies_done = __all_sync(0xffffffffu, mbar_wait(cbar, 0));
    if (!copies_done) {  // the table area may still be written: publish nothing
      if (lane == 0) atomicOr(status_word, STATUS_TIMEOUT_BIT);
      return;
    }
    __syncwarp();
    if (same) {  // the gathered (masked) coefficients against the cached ones
#pragma unroll
      for (int q = 0; q < 5; ++q)
#pragma unroll
        for (int j = 0; j < PL; ++j) {
          const int i = lane + 32 * j;
          if (i < n_pad) same &= same_bits(sf_mask<F>(q, i, n, v[q][j]), cin[q * TR + i]);
        }
    }
    if (__all_sync(0xffffffffu, same)) {  // cached table: already in place
      __threadfence_block();
      __syncwarp();
      if (lane == 0) *ready = n_pad;
      return;
    }
    // lane 0 runs the recurrence, publishing R rows at a time
    if (lane == 0) {
      F pu2 = F(0), pu1 = F(0), pw2 = F(0), pw1 = F(0);
      bool bad = false;
      for (int i = 0; i < n_pad; ++i) {
        const F dsv = coef[i];
        const F ddl = coef[TR + i] - dsv * pu2;
        const F dd = coef[2 * TR + i] - dsv * pw2 - ddl * pu1;
        const F inv = (i < n) ? F(1) / dd : F(0);
        const F du2 = (coef[3 * TR + i] - ddl * pw1) * inv;
        const F dw2 = coef[4 * TR + i] * inv;
        bad |= (i < n) && !isfinite(inv);
        tab[i] = dsv * inv;       // e
        tab[TR + i] = ddl * inv;  // a
        tab[2 * TR + i] = inv;
        tab[3 * TR + i] = du2;
        tab[4 * TR + i] = dw2;
        pu2 = pu1; pu1 = du2;
        pw2 = pw1; pw1 = dw2;
        if ((i + 1) % R == 0) {
          __threadfence_block();
          *ready = i + 1;
        }
      }
      if (bad) atomicOr(status_word, STATUS_ZERO_PIVOT_BIT);
    }
    __syncwarp();
    // refresh the cache (CTA 0): header cleared, table, inputs, then the header
    if (cache != nullptr && blockIdx.x == 0) {
      if (lane == 0) hdr->magic = 0;
      __threadfence();
      __syncwarp();
      for (int k = lane; k < total; k += 32) {
        const int q = k / n_pad, i = k - q * n_pad;
        c_tab[k] = tab[q * TR + i];
      }
      __threadfence();
      __syncwarp();
      for (int k = lane; k < total; k += 32) {
        const int q = k / n_pad, i = k - q * n_pad;
        c_in[k] = coef[q * TR + i];
      }
      __threadfence();
      __syncwarp();
      if (lane == 0) {
        hdr->n = n;
        hdr->elem = (int)sizeof(F);
        __threadfence();
        hdr->magic = kCacheMagic;
      }
    }
    return;
  }

  // ============================ solving warps ===============================
  // warps 0..3 run the forward substitution of their lane quarter's tiles,
  // warps 4..7 the back substitution, one tile behind (a warp reaches the
  // TMEM lanes 32 (warp % 4) .. 32 (warp % 4) + 31)
  const bool fwd = warp < NCONS;
  const int cons = warp % NCONS;
  F *const ring = reinterpret_cast<F *>(base + cons * G::kCons);
  F *const obuf = ring + ST * SE;
  uint64_t *const full = reinterpret_cast<uint64_t *>(base + cons * G::kCons + G::kData);
  uint64_t *const hfull = full + ST;  // [2]: a tile's x2 is in TMEM
  const uint32_t taddr = tmem_base + ((uint32_t)(cons * 32) << 16);
  const int n_stages = n_pad / R;
  const int gw = blockIdx.x * NCONS + cons;
  const int tw = gridDim.x * NCONS;
  const int my_tiles = gw < n_tiles ? (n_tiles - 1 - gw) / tw + 1 : 0;
  const long long total = (long long)my_tiles * n_stages;
  const uint64_t pol_stream = l2_policy_first();  // every access is read or written once

  // element offset of this lane's row r inside a stage tile: along x a
  // 128-byte row per line (128-byte swizzle), along y/z a row of 32 lines
  int off[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    if (CONTIG)
      off[r] = lane * R + ((r / EPC) ^ (lane & 7)) * EPC + r % EPC;
    else
      off[r] = r * SL + lane;
  }

  auto coords = [&](int tile, int &c0, int &c2) {
    if (CONTIG) {
      c0 = tile * SL;
      c2 = 0;
    } else {
      c2 = tile / tpr;
      c0 = (tile - c2 * tpr) * SL;
    }
  };

  if (fwd) {
    // ------------------------- forward substitution --------------------------
    // Tile ti stores stage g's x2 in TMEM block g (even ti) or NB-1-g (odd
    // ti); the back substitution of the previous tile frees the blocks in the
    // order this tile fills them and publishes prog[cons] = tile * 65536 +
    // steps done.
    long long issued = 0;
    int i_t = 0, i_g = 0, i_c0 = 0, i_c2 = 0;
    auto issue = [&](int slot) {
      if (issued >= total) return;
      if (i_g == 0) coords(gw + i_t * tw, i_c0, i_c2);
      if (lane == 0) {
        F *dst = ring + slot * SE;
        mbar_expect_tx(&full[slot], (unsigned)(SE * sizeof(F)));
        if (CONTIG)
          tma_load_2d_hint(dst, &xmap, &full[slot], i_g * R, i_c0, pol_stream);
        else
          tma_load_3d_hint(dst, &xmap, &full[slot], i_c0, i_g * R, i_c2, pol_stream);
      }
      ++issued;
      if (++i_g == n_stages) {
        i_g = 0;
        ++i_t;
      }
    };
    for (int s = 0; s < ST; ++s) issue(s);

    const V2 *const t_e = reinterpret_cast<const V2 *>(tab);
    const V2 *const t_a = reinterpret_cast<const V2 *>(tab + TR);
    const V2 *const t_inv = reinterpret_cast<const V2 *>(tab + 2 * TR);
    const int free_blocks = NB - n_stages;  // blocks a tile never uses
    int slot = 0, seen = 0, fail = 0, ti = 0;
    unsigned phase = 0;
    long long consumed = 0;
    for (; ti < my_tiles; ++ti) {
      const bool flip = (ti & 1) != 0;
      F p2 = F(0), p1 = F(0);
      for (int g = 0; g < n_stages; ++g) {
        const bool ok = (ti > 0 || wait_table(ready, (g + 1) * R)) &&
                        mbar_wait(&full[slot], phase);
        if (!__all_sync(0xffffffffu, ok)) {
          fail = 1;
          break;
        }
        if (ti == 0) __threadfence_block();  // the table rows just published
        F b[R];
        const F *v = ring + slot * SE;
        if (CONTIG) {  // rows 2j, 2j+1 share a 16-byte chunk
#pragma unroll
          for (int j = 0; j < R / 2; ++j) {
            const V2 pv = *reinterpret_cast<const V2 *>(v + off[2 * j]);
            b[2 * j] = pv.x;
            b[2 * j + 1] = pv.y;
          }
        } else {
#pragma unroll
          for (int r = 0; r < R; ++r) b[r] = v[off[r]];
        }
        fence_async_shared();
        __syncwarp();
        ++consumed;
        issue(slot);  // refill the slot just read
        if (++slot == ST) {
          slot = 0;
          phase ^= 1u;
        }
        const int k0 = g * R;
        if (k0 + R > n) {  // rows past n (zero-filled) contribute nothing
#pragma unroll
          for (int r = 0; r < R; ++r)
            if (k0 + r >= n) b[r] = F(0);
        }
        uint32_t tv[32];
#pragma unroll
        for (int j = 0; j < R / 2; ++j) {
          const V2 ev = t_e[k0 / 2 + j], av = t_a[k0 / 2 + j], iv = t_inv[k0 / 2 + j];
          // y = (b - ds y2 - ddl y1) / dd, with e = ds / dd and a = ddl / dd
          const F y0 = fma(-av.x, p1, fma(-ev.x, p2, b[2 * j] * iv.x));
          const F y1 = fma(-av.y, y0, fma(-ev.y, p1, b[2 * j + 1] * iv.y));
          p2 = y0;
          p1 = y1;
          put_x2<F>(tv, 2 * j, y0);
          put_x2<F>(tv, 2 * j + 1, y1);
        }
        // wait (lane 0, bounded) until the previous tile has read this block
        const int need = (ti - 1) * 65536 + max(0, g + 1 - free_blocks);
        int go = 1;
        if (lane == 0 && seen < need) {
          seen = ld_acquire_shared(&prog[cons]);
          if (seen < need) {
            const unsigned long long t0 = global_ns();
            for (;;) {
              __nanosleep(32);
              seen = ld_acquire_shared(&prog[cons]);
              if (seen >= need) break;
              if (stop[cons] != 0) {
                go = 2;
                break;
              }
              if (global_ns() - t0 > 2000000000ull) {
                go = 0;
                break;
              }
            }
          }
        }
        go = __shfl_sync(0xffffffffu, go, 0);
        if (go != 1) {
          fail = go == 0 ? 1 : 2;
          break;
        }
        tmem_fence_after_sync();
        const int blk = flip ? NB - 1 - g : g;
        tmem_store32(taddr + (uint32_t)(blk * G::kCols), tv);
      }
      if (fail) break;
      tmem_fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(&hfull[ti & 1]);
    }
    if (fail) {
      stop[cons] = 1;
      __syncwarp();
      if (lane == 0) mbar_arrive(&hfull[ti & 1]);  // wake the back substitution
      // drain the loads this warp issued (bounded waits)
      for (; consumed < issued; ++consumed) {
        if (!mbar_wait(&full[slot], phase)) break;
        if (++slot == ST) {
          slot = 0;
          phase ^= 1u;
        }
      }
      if (fail == 1 && lane == 0) atomicOr(status_word, STATUS_TIMEOUT_BIT);
    }
  } else {
    // --------------------------- back substitution ---------------------------
    const V2 *const t_du2 = reinterpret_cast<const V2 *>(tab + 3 * TR);
    const V2 *const t_dw2 = reinterpret_cast<const V2 *>(tab + 4 * TR);
    int o_buf = 0, fail = 0;
    for (int ti = 0; ti < my_tiles; ++ti) {
      int c0, c2;
      coords(gw + ti * tw, c0, c2);
      const int count = CONTIG ? min(SL, n_sys - c0) : min(SL, inner - c0);
      const bool flip = (ti & 1) != 0;
      if (!__all_sync(0xffffffffu, mbar_wait(&hfull[ti & 1], (unsigned)(ti >> 1) & 1u))) {
        fail = 1;
        break;
      }
      if (stop[cons] != 0) {
        fail = 2;
        break;
      }
      tmem_fence_after_sync();
      F s0 = F(0), s1 = F(0);  // x of the two rows below
      for (int g = n_stages - 1; g >= 0; --g) {
        const int k0 = g * R;
        const int blk = flip ? NB - 1 - g : g;
        uint32_t tv[32];
        tmem_load32(taddr + (uint32_t)(blk * G::kCols), tv);
        // the block is free for the next tile's forward substitution
        tmem_fence_before_sync();
        __syncwarp();
        if (lane == 0) st_release_shared(&prog[cons], ti * 65536 + (n_stages - g));
        F xo[R];
#pragma unroll
        for (int j = R / 2 - 1; j >= 0; --j) {
          const V2 uv = t_du2[k0 / 2 + j], wv = t_dw2[k0 / 2 + j];
          const F x1 = fma(-uv.y, s0, fma(-wv.y, s1, get_x2<F>(tv, 2 * j + 1)));
          const F x0 = fma(-uv.x, x1, fma(-wv.x, s0, get_x2<F>(tv, 2 * j)));
          s1 = x1;
          s0 = x0;
          xo[2 * j + 1] = x1;
          xo[2 * j] = x0;
        }
        if (CONTIG) {
          F *const ob = obuf + o_buf * SE;
          if (lane == 0) bulk_wait_read<1>();  // this buffer's previous store has read it
          __syncwarp();
#pragma unroll
          for (int j = 0; j < R / 2; ++j) {
            V2 pv;
            pv.x = xo[2 * j];
            pv.y = xo[2 * j + 1];
            *reinterpret_cast<V2 *>(ob + off[2 * j]) = pv;
          }
          fence_async_shared();
          __syncwarp();
          if (lane == 0) {
            tma_store_2d_hint(&xmap, ob, k0, c0, pol_stream);
            bulk_commit();
          }
          o_buf ^= 1;
        } else if (lane < count) {
          F *const p = x + (long long)c2 * inner * n + c0 + lane;
          if (k0 + R <= n) {
#pragma unroll
            for (int r = 0; r < R; ++r) st_hint(p + (long long)(k0 + r) * inner, xo[r], pol_stream);
          } else {
#pragma unroll
            for (int r = 0; r < R; ++r)
              if (k0 + r < n) st_hint(p + (long long)(k0 + r) * inner, xo[r], pol_stream);
          }
        }
      }
      if (lane == 0) st_release_shared(&prog[cons], (ti + 1) * 65536);
    }
    if (fail) {
      stop[cons] = 1;
      if (fail == 1 && lane == 0) atomicOr(status_word, STATUS_TIMEOUT_BIT);
    }
    if (CONTIG && lane == 0) bulk_wait<0>();
  }
  // the solving warps are done with Tensor Memory: warp 0 frees it
  tmem_fence_before_sync();
  asm volatile("bar.sync 1, %0;\n" ::"n"(64 * NCONS) : "memory");
  tmem_fence_after_sync();
  if (warp == 0) tmem_dealloc(tmem_base, kTmemCols);
}

// ---------------------------------------------------------------------------
// Fallback: table by one thread (into the buffer), then one thread per line
// with x2 in the buffer ([row][line], coalesced across adjacent lines).
// ---------------------------------------------------------------------------
template <typename F>
__global__ void sf_build_table_kernel(const F *__restrict__ ds, const F *__restrict__ dl,
                                      const F *__restrict__ d, const F *__restrict__ du,
                                      const F *__restrict__ dw, F *__restrict__ tab, int n,
                                      long long stride, int *__restrict__ status_word) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const F *arr[5] = {ds, dl, d, du, dw};
  F pu2 = F(0), pu1 = F(0), pw2 = F(0), pw1 = F(0);
  bool bad = false;
  for (int i = 0; i < n; ++i) {
    F c[5];
    for (int q = 0; q < 5; ++q) c[q] = sf_mask<F>(q, i, n, arr[q][(long long)i * stride]);
    const F ddl = c[1] - c[0] * pu2;
    const F dd = c[2] - c[0] * pw2 - ddl * pu1;
    const F inv = F(1) / dd;
    const F du2 = (c[3] - ddl * pw1) * inv;
    const F dw2 = c[4] * inv;
    bad |= !isfinite(inv);
    tab[i] = c[0];
    tab[n + i] = ddl;
    tab[2 * n + i] = inv;
    tab[3 * n + i] = du2;
    tab[4 * n + i] = dw2;
    pu2 = pu1; pu1 = du2;
    pw2 = pw1; pw1 = dw2;
  }
  if (bad) atomicOr(status_word, STATUS_ZERO_PIVOT_BIT);
}

template <typename F>
__global__ void __launch_bounds__(128)
sf_lines_kernel(const F *__restrict__ tab, F *__restrict__ x, F *__restrict__ x2g, Lines L) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= L.n_sys) return;
  const int n = (int)L.n;
  F *const b = x + line_base(L, s);
  F *const x2 = x2g + s;
  const long long st = L.inner;
  F p2 = F(0), p1 = F(0);
  for (int i = 0; i < n; ++i) {
    const F y = (b[i * st] - tab[i] * p2 - tab[n + i] * p1) * tab[2 * n + i];
    p2 = p1;
    p1 = y;
    x2[(long long)i * L.n_sys] = y;
  }
  F s0 = F(0), s1 = F(0);
  for (int i = n - 1; i >= 0; --i) {
    const F xj = x2[(long long)i * L.n_sys] - tab[3 * n + i] * s0 - tab[4 * n + i] * s1;
    s1 = s0;
    s0 = xj;
    b[i * st] = xj;
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
template <typename F>
bool sf_encode(CUtensorMap *m, const F *ptr, const Lines &L, bool contig, int R) {
  auto fn = tensor_map_encoder();
  if (fn == nullptr) return false;
  const CUtensorMapDataType dt =
      sizeof(F) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  CUresult r;
  if (contig) {
    const cuuint64_t dims[2] = {(cuuint64_t)L.n, (cuuint64_t)L.n_sys};
    const cuuint64_t strides[1] = {(cuuint64_t)L.n * sizeof(F)};
    const cuuint32_t box[2] = {(cuuint32_t)R, (cuuint32_t)SL};
    const cuuint32_t es[2] = {1, 1};
    r = fn(m, dt, 2, const_cast<F *>(ptr), dims, strides, box, es,
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  } else {
    const cuuint64_t dims[3] = {(cuuint64_t)L.inner, (cuuint64_t)L.n,
                                (cuuint64_t)(L.n_sys / L.inner)};
    const cuuint64_t strides[2] = {(cuuint64_t)L.inner * sizeof(F),
                                   (cuuint64_t)L.inner * L.n * sizeof(F)};
    const cuuint32_t box[3] = {(cuuint32_t)SL, (cuuint32_t)R, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    r = fn(m, dt, 3, const_cast<F *>(ptr), dims, strides, box, es,
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  }
  return r == CUDA_SUCCESS;
}

long long sf_tiles(const Lines &L, bool contig) {
  return contig ? (L.n_sys + SL - 1) / SL : (L.n_sys / L.inner) * ((L.inner + SL - 1) / SL);
}

template <typename F> size_t sf_cache_bytes(long long n_pad) {
  return 128 + (size_t)10 * n_pad * sizeof(F);
}

template <typename F, bool CONTIG, int ST>
cudaError_t sf_tmem_launch(const SolveArgs<F> &a, int sm_count, size_t usable_buf,
                           cudaStream_t stream) {
  using G = SfGeom<F, CONTIG, ST>;
  CUtensorMap xmap;
  if (!sf_encode<F>(&xmap, a.x, a.L, CONTIG, G::R)) return cudaErrorInvalidValue;
  auto kern = sf_tmem_kernel<F, CONTIG, ST>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)G::kSmem);
  if (err != cudaSuccess) return err;
  const int n = (int)a.L.n;
  const int n_pad = (n + G::R - 1) / G::R * G::R;
  const int inner = (int)a.L.inner;
  const int tpr = CONTIG ? 1 : (inner + SL - 1) / SL;
  const long long n_tiles = sf_tiles(a.L, CONTIG);
  // the table cache sits at the (16-byte aligned) end of the caller's buffer
  unsigned char *cache = nullptr;
  const size_t cb = sf_cache_bytes<F>(n_pad);
  if (a.scratch != nullptr && usable_buf >= cb) {
    const uintptr_t end = reinterpret_cast<uintptr_t>(a.scratch) + usable_buf;
    const uintptr_t start = (end - cb) & ~uintptr_t(127);
    if (start >= reinterpret_cast<uintptr_t>(a.scratch))
      cache = reinterpret_cast<unsigned char *>(start);
  }
  const long long need = (n_tiles + NCONS - 1) / NCONS;
  const int grid = (int)(need < sm_count ? need : sm_count);
  kern<<<grid, 32 * (2 * NCONS + 1), G::kSmem, stream>>>(xmap, a.ds, a.dl, a.d, a.du, a.dw, a.x,
                                                     cache, n, n_pad, inner, tpr,
                                                     (int)a.L.n_sys, (int)n_tiles, a.status);
  return cudaGetLastError();
}

template <typename F, bool CONTIG, int ST> int sf_occ() {
  using G = SfGeom<F, CONTIG, ST>;
  auto kern = sf_tmem_kernel<F, CONTIG, ST>;
  int blocks = 0;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)G::kSmem) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, 32 * (2 * NCONS + 1),
                                                    G::kSmem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return blocks;
}

constexpr int kSfStages = 8;

}  // namespace

template <typename F>
bool sf_tmem_supported(const SolveArgs<F> &a, bool contig, int smem_optin) {
  if (tensor_map_encoder() == nullptr) return false;
  const Lines &L = a.L;
  if (contig) {
    if (L.inner != 1 || (L.n * sizeof(F)) % 16 != 0) return false;
  } else {
    if (L.inner <= 1 || (L.inner * sizeof(F)) % 16 != 0) return false;
  }
  const long long R = sf_rows_per_stage<F>();
  if ((L.n + R - 1) / R * R > sf_max_rows<F>()) return false;  // TMEM capacity
  if (L.n * L.n_sys >= (1LL << 31) || sf_tiles(L, contig) >= (1LL << 31)) return false;
  if (reinterpret_cast<uintptr_t>(a.x) % 16 != 0) return false;
  const size_t smem = contig ? SfGeom<F, true, kSfStages>::kSmem
                             : SfGeom<F, false, kSfStages>::kSmem;
  return smem <= (size_t)smem_optin;
}

template <typename F> int sf_tmem_occupancy(bool contig) {
  return contig ? sf_occ<F, true, kSfStages>() : sf_occ<F, false, kSfStages>();
}

template <typename F>
cudaError_t launch_sf_tmem(const SolveArgs<F> &a, bool contig, int sm_count,
                           size_t usable_buf, cudaStream_t stream) {
  return contig ? sf_tmem_launch<F, true, kSfStages>(a, sm_count, usable_buf, stream)
                : sf_tmem_launch<F, false, kSfStages>(a, sm_count, usable_buf, stream);
}

template <typename F> size_t sf_lines_scratch_bytes(const Lines &L) {
  return ((size_t)L.n * (size_t)L.n_sys + (size_t)5 * L.n) * sizeof(F);
}

template <typename F>
cudaError_t launch_sf_lines(const SolveArgs<F> &a, cudaStream_t stream) {
  F *x2 = static_cast<F *>(a.scratch);
  F *tab = x2 + (size_t)a.L.n * (size_t)a.L.n_sys;
  const long long stride = a.L.inner;
  sf_build_table_kernel<F><<<1, 32, 0, stream>>>(a.ds, a.dl, a.d, a.du, a.dw, tab,
                                                 (int)a.L.n, stride, a.status);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  const long long blocks = (a.L.n_sys + 127) / 128;
  sf_lines_kernel<F><<<(unsigned)blocks, 128, 0, stream>>>(tab, a.x, x2, a.L);
  return cudaGetLastError();
}

template bool sf_tmem_supported<double>(const SolveArgs<double> &, bool, int);
template bool sf_tmem_supported<float>(const SolveArgs<float> &, bool, int);
template int sf_tmem_occupancy<double>(bool);
template int sf_tmem_occupancy<float>(bool);
template cudaError_t launch_sf_tmem<double>(const SolveArgs<double> &, bool, int, size_t,
                                            cudaStream_t);
template cudaError_t launch_sf_tmem<float>(const SolveArgs<float> &, bool, int, size_t,
                                           cudaStream_t);
template size_t sf_lines_scratch_bytes<double>(const Lines &);
template size_t sf_lines_scratch_bytes<float>(const Lines &);
template cudaError_t launch_sf_lines<double>(const SolveArgs<double> &, cudaStream_t);
template cudaError_t launch_sf_lines<float>(const SolveArgs<float> &, cudaStream_t);

}  // namespace penta
