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
// The Tensor-Memory kernel (aligned lines, n <= 512 in FP64, n <= 1024 in FP32):
//  * every line is split into an upper half (rows [0, m), eliminated
//    downwards with the table of line 0's top rows) and a lower half (rows
//    [m, n), eliminated upwards on the mirrored band with a second table built
//    from the bottom, after 2m - n identity rows), m = R ceil(n / 2R); the
//    halves meet in the same 4x4 interface solve as the general kernels
//    (penta_device.cuh) and substitute back towards their own ends.
//  * one CTA per SM: for each TMEM lane quarter c, warp c runs the forward
//    substitution and warp 4 + c the back substitution of the same tiles, one
//    tile behind; warp 8 builds the tables.  A tile is 16 lines: lanes 0-15
//    take their upper halves, lanes 16-31 their lower halves.  The forward
//    warp streams the right-hand sides through a ring of TMA tiles {R rows x
//    16 lines} per half (along x: 128-byte rows, 128-byte swizzle, read in row
//    pairs) that it refills itself and keeps x2 of every row in its TMEM lane
//    quarter (one tcgen05.st of 32 columns per stage); the back substitution
//    reads it back and writes x through a shared tile and one TMA store per
//    half and step.  Consecutive tiles fill TMEM blocks in opposite orders and
//    a progress word hands blocks over, as in tmem_kernels.cu.  HBM traffic is
//    the algorithmic 2 x sizeof(F) per point; loads and stores carry an
//    evict-first L2 policy.
//  * The builder warp gathers line 0's coefficients (issued at kernel entry,
//    ahead of the ring loads), masks them and runs the two serial recurrences
//    (lanes 0 and 1, in lockstep) into shared-memory tables, publishing them R
//    rows at a time; forward warps on their first tile follow them.
//  * The tables are cached at the end of the caller's buffer together with the
//    coefficients they came from.  When a later call finds its line-0
//    coefficients identical, bit for bit, to the cached ones, the builder
//    copies the tables instead of recomputing them (e.g. the 50 iterations of
//    an ADI run); otherwise it recomputes and refreshes the cache.  The result
//    is the same either way.
//
// Other shapes use a one-thread-per-line kernel with x2 in the caller's buffer
// and a table built by a single-thread kernel, as in the reference.
#include <cstdlib>
#include <type_traits>

#include "penta_internal.hpp"
#include "tma_device.cuh"

namespace penta {
namespace {

constexpr int TS = 16;              // lines per tile; lanes 0-15 the upper halves, 16-31 the lower
constexpr int NCONS = 4;            // lane quarters: one forward and one back-substitution warp each
constexpr uint32_t kTmemCols = 512;
// cache layout [inputs 5 x 2m | upper table 5 x m | lower table 5 x m], tables [e|a|inv|du2|dw2]
constexpr int kCacheMagic = 0x5f4a4356;

// A stage is R = 16 (FP64) / 32 (FP32) rows of each half, 128 bytes of a line
// along x (TMA tiles {R rows, 16 lines}, 128-byte swizzle), 32 TMEM columns.
template <typename F> constexpr int sf_rows_per_stage() { return 128 / (int)sizeof(F); }

// TMEM holds x2 of a half line: m <= 256 rows (FP64, 2 columns a row) / 512 (FP32).
template <typename F> constexpr int sf_max_half() {
  return (int)kTmemCols / ((int)sizeof(F) / 4);
}

template <typename F, bool CONTIG, int ST> struct SfGeom {
  static constexpr int R = sf_rows_per_stage<F>();
  static constexpr int BOX = R * TS;                      // one half's tile
  static constexpr int SE = 2 * BOX;                      // a stage: both halves
  static constexpr int OBE = 2 * SE;                      // output tiles (2 buffers)
  static constexpr int HE = 2 * 2 * 32;                   // carries y1, y2: 2 slots
  static constexpr size_t kData = (size_t)(ST * SE + OBE + HE) * sizeof(F);
  static constexpr size_t kCons = (kData + (ST + 2) * 8 + 1023) / 1024 * 1024;
  static constexpr int TR = sf_max_half<F>();             // table rows per half
  // line-0 inputs (rows < 2m) and the two tables
  static constexpr size_t kTable = (size_t)20 * TR * sizeof(F);
  static constexpr size_t kUsed = NCONS * kCons + kTable + 128 + 1024;
  // at least 116 KB, so that one CTA holds an SM (and all of its TMEM)
  static constexpr size_t kSmem = kUsed > 118784 ? kUsed : 118784;
  static constexpr int kCols = R * (int)sizeof(F) / 4;    // TMEM columns per stage (32)
  static constexpr int NB = (int)kTmemCols / kCols;       // TMEM blocks of one stage each
  static_assert(kCols == 32, "32 TMEM columns per stage");
  static_assert(kSmem <= 232448, "shared memory per CTA");
};

// The cache at the end of the caller's buffer:
// [header 128 B][inputs 5 x 2m][upper table 5 x m][lower table 5 x m].
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
               int n, int mt, int inner, int tpr, int n_sys, int n_tiles,
               int *__restrict__ status_word) {
  using G = SfGeom<F, CONTIG, ST>;
  using V2 = typename Vec2<F>::T;
  constexpr int R = G::R, BOX = G::BOX, SE = G::SE, NB = G::NB, TR = G::TR;
  constexpr int EPC = 16 / (int)sizeof(F);
  constexpr int kMirror[5] = {4, 3, 2, 1, 0};

  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *const base =
      smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const int warp = threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  F *const coef = reinterpret_cast<F *>(base + NCONS * G::kCons);  // line-0 inputs [5][2 TR]
  F *const tup = coef + 10 * TR;                                    // upper table [5][TR]
  F *const tdn = tup + 5 * TR;                                      // lower table [5][TR]
  unsigned char *const tail = base + NCONS * G::kCons + G::kTable;
  uint32_t *const tmem_slot = reinterpret_cast<uint32_t *>(tail);
  volatile int *const ready = reinterpret_cast<volatile int *>(tail + 16);
  volatile int *const stop = reinterpret_cast<volatile int *>(tail + 32);  // [NCONS]
  uint64_t *const cbar = reinterpret_cast<uint64_t *>(tail + 64);
  int *const prog = reinterpret_cast<int *>(tail + 96);                    // [NCONS]
  const int n2 = 2 * mt;          // rows of line 0 kept (rows >= n are zeros)
  const int nv = n2 - n;          // virtual rows ahead of the lower half's first real row

  // The builder warp starts first: the table cache's bulk copies and the
  // first round of the line-0 gather (every load of a lane issued before any
  // is used; rows lane + 32 j of each array, next to the cached inputs they
  // are compared with) go out before the solving warps' ring loads.
  constexpr int JB = 32 / (int)sizeof(F);  // rows per lane per gather round
  const bool builder = warp == 2 * NCONS;
  const long long stride = CONTIG ? 1 : inner;  // line 0's row stride
  SfCacheHeader *const hdr = reinterpret_cast<SfCacheHeader *>(cache);
  F *const c_in = cache ? reinterpret_cast<F *>(cache + 128) : nullptr;
  F *const c_up = c_in ? c_in + 5 * (long long)n2 : nullptr;
  F *const c_dn = c_up ? c_up + 5 * (long long)mt : nullptr;
  const F *const src[5] = {ds, dl, d, du, dw};
  F v[5][JB], w[5][JB];
  bool same = cache != nullptr;
  auto gather = [&](int j0) {  // rows lane + 32 (j0 + j), j < JB
#pragma unroll
    for (int q = 0; q < 5; ++q)
#pragma unroll
      for (int j = 0; j < JB; ++j) {
        const int i = lane + 32 * (j0 + j);
        v[q][j] = i < n ? src[q][(long long)i * stride] : F(0);
        w[q][j] = (cache != nullptr && i < n2) ? c_in[(long long)q * n2 + i] : F(0);
      }
  };
  auto keep = [&](int j0) {  // masked into shared memory, and compared with the cache
#pragma unroll
    for (int q = 0; q < 5; ++q)
#pragma unroll
      for (int j = 0; j < JB; ++j) {
        const int i = lane + 32 * (j0 + j);
        if (i < n2) {
          const F c = sf_mask<F>(q, i, n, v[q][j]);
          coef[q * 2 * TR + i] = c;
          same = same && same_bits(c, w[q][j]);
        }
      }
  };
  // Programmatic dependent launch: the next solve on the stream may start its
  // on-chip prologue on SMs this grid has left; every global access of this
  // grid comes after griddepcontrol.wait (the previous grid complete and its
  // writes visible) -- the builder's before its first read, the others' after
  // the prologue.
  if (threadIdx.x == 0) asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  if (builder) {
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
    if (cache != nullptr && lane == 0) {
      const unsigned comp = (unsigned)(mt * sizeof(F));
      mbar_init(cbar, 1);
      mbar_init_fence();
      mbar_expect_tx(cbar, 10u * comp);
      for (int q = 0; q < 5; ++q) {
        bulk_load(tup + q * TR, c_up + (long long)q * mt, comp, cbar);
        bulk_load(tdn + q * TR, c_dn + (long long)q * mt, comp, cbar);
      }
    }
    gather(0);
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
  if (!builder) asm volatile("griddepcontrol.wait;\n" ::: "memory");

  // ================================ builder =================================
  if (builder) {
    keep(0);
    for (int j0 = JB; 32 * j0 < n2; j0 += JB) {
      gather(j0);
      keep(j0);
    }
    bool copies_done = true;
    if (cache != nullptr) copies_done = __all_sync(0xffffffffu, mbar_wait(cbar, 0));
    if (!copies_done) {  // the table area may still be written: publish nothing
      if (lane == 0) atomicOr(status_word, STATUS_TIMEOUT_BIT);
      return;
    }
    __syncwarp();
    if (__all_sync(0xffffffffu, same)) {  // cached tables: already in place
      __threadfence_block();
      __syncwarp();
      if (lane == 0) *ready = mt;
      return;
    }
    // lane 0 runs the upper recurrence (rows 0 .. m-1 downwards), lane 1 the
    // lower one (rows n-1 .. m upwards on the mirrored band, after nv
    // identity rows), in lockstep, publishing R rows of both at a time
    if (lane < 2) {
      F *const t = lane ? tdn : tup;
      F pu2 = F(0), pu1 = F(0), pw2 = F(0), pw1 = F(0);
      bool bad = false;
      for (int k = 0; k < mt; ++k) {
        F c[5];
        if (lane == 0) {
#pragma unroll
          for (int q = 0; q < 5; ++q) c[q] = coef[q * 2 * TR + k];
        } else if (k < nv) {
          c[0] = c[1] = c[3] = c[4] = F(0);
          c[2] = F(1);
        } else {
          const int i = n2 - 1 - k;  // the original row
#pragma unroll
          for (int q = 0; q < 5; ++q) c[q] = coef[kMirror[q] * 2 * TR + i];
        }
        const F ddl = c[1] - c[0] * pu2;
        const F dd = c[2] - c[0] * pw2 - ddl * pu1;
        const F inv = F(1) / dd;
        const F du2 = (c[3] - ddl * pw1) * inv;
        const F dw2 = c[4] * inv;
        bad |= !isfinite(inv);
        t[k] = c[0] * inv;       // e
        t[TR + k] = ddl * inv;   // a
        t[2 * TR + k] = inv;
        t[3 * TR + k] = du2;
        t[4 * TR + k] = dw2;
        pu2 = pu1; pu1 = du2;
        pw2 = pw1; pw1 = dw2;
        if ((k + 1) % R == 0) {
          __threadfence_block();
          __syncwarp(0x3u);
          if (lane == 0) *ready = k + 1;
        }
      }
      if (bad) atomicOr(status_word, STATUS_ZERO_PIVOT_BIT);
    }
    __syncwarp();
    // refresh the cache (CTA 0): header cleared, tables, inputs, then the header
    if (cache != nullptr && blockIdx.x == 0) {
      if (lane == 0) hdr->magic = 0;
      __threadfence();
      __syncwarp();
      for (int k = lane; k < 5 * mt; k += 32) {
        const int q = k / mt, i = k - q * mt;
        c_up[k] = tup[q * TR + i];
        c_dn[k] = tdn[q * TR + i];
      }
      for (int k = lane; k < 5 * n2; k += 32) {
        const int q = k / n2, i = k - q * n2;
        c_in[k] = coef[q * 2 * TR + i];
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
  const int sys = lane % TS;
  const int part = lane / TS;  // 0: upper half, 1: lower half (mirrored)
  F *const ring = reinterpret_cast<F *>(base + cons * G::kCons);
  F *const obuf = ring + ST * SE;
  F *const hand = obuf + G::OBE;  // [2 slots][y1, y2][32 lanes]
  uint64_t *const full = reinterpret_cast<uint64_t *>(base + cons * G::kCons + G::kData);
  uint64_t *const hfull = full + ST;  // [2]: a tile's x2 is in TMEM
  const uint32_t taddr = tmem_base + ((uint32_t)(cons * 32) << 16);
  const int n_stages = mt / R;
  const int gw = blockIdx.x * NCONS + cons;
  const int tw = gridDim.x * NCONS;
  const int my_tiles = gw < n_tiles ? (n_tiles - 1 - gw) / tw + 1 : 0;
  const long long total = (long long)my_tiles * n_stages;
  const uint64_t pol_stream = l2_policy_first();  // every access is read or written once
  const F *const th = part ? tdn : tup;           // this half's table

  auto coords = [&](int tile, int &c0, int &c2) {
    if (CONTIG) {
      c0 = tile * TS;
      c2 = 0;
    } else {
      c2 = tile / tpr;
      c0 = (tile - c2 * tpr) * TS;
    }
  };

  if (fwd) {
    // ------------------------- forward substitution --------------------------
    // Tile ti stores stage g's x2 in TMEM block g (even ti) or NB-1-g (odd
    // ti); the back substitution of the previous tile frees the blocks in the
    // order this tile fills them and publishes prog[cons] = tile * 65536 +
    // steps done.
    // element offset, in a stage, of this lane's row r (strided), or of the
    // 16-byte chunk holding its rows 2j and 2j+1 (along x, read in pairs)
    int ld[CONTIG ? R / 2 : R];
    if constexpr (CONTIG) {
#pragma unroll
      for (int j = 0; j < R / 2; ++j) {
        const int e = part ? (R - 2 - 2 * j) : 2 * j;  // the pair's even row in the tile
        ld[j] = part * BOX + sys * R + ((e / EPC) ^ (sys & 7)) * EPC + e % EPC;
      }
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) ld[r] = part * BOX + (part ? (R - 1 - r) : r) * TS + sys;
    }
    long long issued = 0;
    int i_t = 0, i_g = 0, i_c0 = 0, i_c2 = 0;
    auto issue = [&](int slot) {
      if (issued >= total) return;
      if (i_g == 0) coords(gw + i_t * tw, i_c0, i_c2);
      if (lane == 0) {
        F *dst = ring + slot * SE;
        const int r_up = i_g * R, r_dn = n2 - (i_g + 1) * R;
        const bool lower = r_dn < n;  // else all of the lower tile is virtual
        mbar_expect_tx(&full[slot], (unsigned)((lower ? 2 : 1) * BOX * sizeof(F)));
        if (CONTIG) {
          tma_load_2d_hint(dst, &xmap, &full[slot], r_up, i_c0, pol_stream);
          if (lower) tma_load_2d_hint(dst + BOX, &xmap, &full[slot], r_dn, i_c0, pol_stream);
        } else {
          tma_load_3d_hint(dst, &xmap, &full[slot], i_c0, r_up, i_c2, pol_stream);
          if (lower)
            tma_load_3d_hint(dst + BOX, &xmap, &full[slot], i_c0, r_dn, i_c2, pol_stream);
        }
      }
      ++issued;
      if (++i_g == n_stages) {
        i_g = 0;
        ++i_t;
      }
    };
    for (int s = 0; s < ST; ++s) issue(s);

    const V2 *const t_e = reinterpret_cast<const V2 *>(th);
    const V2 *const t_a = reinterpret_cast<const V2 *>(th + TR);
    const V2 *const t_inv = reinterpret_cast<const V2 *>(th + 2 * TR);
    const int nvp = part ? nv : 0;  // this half's virtual rows
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
        const F *vs = ring + slot * SE;
        if constexpr (CONTIG) {  // the lower half reads its tile backwards
#pragma unroll
          for (int j = 0; j < R / 2; ++j) {
            const V2 pv = *reinterpret_cast<const V2 *>(vs + ld[j]);
            b[2 * j] = part ? pv.y : pv.x;
            b[2 * j + 1] = part ? pv.x : pv.y;
          }
        } else {
#pragma unroll
          for (int r = 0; r < R; ++r) b[r] = vs[ld[r]];
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
        if (k0 < nvp) {  // virtual rows (their tile may not have been loaded)
#pragma unroll
          for (int r = 0; r < R; ++r)
            if (k0 + r < nvp) b[r] = F(0);
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
      // this half's last two y values go to the back substitution
      F *const h = hand + (ti & 1) * 64 + lane;
      h[0] = p1;
      h[32] = p2;
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
    // offset, in a half's output tile, of the chunk holding this lane's rows
    // 2j and 2j+1 of a step (back substitution order), along x
    int st2[R / 2];
#pragma unroll
    for (int j = 0; j < R / 2; ++j) {
      const int rr = part ? 2 * j : (R - 2 - 2 * j);
      st2[j] = CONTIG ? part * BOX + sys * R + ((rr / EPC) ^ (sys & 7)) * EPC + rr % EPC : 0;
    }
    const V2 *const t_du2 = reinterpret_cast<const V2 *>(th + 3 * TR);
    const V2 *const t_dw2 = reinterpret_cast<const V2 *>(th + 4 * TR);
    int o_buf = 0, fail = 0;
    for (int ti = 0; ti < my_tiles; ++ti) {
      int c0, c2;
      coords(gw + ti * tw, c0, c2);
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
      // ---- interface: rows m-2, m-1 (upper) and m, m+1 (lower) of each line.
      // The factors of the last two rows of each half are the same for every
      // line; read only now: the hand-over above orders these reads after the
      // forward warp saw the finished table
      const F uu1 = tup[3 * TR + mt - 1], uu2 = tup[3 * TR + mt - 2];
      const F uw1 = tup[4 * TR + mt - 1], uw2 = tup[4 * TR + mt - 2];
      const F lu1 = tdn[3 * TR + mt - 1], lu2 = tdn[3 * TR + mt - 2];
      const F lw1 = tdn[4 * TR + mt - 1], lw2 = tdn[4 * TR + mt - 2];
      const F *const h = hand + (ti & 1) * 64 + lane;
      const F y1 = h[0], y2 = h[32];
      const F py1 = __shfl_xor_sync(0xffffffffu, y1, TS);
      const F py2 = __shfl_xor_sync(0xffffffffu, y2, TS);
      F u0, u1, u2, u3;
      if (part == 0)
        solve_interface(uu2, uw2, y2, uu1, uw1, y1, lu1, lw1, py1, lu2, lw2, py2, u0, u1, u2,
                        u3);
      else
        solve_interface(uu2, uw2, py2, uu1, uw1, py1, lu1, lw1, y1, lu2, lw2, y2, u0, u1, u2,
                        u3);
      F xa = part ? u1 : u2;  // x of the row just past this half's last row
      F xb = part ? u0 : u3;  // and of the one after it
      for (int g = n_stages - 1; g >= 0; --g) {
        const int k0 = g * R;
        const int blk = flip ? NB - 1 - g : g;
        uint32_t tv[32];
        tmem_load32(taddr + (uint32_t)(blk * G::kCols), tv);
        // the block is free for the next tile's forward substitution
        tmem_fence_before_sync();
        __syncwarp();
        if (lane == 0) st_release_shared(&prog[cons], ti * 65536 + (n_stages - g));
        F xo[R];  // back-substitution order: xo[r] is elimination row k0 + R - 1 - r
#pragma unroll
        for (int j = R / 2 - 1; j >= 0; --j) {
          const V2 uv = t_du2[k0 / 2 + j], wv = t_dw2[k0 / 2 + j];
          const F xh = fma(-uv.y, xa, fma(-wv.y, xb, get_x2<F>(tv, 2 * j + 1)));
          const F xl = fma(-uv.x, xh, fma(-wv.x, xa, get_x2<F>(tv, 2 * j)));
          xb = xh;
          xa = xl;
          xo[R - 2 - 2 * j] = xh;
          xo[R - 1 - 2 * j] = xl;
        }
        // elimination row k is row k (upper half) or n2 - 1 - k (lower half);
        // the step's results leave as one TMA tile per half (rows past n and
        // lines past the grid are not written)
        F *const ob = obuf + o_buf * SE;
        if (lane == 0) bulk_wait_read<1>();  // this buffer's previous stores have read it
        __syncwarp();
        if (CONTIG) {
#pragma unroll
          for (int j = 0; j < R / 2; ++j) {
            V2 pv;
            pv.x = part ? xo[2 * j] : xo[2 * j + 1];
            pv.y = part ? xo[2 * j + 1] : xo[2 * j];
            *reinterpret_cast<V2 *>(ob + st2[j]) = pv;
          }
        } else {
#pragma unroll
          for (int r = 0; r < R; ++r) ob[part * BOX + (part ? r : R - 1 - r) * TS + sys] = xo[r];
        }
        fence_async_shared();
        __syncwarp();
        if (lane == 0) {
          const bool lower = n2 - k0 - R < n;  // else all of the lower tile is virtual
          if (CONTIG) {
            tma_store_2d_hint(&xmap, ob, k0, c0, pol_stream);
            if (lower) tma_store_2d_hint(&xmap, ob + BOX, n2 - k0 - R, c0, pol_stream);
          } else {
            tma_store_3d_hint(&xmap, ob, c0, k0, c2, pol_stream);
            if (lower) tma_store_3d_hint(&xmap, ob + BOX, c0, n2 - k0 - R, c2, pol_stream);
          }
          bulk_commit();
        }
        o_buf ^= 1;
      }
      if (lane == 0) st_release_shared(&prog[cons], (ti + 1) * 65536);
    }
    if (fail) {
      stop[cons] = 1;
      if (fail == 1 && lane == 0) atomicOr(status_word, STATUS_TIMEOUT_BIT);
    }
    if (lane == 0) bulk_wait<0>();
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
    const cuuint32_t box[2] = {(cuuint32_t)R, (cuuint32_t)TS};
    const cuuint32_t es[2] = {1, 1};
    r = fn(m, dt, 2, const_cast<F *>(ptr), dims, strides, box, es,
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  } else {
    const cuuint64_t dims[3] = {(cuuint64_t)L.inner, (cuuint64_t)L.n,
                                (cuuint64_t)(L.n_sys / L.inner)};
    const cuuint64_t strides[2] = {(cuuint64_t)L.inner * sizeof(F),
                                   (cuuint64_t)L.inner * L.n * sizeof(F)};
    const cuuint32_t box[3] = {(cuuint32_t)TS, (cuuint32_t)R, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    r = fn(m, dt, 3, const_cast<F *>(ptr), dims, strides, box, es,
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  }
  return r == CUDA_SUCCESS;
}

long long sf_tiles(const Lines &L, bool contig) {
  return contig ? (L.n_sys + TS - 1) / TS : (L.n_sys / L.inner) * ((L.inner + TS - 1) / TS);
}

// m = R ceil(n / 2R): rows per half (the lower half padded with 2m - n virtual rows)
template <typename F> long long sf_split(long long n) {
  const long long R = sf_rows_per_stage<F>();
  return (n + 2 * R - 1) / (2 * R) * R;
}

template <typename F> size_t sf_cache_bytes(long long mt) {
  return 128 + (size_t)20 * mt * sizeof(F);  // inputs 5 x 2m, two tables 5 x m
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
  const int mt = (int)sf_split<F>(n);
  const int inner = (int)a.L.inner;
  const int tpr = CONTIG ? 1 : (inner + TS - 1) / TS;
  const long long n_tiles = sf_tiles(a.L, CONTIG);
  // the table cache sits at the (16-byte aligned) end of the caller's buffer
  unsigned char *cache = nullptr;
  const size_t cb = sf_cache_bytes<F>(mt);
  if (a.scratch != nullptr && usable_buf >= cb) {
    const uintptr_t end = reinterpret_cast<uintptr_t>(a.scratch) + usable_buf;
    const uintptr_t start = (end - cb) & ~uintptr_t(127);
    if (start >= reinterpret_cast<uintptr_t>(a.scratch))
      cache = reinterpret_cast<unsigned char *>(start);
  }
  const long long need = (n_tiles + NCONS - 1) / NCONS;
  const int grid = (int)(need < sm_count ? need : sm_count);
  // programmatic stream serialization: see the kernel's griddepcontrol.wait
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(32 * (2 * NCONS + 1));
  cfg.dynamicSmemBytes = G::kSmem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  err = cudaLaunchKernelEx(&cfg, kern, xmap, a.ds, a.dl, a.d, a.du, a.dw, a.x, cache, n, mt,
                           inner, tpr, (int)a.L.n_sys, (int)n_tiles, a.status);
  if (err != cudaSuccess) return err;
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
  const long long mt = sf_split<F>(L.n);
  if (mt > sf_max_half<F>() || L.n - mt < 2) return false;  // TMEM capacity; two rows a half
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
