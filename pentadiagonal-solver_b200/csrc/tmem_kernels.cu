// tmem_kernels.cu -- batched Thomas for all three directions with the
// factors held in Tensor Memory.
//
// Algorithm (as tiled_kernels.cu with P = 2): a consumer warp owns tiles of 16
// systems.  Lanes 0..15 eliminate the upper rows [0, m) of their system
// downwards, lanes 16..31 the lower rows [m, n) upwards on the mirrored band
// (dw, du, d, dl, ds), the halves meet in a 4x4 interface solve done with warp
// shuffles, and each half substitutes back towards its own end.
//
// m = R ceil(n / 2R) is a multiple of the rows per stage R, and the lower half
// is extended by v = 2m - n virtual rows ahead of its first real row (rows
// n .. n+v-1 of the mirrored sweep): identity rows (d = 1, everything else 0)
// whose factors are exact zeros, so the carries reach the first real row as
// exact zeros, as if the sweep had started there.  Both halves then run m
// rows in lockstep: every stage is full and every offset below is the same
// for both halves.
//
// Per CTA (one per SM): warps 0..3 compute, warps 4..7 feed them.
//  * Producer warp 4 + c fills consumer c's ring of ST stages.  A stage is 12
//    TMA tiles (6 arrays x 2 halves) of R rows x 16 systems on one mbarrier;
//    the lower half's tiles come from the mirrored arrays.  The consumer
//    copies a stage into registers and releases the slot at once.
//  * The factors du2, dw2 of every row go to Tensor Memory with one
//    tcgen05.st of 32 columns per stage (consumer c uses TMEM lanes
//    32c..32c+31, the lane quarter its warp can reach; FP64 rows take 4
//    columns, FP32 rows 2).  512 columns hold m <= 16 R rows: n <= 256 in
//    FP64, n <= 512 in FP32.  They come back with one tcgen05.ld per stage.
//  * x2 makes an L2 round trip through the caller's buffer ([tile][half][m]
//    [16]), written once per row and read back, most recent first, by two
//    bulk copies per stage into a small ring; each 128-byte line is dropped
//    from L2 (discard.global.L2) once read, so it never reaches HBM.
//  * Output: strided directions store x directly (16 consecutive systems are
//    one 128-byte segment).  Along x, a lane's rows are contiguous in memory:
//    the R results per half go into a 64-byte-swizzled shared tile (the layout
//    of the loads) and leave as TMA tile stores.
//
// Tensor views: along x {n, n_sys} with tiles {R, 16} (64-byte rows, 64-byte
// swizzle); strided {inner, n, outer} with tiles {16, R, 1}.  TMA needs
// 16-byte aligned bases and row strides and 16-byte aligned innermost
// coordinates: n * sizeof(F) % 16 == 0 along x (every row coordinate used is
// a multiple of R), inner * sizeof(F) % 16 == 0 for the strided views.
//
// Waits are bounded (tma_device.cuh).  A wait that runs out raises
// STATUS_TIMEOUT_BIT; the consumer stops its producer, drains the copies in
// flight into its buffers (again bounded) and the CTA frees its TMEM before
// returning.  A zero or non-finite pivot turns the carries into NaN or
// infinity, which is checked once per tile (STATUS_ZERO_PIVOT_BIT).
#include <cstdlib>
#include <cstring>
#include <type_traits>

#include "penta_internal.hpp"
#include "tma_device.cuh"

namespace penta {
namespace {

constexpr int TS = 16;              // systems per tile
constexpr int NCONS = 4;            // consumer warps per CTA, one per TMEM lane quarter
constexpr uint32_t kTmemCols = 512; // the whole of Tensor Memory
constexpr int kColsPerStage = 32;

template <typename F, bool CONTIG> constexpr int tmem_rows_per_stage() {
  return CONTIG ? 64 / (int)sizeof(F) : 1024 / (TS * (int)sizeof(F));
}

template <typename F, bool CONTIG, int ST, int XST> struct TmemGeom {
  static constexpr int R = tmem_rows_per_stage<F, CONTIG>();
  static constexpr int BOX = R * TS;                 // elements per TMA tile
  static constexpr int SE = 12 * BOX;                // forward stage
  static constexpr int XE = 2 * R * TS;              // x2 read-back stage
  static constexpr int OBE = CONTIG ? 4 * BOX : 0;   // output tiles: 2 buffers x 2 halves
  static constexpr size_t kData = (size_t)(ST * SE + XST * XE + OBE) * sizeof(F);
  static constexpr size_t kBars = (size_t)(2 * ST + XST) * 8;
  static constexpr size_t kCons = (kData + kBars + 1023) / 1024 * 1024;
  static constexpr size_t kTail = 64;                // TMEM address + stop flags
  static constexpr size_t kUsed = NCONS * kCons + kTail + 1024;  // + alignment slack
  // at least 116 KB, so that one CTA holds an SM (and all of its TMEM)
  static constexpr size_t kSmem = kUsed > 118784 ? kUsed : 118784;
  static_assert(R * (2 * (int)sizeof(F) / 4) == kColsPerStage, "32 TMEM columns per stage");
};

template <typename F> __device__ __forceinline__ void pack_factors(uint32_t (&tv)[32], int r,
                                                                  F u, F w);
template <> __device__ __forceinline__ void pack_factors<double>(uint32_t (&tv)[32], int r,
                                                                 double u, double w) {
  tv[4 * r + 0] = (uint32_t)__double2loint(u);
  tv[4 * r + 1] = (uint32_t)__double2hiint(u);
  tv[4 * r + 2] = (uint32_t)__double2loint(w);
  tv[4 * r + 3] = (uint32_t)__double2hiint(w);
}
template <> __device__ __forceinline__ void pack_factors<float>(uint32_t (&tv)[32], int r,
                                                                float u, float w) {
  tv[2 * r + 0] = __float_as_uint(u);
  tv[2 * r + 1] = __float_as_uint(w);
}
template <typename F> __device__ __forceinline__ void unpack_factors(const uint32_t (&tv)[32],
                                                                    int r, F &u, F &w);
template <> __device__ __forceinline__ void unpack_factors<double>(const uint32_t (&tv)[32],
                                                                   int r, double &u,
                                                                   double &w) {
  u = __hiloint2double((int)tv[4 * r + 1], (int)tv[4 * r + 0]);
  w = __hiloint2double((int)tv[4 * r + 3], (int)tv[4 * r + 2]);
}
template <> __device__ __forceinline__ void unpack_factors<float>(const uint32_t (&tv)[32],
                                                                  int r, float &u, float &w) {
  u = __uint_as_float(tv[2 * r + 0]);
  w = __uint_as_float(tv[2 * r + 1]);
}

template <typename F, bool CONTIG, int ST, int XST>
__global__ void __launch_bounds__(64 * NCONS, 1)
tmem_thomas_kernel(const __grid_constant__ TmaMaps maps, F *__restrict__ x,
                   F *__restrict__ scratch, int n, int mt, int inner, int tpr, int n_sys,
                   int n_tiles, int flags, int *__restrict__ status_word) {
  using G = TmemGeom<F, CONTIG, ST, XST>;
  constexpr int R = G::R, BOX = G::BOX, SE = G::SE, XE = G::XE;
  constexpr int EPC = 16 / (int)sizeof(F);  // elements per 16-byte chunk
  constexpr int kMirror[6] = {4, 3, 2, 1, 0, 5};

  extern __shared__ __align__(128) unsigned char smem_raw[];
  // swizzled tiles need 1 KB aligned destinations; the launch adds 1 KB slack
  unsigned char *const base =
      smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const int warp = threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  const int cons = warp % NCONS;  // the consumer this warp is, or feeds
  auto region = [&](int c) { return base + c * G::kCons; };
  F *const ring = reinterpret_cast<F *>(region(cons));
  F *const xr = ring + ST * SE;    // x2 read-back stages [XST][2 halves][R][16]
  F *const obuf = xr + XST * XE;   // along x: [2 buffers][2 halves][BOX]
  uint64_t *const full = reinterpret_cast<uint64_t *>(region(cons) + G::kData);
  uint64_t *const empty = full + ST;
  uint64_t *const rfull = empty + ST;
  uint32_t *const tmem_slot = reinterpret_cast<uint32_t *>(base + NCONS * G::kCons);
  volatile int *const stop = reinterpret_cast<volatile int *>(tmem_slot + 4);  // [NCONS]

  const int n_stages = mt / R;
  const int nv = 2 * mt - n;  // virtual rows ahead of the lower half's first real row
  const int gw = blockIdx.x * NCONS + cons;
  const int tw = gridDim.x * NCONS;
  const int my_tiles = gw < n_tiles ? (n_tiles - 1 - gw) / tw + 1 : 0;

  if (threadIdx.x == 0) {
    for (int c = 0; c < NCONS; ++c) {
      uint64_t *f = reinterpret_cast<uint64_t *>(region(c) + G::kData);
      for (int s = 0; s < 2 * ST + XST; ++s) mbar_init(&f[s], 1);
      stop[c] = 0;
    }
    mbar_init_fence();
  }
  if (warp == 0) tmem_alloc(tmem_slot, kTmemCols);
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  const uint32_t tmem_base = *tmem_slot;

  auto tile_coords = [&](int tile, int &c0, int &c2) {
    if (CONTIG) {
      c0 = tile * TS;  // first system
      c2 = 0;
    } else {
      c2 = tile / tpr;  // run
      c0 = (tile - c2 * tpr) * TS;
    }
  };

  // ================================ producer ================================
  if (warp >= NCONS) {
    if (lane != 0) return;
    int slot = 0, use = 0;
    for (int ti = 0; ti < my_tiles; ++ti) {
      int c0, c2;
      tile_coords(gw + ti * tw, c0, c2);
      for (int g = 0; g < n_stages; ++g) {
        if (use > 0 && !mbar_wait(&empty[slot], (unsigned)(use - 1) & 1u)) {
          atomicOr(status_word, STATUS_TIMEOUT_BIT);
          return;
        }
        if (stop[cons]) return;
        const int r_up = g * R;
        const int r_dn = 2 * mt - (g + 1) * R;  // lower half, virtual rows included
        const bool lower = r_dn < n;            // else all rows are virtual: not loaded
        mbar_expect_tx(&full[slot], (lower ? 12u : 6u) * BOX * (unsigned)sizeof(F));
        F *dst = ring + slot * SE;
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          if (CONTIG) {
            tma_load_2d(dst + (2 * q) * BOX, &maps.m[q], &full[slot], r_up, c0);
            if (lower)
              tma_load_2d(dst + (2 * q + 1) * BOX, &maps.m[kMirror[q]], &full[slot], r_dn,
                          c0);
          } else {
            tma_load_3d(dst + (2 * q) * BOX, &maps.m[q], &full[slot], c0, r_up, c2);
            if (lower)
              tma_load_3d(dst + (2 * q + 1) * BOX, &maps.m[kMirror[q]], &full[slot], c0,
                          r_dn, c2);
          }
        }
        if (++slot == ST) {
          slot = 0;
          ++use;
        }
      }
    }
    return;
  }

  // ================================ consumer ================================
  const int sys = lane % TS;
  const int part = lane / TS;
  const uint32_t taddr = tmem_base + ((uint32_t)(cons * 32) << 16);
  // element offsets, inside a stage, of this lane's r-th row in elimination
  // order (ld) and, inside an output buffer, in back-substitution order (st)
  int ld[R], st[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int rl = part ? (R - 1 - r) : r;
    const int rs = part ? r : (R - 1 - r);
    if (CONTIG) {
      const int sw = (sys >> 1) & 3;  // 64-byte swizzle: 16-byte chunk ^= (row / 2) % 4
      ld[r] = part * BOX + sys * R + ((rl / EPC) ^ sw) * EPC + rl % EPC;
      st[r] = part * BOX + sys * R + ((rs / EPC) ^ sw) * EPC + rs % EPC;
    } else {
      ld[r] = part * BOX + rl * TS + sys;
      st[r] = 0;
    }
  }
  const int nvp = part ? nv : 0;  // this half's virtual rows
  const bool drop = (flags & 1) != 0;

  int slot = 0, r_slot = 0, o_buf = 0;
  unsigned phase = 0, r_phase = 0;
  int consumed = 0;
  long long r_issued = 0, r_consumed = 0;
  bool bad = false, timed_out = false;

  for (int ti = 0; ti < my_tiles && !timed_out; ++ti) {
    const int tile = gw + ti * tw;
    int c0, c2;
    tile_coords(tile, c0, c2);
    const int count = CONTIG ? min(TS, n_sys - c0) : min(TS, inner - c0);
    const bool active = sys < count;
    F *const x2t = scratch + (long long)tile * 2 * mt * TS;  // [2 halves][m][16]
    F *const x2w = x2t + part * mt * TS + sys;               // row k at + k * 16

    // ------------------------------ forward ---------------------------------
    Carry<F> c;
    c.zero();
    for (int g = 0; g < n_stages; ++g) {
      if (!__all_sync(0xffffffffu, mbar_wait(&full[slot], phase))) {
        timed_out = true;
        break;
      }
      const F *v = ring + slot * SE;
      F a[R][6];
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int q = 0; q < 6; ++q) a[r][q] = v[ld[r] + q * 2 * BOX];
      if (g * R < nvp + 2) {  // virtual rows, and couplings that leave the line
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int k = g * R + r;
          if (k < nvp) {
#pragma unroll
            for (int q = 0; q < 6; ++q) a[r][q] = (q == 2) ? F(1) : F(0);
          }
          if (k == nvp || k == nvp + 1) a[r][0] = F(0);
          if (k == nvp) a[r][1] = F(0);
        }
      }
      fence_async_shared();
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[slot]);
      ++consumed;
      if (++slot == ST) {
        slot = 0;
        phase ^= 1u;
      }
      F u[R], w[R], y[R];
#pragma unroll
      for (int r = 0; r < R; ++r)
        fwd_row_lean(a[r][0], a[r][1], a[r][2], a[r][3], a[r][4], a[r][5], c, u[r], w[r],
                     y[r]);
      uint32_t tv[32];
#pragma unroll
      for (int r = 0; r < R; ++r) pack_factors<F>(tv, r, u[r], w[r]);
      tmem_store32(taddr + (uint32_t)(g * kColsPerStage), tv);
      F *const x2g = x2w + g * R * TS;
#pragma unroll
      for (int r = 0; r < R; ++r) x2g[r * TS] = y[r];
    }
    if (timed_out) break;
    if (active)
      bad |= !(isfinite(c.u1) && isfinite(c.u2) && isfinite(c.w1) && isfinite(c.w2) &&
               isfinite(c.y1) && isfinite(c.y2));
    // the read-back copies (async proxy) read what this warp has just stored
    fence_async_global();
    __syncwarp();

    // ------------------------------ interface -------------------------------
    const F pu1 = __shfl_xor_sync(0xffffffffu, c.u1, TS);
    const F pu2 = __shfl_xor_sync(0xffffffffu, c.u2, TS);
    const F pw1 = __shfl_xor_sync(0xffffffffu, c.w1, TS);
    const F pw2 = __shfl_xor_sync(0xffffffffu, c.w2, TS);
    const F py1 = __shfl_xor_sync(0xffffffffu, c.y1, TS);
    const F py2 = __shfl_xor_sync(0xffffffffu, c.y2, TS);
    F u0, u1, u2, u3;
    if (part == 0)
      solve_interface(c.u2, c.w2, c.y2, c.u1, c.w1, c.y1, pu1, pw1, py1, pu2, pw2, py2, u0,
                      u1, u2, u3);
    else
      solve_interface(pu2, pw2, py2, pu1, pw1, py1, c.u1, c.w1, c.y1, c.u2, c.w2, c.y2, u0,
                      u1, u2, u3);
    F xa = part ? u1 : u2;  // x of the row just past this half's last row
    F xb = part ? u0 : u3;  // and of the one after it

    // ------------------------------ backward --------------------------------
    // stage s: elimination rows k in [m - (s+1) R, m - s R) of both halves
    int ri_slot = r_slot;
    auto rissue = [&](int s) {
      if (s >= n_stages) return;
      if (lane == 0) {
        const int k0 = mt - (s + 1) * R;
        F *dst = xr + ri_slot * XE;
        mbar_expect_tx(&rfull[ri_slot], 2u * R * TS * (unsigned)sizeof(F));
        bulk_load(dst, x2t + (long long)k0 * TS, R * TS * sizeof(F), &rfull[ri_slot]);
        bulk_load(dst + R * TS, x2t + (long long)(mt + k0) * TS, R * TS * sizeof(F),
                  &rfull[ri_slot]);
      }
      ++r_issued;
      if (++ri_slot == XST) ri_slot = 0;
    };
    for (int s = 0; s < XST; ++s) rissue(s);

    for (int s = 0; s < n_stages; ++s) {
      if (!__all_sync(0xffffffffu, mbar_wait(&rfull[r_slot], r_phase))) {
        timed_out = true;
        break;
      }
      const F *xsrc = xr + r_slot * XE + part * R * TS + sys;
      F xs[R], du[R], dw[R];
#pragma unroll
      for (int r = 0; r < R; ++r) xs[r] = xsrc[(R - 1 - r) * TS];
      uint32_t tv[32];
      tmem_load32(taddr + (uint32_t)((n_stages - 1 - s) * kColsPerStage), tv);
#pragma unroll
      for (int r = 0; r < R; ++r) unpack_factors<F>(tv, R - 1 - r, du[r], dw[r]);
      if (CONTIG && lane == 0) bulk_wait_read<1>();  // output buffer o_buf is free
      fence_async_shared();
      __syncwarp();
      ++r_consumed;
      rissue(s + XST);  // refills the slot just read (ri_slot == r_slot here)
      if (++r_slot == XST) {
        r_slot = 0;
        r_phase ^= 1u;
      }
      if (drop && sys < 8)  // the stage's 1 KB of x2 per half is dead: drop it
        discard_l2_line(x2t + (long long)(part * mt + mt - (s + 1) * R) * TS +
                        sys * (128 / (int)sizeof(F)));
      F xk[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        xk[r] = xs[r] - dw[r] * xb - du[r] * xa;
        xb = xa;
        xa = xk[r];
      }
      if (CONTIG) {
        F *const ob = obuf + o_buf * 2 * BOX;
#pragma unroll
        for (int r = 0; r < R; ++r) ob[st[r]] = xk[r];
        fence_async_shared();
        __syncwarp();
        if (lane == 0) {
          tma_store_2d(&maps.m[5], ob, mt - (s + 1) * R, c0);
          if (mt + s * R < n) tma_store_2d(&maps.m[5], ob + BOX, mt + s * R, c0);
          bulk_commit();
        }
        o_buf ^= 1;
      } else if (active) {
        // the upper half runs towards row 0, the lower half towards row n - 1
        const int row0 = part ? (mt + s * R) : (mt - 1 - s * R);
        const long long step = part ? (long long)inner : -(long long)inner;
        F *const p = x + (long long)c2 * inner * n + c0 + sys + (long long)row0 * inner;
        if (part == 0 || mt + (s + 1) * R <= n) {
#pragma unroll
          for (int r = 0; r < R; ++r) p[r * step] = xk[r];
        } else {  // the lower half's last stages end in virtual rows
#pragma unroll
          for (int r = 0; r < R; ++r)
            if (row0 + r < n) p[r * step] = xk[r];
        }
      }
    }
  }

  if (timed_out) {
    stop[cons] = 1;  // the producer issues nothing more
    // drain what may still land in this consumer's buffers (bounded waits)
    for (int k = 0; k < ST; ++k) {
      if (!mbar_wait(&full[slot], phase)) break;
      if (++slot == ST) {
        slot = 0;
        phase ^= 1u;
      }
    }
    for (; r_consumed < r_issued; ++r_consumed) {
      if (!mbar_wait(&rfull[r_slot], r_phase)) break;
      if (++r_slot == XST) {
        r_slot = 0;
        r_phase ^= 1u;
      }
    }
    if (lane == 0) atomicOr(status_word, STATUS_TIMEOUT_BIT);
  }
  (void)consumed;
  if (CONTIG && lane == 0) bulk_wait<0>();
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(status_word, STATUS_ZERO_PIVOT_BIT);
  // all consumers are done with Tensor Memory: warp 0 frees it
  tmem_fence_before_sync();
  asm volatile("bar.sync 1, %0;\n" ::"n"(32 * NCONS) : "memory");
  tmem_fence_after_sync();
  if (warp == 0) tmem_dealloc(tmem_base, kTmemCols);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
template <typename F>
bool encode(CUtensorMap *m, const F *ptr, const Lines &L, bool contig, int R) {
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
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
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

template <typename F> long long split_row(const Lines &L, bool contig) {
  const long long R = contig ? tmem_rows_per_stage<F, true>() : tmem_rows_per_stage<F, false>();
  return (L.n + 2 * R - 1) / (2 * R) * R;  // m = R ceil(n / 2R)
}

long long tile_count(const Lines &L, bool contig) {
  return contig ? (L.n_sys + TS - 1) / TS : (L.n_sys / L.inner) * ((L.inner + TS - 1) / TS);
}

template <typename F, bool CONTIG, int ST, int XST>
cudaError_t tmem_launch(const SolveArgs<F> &a, int sm_count, cudaStream_t stream) {
  using G = TmemGeom<F, CONTIG, ST, XST>;
  TmaMaps maps;
  const F *ptrs[6] = {a.ds, a.dl, a.d, a.du, a.dw, a.x};
  for (int q = 0; q < 6; ++q)
    if (!encode<F>(&maps.m[q], ptrs[q], a.L, CONTIG, G::R)) return cudaErrorInvalidValue;
  auto kern = tmem_thomas_kernel<F, CONTIG, ST, XST>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)G::kSmem);
  if (err != cudaSuccess) return err;
  const int n = (int)a.L.n;
  const int inner = (int)a.L.inner;
  const int tpr = CONTIG ? 1 : (inner + TS - 1) / TS;
  const long long n_tiles = tile_count(a.L, CONTIG);
  const int mt = (int)split_row<F>(a.L, CONTIG);
  const long long need = (n_tiles + NCONS - 1) / NCONS;
  const int grid = (int)(need < sm_count ? need : sm_count);
  const int flags = (reinterpret_cast<uintptr_t>(a.scratch) % 128 == 0) ? 1 : 0;  // L2 discards
  kern<<<grid, 64 * NCONS, G::kSmem, stream>>>(maps, a.x, static_cast<F *>(a.scratch), n,
                                                mt, inner, tpr, (int)a.L.n_sys,
                                                (int)n_tiles, flags, a.status);
  return cudaGetLastError();
}

template <typename F, bool CONTIG, int ST, int XST> int tmem_occ() {
  using G = TmemGeom<F, CONTIG, ST, XST>;
  auto kern = tmem_thomas_kernel<F, CONTIG, ST, XST>;
  int blocks = 0;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)G::kSmem) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, 64 * NCONS, G::kSmem) !=
          cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return blocks;
}

}  // namespace

// (type, contiguous, forward stages, read-back stages); the first that fits
// shared memory is the default.
#define PENTA_TMEM_CONFIGS(X) \
  X(double, true, 3, 4)       \
  X(double, true, 3, 3)       \
  X(double, false, 3, 4)      \
  X(double, false, 4, 3)      \
  X(float, true, 3, 4)        \
  X(float, false, 3, 4)       \
  X(float, false, 4, 3)

template <typename F> const std::vector<TmemConfig> &tmem_configs() {
  static const std::vector<TmemConfig> v = [] {
    std::vector<TmemConfig> out;
#define PENTA_X(FT_, C_, ST_, XST_)                                                    \
  if (std::is_same<F, FT_>::value)                                                     \
    out.push_back(TmemConfig{C_, ST_, XST_, TmemGeom<FT_, C_, ST_, XST_>::R,           \
                             TmemGeom<FT_, C_, ST_, XST_>::kSmem});
    PENTA_TMEM_CONFIGS(PENTA_X)
#undef PENTA_X
    return out;
  }();
  return v;
}

template <typename F> int tmem_occupancy(const TmemConfig &c) {
#define PENTA_X(FT_, C_, ST_, XST_)                                                    \
  if (std::is_same<F, FT_>::value && c.contig == C_ && c.stages == ST_ &&              \
      c.xstages == XST_)                                                               \
    return tmem_occ<FT_, C_, ST_, XST_>();
  PENTA_TMEM_CONFIGS(PENTA_X)
#undef PENTA_X
  return 0;
}

template <typename F> size_t tmem_scratch_bytes(const Lines &L, bool contig) {
  return (size_t)tile_count(L, contig) * 2 * (size_t)split_row<F>(L, contig) * TS * sizeof(F);
}

template <typename F>
bool tmem_supported(const SolveArgs<F> &a, bool contig, size_t usable_buf) {
  if (tensor_map_encoder() == nullptr) return false;
  const Lines &L = a.L;
  if (contig) {
    if (L.inner != 1 || (L.n * sizeof(F)) % 16 != 0) return false;
  } else {
    if (L.inner <= 1 || (L.inner * sizeof(F)) % 16 != 0) return false;
  }
  const long long R =
      contig ? tmem_rows_per_stage<F, true>() : tmem_rows_per_stage<F, false>();
  const long long mt = split_row<F>(L, contig);
  if (L.n - mt < 2) return false;                          // two real rows per half
  if (mt / R > (long long)(kTmemCols / kColsPerStage)) return false;  // TMEM capacity
  if (L.n * L.n_sys >= (1LL << 31) || tile_count(L, contig) >= (1LL << 31)) return false;
  if (a.scratch == nullptr || reinterpret_cast<uintptr_t>(a.scratch) % 16 != 0 ||
      tmem_scratch_bytes<F>(L, contig) > usable_buf)
    return false;
  const void *ptrs[6] = {a.ds, a.dl, a.d, a.du, a.dw, a.x};
  for (const void *p : ptrs)
    if (reinterpret_cast<uintptr_t>(p) % 16 != 0) return false;
  return true;
}

template <typename F>
cudaError_t launch_tmem(const SolveArgs<F> &a, const TmemConfig &c, int sm_count,
                        cudaStream_t stream) {
#define PENTA_X(FT_, C_, ST_, XST_)                                                    \
  if (std::is_same<F, FT_>::value && c.contig == C_ && c.stages == ST_ &&              \
      c.xstages == XST_)                                                               \
    return tmem_launch<FT_, C_, ST_, XST_>(reinterpret_cast<const SolveArgs<FT_> &>(a), \
                                           sm_count, stream);
  PENTA_TMEM_CONFIGS(PENTA_X)
#undef PENTA_X
  return cudaErrorInvalidConfiguration;
}

template const std::vector<TmemConfig> &tmem_configs<double>();
template const std::vector<TmemConfig> &tmem_configs<float>();
template int tmem_occupancy<double>(const TmemConfig &);
template int tmem_occupancy<float>(const TmemConfig &);
template size_t tmem_scratch_bytes<double>(const Lines &, bool);
template size_t tmem_scratch_bytes<float>(const Lines &, bool);
template bool tmem_supported<double>(const SolveArgs<double> &, bool, size_t);
template bool tmem_supported<float>(const SolveArgs<float> &, bool, size_t);
template cudaError_t launch_tmem<double>(const SolveArgs<double> &, const TmemConfig &, int,
                                         cudaStream_t);
template cudaError_t launch_tmem<float>(const SolveArgs<float> &, const TmemConfig &, int,
                                        cudaStream_t);

}  // namespace penta
