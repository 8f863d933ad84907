// tmem_kernels.cu -- batched Thomas for all three directions with the
// factors held in Tensor Memory; one grid per launch, or many uneven grids in
// one persistent launch.
//
// Algorithm (as tiled_kernels.cu with P = 2): a consumer warp owns tiles of 16
// lines.  Lanes 0..15 eliminate the upper rows [0, m) of their line downwards,
// lanes 16..31 the lower rows [m, n) upwards on the mirrored band (dw, du, d,
// dl, ds), the halves meet in a 4x4 interface solve done with warp shuffles,
// and each half substitutes back towards its own end.
//
// m = R ceil(n / 2R) is a multiple of the rows per stage R, and the lower half
// is extended by v = 2m - n virtual rows ahead of its first real row (rows
// n .. n+v-1 of the mirrored sweep): identity rows (d = 1, everything else 0)
// whose factors are exact zeros, so the carries reach the first real row as
// exact zeros, as if the sweep had started there.  Both halves then run m
// rows in lockstep: every stage is full and every offset below is the same
// for both halves.
//
// Per CTA (one per SM), for each TMEM lane quarter c (0..3) three warps:
// warp c eliminates (forward sweep), warp 4 + c feeds it, warp 8 + c
// substitutes back.  The forward sweep of a tile overlaps the back
// substitution of the previous one, so the load ring keeps draining while
// results are written.
//  * The feeding warp fills its ring of ST stages.  A stage is 12 TMA tiles
//    (6 arrays x 2 halves) of R rows x 16 lines on one mbarrier; the lower
//    half's tiles come from the mirrored arrays.  The eliminating warp copies
//    a stage into registers and releases the slot at once.
//  * Factors in Tensor Memory (lanes 32c..32c+31, the quarter these warps can
//    reach), one tcgen05.st per stage on the way down and one tcgen05.ld per
//    stage on the way back, in one of four factor modes FM:
//      - 3, du2, dw2 and x2 all in TMEM (short lines): 6 columns per FP64
//        row, 3 per FP32 row, 10 blocks of a stage in 480 of the 512
//        columns, used up to 8 stages (4 for FP32 along y/z): n <= 128 FP64,
//        256 FP32 along x, 128 FP32 along y/z;
//        nothing goes through the buffer, so the back substitution waits for
//        no read-back and a call needs no buffer;
//      - 0, du2 and dw2 in TMEM: 4 columns per FP64 row, 2 per FP32 row;
//        512 columns hold m <= 128 (FP64) / 256 (FP32) rows, n <= 256 / 512;
//      - 1, du2 only: half the columns, n <= 512 / 1024, with dw2 travelling
//        with x2 through the caller's buffer;
//      - 2, none (longer lines): du2, dw2 and x2 all travel through the
//        buffer, and n is bounded only by the buffer.
//    Consecutive tiles of a warp fill TMEM blocks in opposite orders, so the
//    blocks the back substitution of tile t frees first are the ones the
//    forward sweep of tile t + 1 fills first; a progress word in shared
//    memory (tile, steps done) tells the eliminating warp when a block is
//    free.  The carries of the two halves are handed over in shared memory
//    behind an mbarrier.
//  * x2 (and dw2, du2 as the mode has it) make an L2 round trip through the
//    caller's buffer ([tile][half][m][16] of x2, [..][16][2] (dw2, x2) pairs,
//    or [..][m][3][16] with du2, dw2, x2 each a 128-byte line per row),
//    written once per row and read back, most recent first, by two bulk
//    copies per stage into a small ring; each 128-byte line is dropped from
//    L2 (discard.global.L2) once read, so it never reaches HBM while it fits
//    in L2.  The stores carry an evict-last L2 policy and the streamed
//    accesses (coefficient and right-hand-side loads -- along x with factors
//    in the buffer excepted --, results, read-backs) an evict-first one, so
//    that the scratch survives in L2 while the arrays stream past it.
//  * Output: strided directions store x directly (16 consecutive lines are one
//    128-byte segment).  Along x, a lane's rows are contiguous in memory: the
//    results of two steps go into a 128-byte-swizzled shared tile of 2R rows
//    per half and leave as one TMA tile store (128-byte rows).
//
// Grids are described by jobs (tensor maps, x, buffer region, geometry).  A
// single-grid launch passes its job as a kernel parameter; a batched launch
// reads a job table from device memory and walks the concatenated tile list
// of all its grids, so one launch -- and one CUDA-graph node -- solves them all.
//
// Tensor views: along x {n, n_sys} with tiles {R, 16} (64-byte rows, 64-byte
// swizzle; 256-byte L2 promotion, so a line's next rows are already in L2)
// and, for the stores, {2R, 16} (128-byte swizzle); strided {inner, n, outer}
// with tiles {16, R, 1}.  TMA needs
// 16-byte aligned bases and row strides and 16-byte aligned innermost
// coordinates: n * sizeof(F) % 16 == 0 along x (every row coordinate used is
// a multiple of R), inner * sizeof(F) % 16 == 0 for the strided views.
//
// Waits are bounded (tma_device.cuh).  A wait that runs out raises
// STATUS_TIMEOUT_BIT; the warp raises its quarter's stop flag (the feeding
// warp then issues nothing more, the other warps leave at their next wait),
// drains the copies it has in flight (again bounded) and the CTA frees its
// TMEM before returning.  A zero or non-finite pivot turns the carries into NaN or
// infinity, which is checked once per tile (STATUS_ZERO_PIVOT_BIT).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>

#include "penta_internal.hpp"
#include "tma_device.cuh"

namespace penta {

// One grid of a launch.  Layout shared by host and device; 64-byte aligned
// for the tensor maps.
template <typename F> struct alignas(64) TmemJob {
  CUtensorMap maps[7];  // ds, dl, d, du, dw, x; x again with 2R-row boxes (along x)
  const F *arr[6];      // the same arrays
  F *x;
  F *scratch;           // this grid's region of the caller's buffer
  int n, mt, inner, tpr, n_sys, n_tiles, tile_base;
  int tma;              // 1: TMA tiles; 0: element copies (misaligned grid)
  int bulk;             // 1: every array 16-byte aligned (bulk-copy loads possible)
  int grp;              // pitched layout: maps[0..5] view groups of grp rows (strided)
                        // or lines (x) so that each group is 16-byte periodic; 0: none
  int tail;             // first tile (x) / the run (strided) whose rows or lines lie
                        // outside whole groups: fetched by bulk copies
  int chunks;           // pitched layout filled by 16-byte cp.async copies (no groups)
};

namespace {

constexpr int TS = 16;              // lines per tile
constexpr int NCONS = 4;            // consumer warps per CTA, one per TMEM lane quarter
constexpr uint32_t kTmemCols = 512; // the whole of Tensor Memory

template <typename F, bool CONTIG> constexpr int tmem_rows_per_stage() {
  return CONTIG ? 64 / (int)sizeof(F) : 1024 / (TS * (int)sizeof(F));
}
// Factor modes: 0 du2 and dw2 in TMEM, x2 through the buffer; 1 du2 in TMEM,
// (dw2, x2) through the buffer; 2 all three through the buffer; 3 all three in
// TMEM (short lines: no buffer round trip at all).
template <typename F, int FM> __host__ __device__ constexpr int tmem_values_per_row() {
  return FM == 0 ? 2 : FM == 3 ? 3 : 1;
}
// TMEM columns per stage: R rows of the values kept there, sizeof(F)/4 each.
template <typename F, int FM> constexpr int tmem_cols_per_stage() {
  return 64 / (int)sizeof(F) * tmem_values_per_row<F, FM>() * (int)sizeof(F) / 4;
}

// LD: how the forward stages are filled.  0: TMA tensor tiles of R x 16 (or,
// for a misaligned grid, element copies into the same layout); 1: bulk copies
// of 16-byte aligned supersets into a pitched layout -- each row of 16 lines
// (strided) or each line's R rows (along x) widened by one 16-byte chunk, so a
// grid whose rows or runs start anywhere is fetched with 16-byte requests.
template <typename F, bool CONTIG, int FM, int ST, int XST, int LD> struct TmemGeom {
  static constexpr int R = tmem_rows_per_stage<F, CONTIG>();
  static constexpr int EPC = 16 / (int)sizeof(F);     // elements per 16-byte chunk
  static constexpr int PW = FM == 2 ? 3 : FM == 1 ? 2 : FM == 3 ? 0 : 1;  // scratch values per row
  static constexpr int BOX = R * TS;                  // elements per TMA tile
  // bulk layout pitches: a strided row of 16 lines + one chunk; a line's R rows
  // + one chunk (along x)
  static constexpr int PS = TS + EPC;
  static constexpr int PL = R + EPC;
  // The group view's residue classes each land in a block of rows/grp rows
  // (strided, pitch PS) or 16/grp lines (x, pitch PL), and a TMA destination
  // must start on a 128-byte boundary: CPg = one class block of group size g,
  // rounded up to 128 bytes.  A tile holds g of them, or the bulk layout.
  static constexpr int kRows = CONTIG ? TS : R;
  static constexpr int kPitch = CONTIG ? PL : PS;
  static constexpr int cls(int g) {
    return ((kRows / g) * kPitch * (int)sizeof(F) + 127) / 128 * 128 / (int)sizeof(F);
  }
  static constexpr int CP2 = cls(2), CP4 = cls(4);
  // along x, lines 8-15 of a tile sit one chunk further (line_off): lines l
  // and l + 8 would otherwise start on the same banks with the same shift
  __host__ __device__ static constexpr int line_off(int l) { return l * PL + (l >= 8 ? EPC : 0); }
  static constexpr int kPitched0 = kRows * kPitch + (CONTIG ? EPC : 0);
  static constexpr int kPitched1 = 2 * CP2 > kPitched0 ? 2 * CP2 : kPitched0;
  static constexpr int kPitched =
      (sizeof(F) == 4 && 4 * CP4 > kPitched1) ? 4 * CP4 : kPitched1;  // FP32 groups of 4
  static constexpr int kUnit = 128 / (int)sizeof(F);
  static constexpr int BOXL =
      LD == 0 ? BOX : (kPitched + kUnit - 1) / kUnit * kUnit;  // per tile, 128 B multiple
  static constexpr int SE = 12 * BOXL;                // forward stage
  static constexpr int XE = 2 * R * TS * PW;          // read-back stage
  static constexpr int OBE = CONTIG ? 8 * BOX : 0;    // output: 2 buffers x 2 halves x 2R rows
  static constexpr int HE = 2 * 6 * 32;               // carries: 2 slots x 6 values x 32 lanes
  static constexpr int kCols = tmem_cols_per_stage<F, FM>();
  static constexpr int NB = (int)kTmemCols / kCols;   // TMEM blocks of one stage each
  static constexpr size_t kData = (size_t)(ST * SE + XST * XE + OBE + HE) * sizeof(F);
  static constexpr size_t kBars = (size_t)(2 * ST + XST + 2) * 8;
  static constexpr size_t kCons = (kData + kBars + 1023) / 1024 * 1024;
  static constexpr size_t kTail = 64;                 // TMEM address, stop flags, progress
  static constexpr size_t kUsed = NCONS * kCons + kTail + 1024;  // + alignment slack
  // at least 116 KB, so that one CTA holds an SM (and all of its TMEM)
  static constexpr size_t kSmem = kUsed > 118784 ? kUsed : 118784;
  static_assert(kSmem <= 232448, "shared memory per CTA");
  static_assert((BOXL * sizeof(F)) % 128 == 0 && (CP2 * sizeof(F)) % 128 == 0 &&
                    (CP4 * sizeof(F)) % 128 == 0,
                "TMA destinations must stay 128-byte aligned");
  static_assert((PS * sizeof(F)) % 16 == 0 && (PL * sizeof(F)) % 16 == 0,
                "bulk-copy destinations must stay 16-byte aligned");
  static_assert(R * tmem_values_per_row<F, FM>() * (int)sizeof(F) / 4 == kCols,
                "TMEM columns per stage");
  static_assert(kCols == 16 || kCols == 32 || kCols == 48, "a TMEM load or store per stage");
};

template <typename F> __device__ __forceinline__ void put_bits(uint32_t *tv, int c, F v);
template <> __device__ __forceinline__ void put_bits<double>(uint32_t *tv, int c, double v) {
  tv[c] = (uint32_t)__double2loint(v);
  tv[c + 1] = (uint32_t)__double2hiint(v);
}
template <> __device__ __forceinline__ void put_bits<float>(uint32_t *tv, int c, float v) {
  tv[c] = __float_as_uint(v);
}
template <typename F> __device__ __forceinline__ F get_bits(const uint32_t *tv, int c);
template <> __device__ __forceinline__ double get_bits<double>(const uint32_t *tv, int c) {
  return __hiloint2double((int)tv[c + 1], (int)tv[c]);
}
template <> __device__ __forceinline__ float get_bits<float>(const uint32_t *tv, int c) {
  return __uint_as_float(tv[c]);
}

template <typename F, bool CONTIG, int FM, int ST, int XST, int LD, bool BATCH>
__global__ void __launch_bounds__(96 * NCONS, 1)
tmem_thomas_kernel(const __grid_constant__ TmemJob<F> job1, const TmemJob<F> *__restrict__ jobs,
                   int n_jobs, int total_tiles, int flags, int *__restrict__ status_word) {
  using G = TmemGeom<F, CONTIG, FM, ST, XST, LD>;
  using V2 = typename Vec2<F>::T;
  constexpr int R = G::R, BOX = G::BOX, SE = G::SE, XE = G::XE, PW = G::PW, NB = G::NB;
  constexpr int BOXL = G::BOXL, PS = G::PS, PL = G::PL, CP2 = G::CP2, CP4 = G::CP4;
  constexpr int EPC = 16 / (int)sizeof(F);  // elements per 16-byte chunk
  constexpr int CW = (int)sizeof(F) / 4;    // TMEM columns per value
  constexpr int kMirror[6] = {4, 3, 2, 1, 0, 5};

  extern __shared__ __align__(128) unsigned char smem_raw[];
  // swizzled tiles need 1 KB aligned destinations; the launch adds 1 KB slack
  unsigned char *const base =
      smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const int warp = threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  const int role = warp / NCONS;  // 0 eliminates, 1 feeds, 2 substitutes back
  const int cons = warp % NCONS;  // the lane quarter (and ring) this warp works on
  auto region = [&](int c) { return base + c * G::kCons; };
  F *const ring = reinterpret_cast<F *>(region(cons));
  F *const xr = ring + ST * SE;    // read-back stages [XST][2 halves][R][16][PW]
  F *const obuf = xr + XST * XE;   // along x: [2 buffers][2 halves][2R rows x 16 lines]
  F *const hand = obuf + G::OBE;   // carries handed over: [2 slots][6][32 lanes]
  uint64_t *const full = reinterpret_cast<uint64_t *>(region(cons) + G::kData);
  uint64_t *const empty = full + ST;
  uint64_t *const rfull = empty + ST;
  uint64_t *const hfull = rfull + XST;  // [2]: a tile's forward sweep is done
  uint32_t *const tmem_slot = reinterpret_cast<uint32_t *>(base + NCONS * G::kCons);
  volatile int *const stop = reinterpret_cast<volatile int *>(tmem_slot + 4);  // [NCONS]
  int *const prog = reinterpret_cast<int *>(tmem_slot + 8);                    // [NCONS]

  const int gw = blockIdx.x * NCONS + cons;
  const int tw = gridDim.x * NCONS;
  const int my_tiles = gw < total_tiles ? (total_tiles - 1 - gw) / tw + 1 : 0;

  if (threadIdx.x == 0) {
    for (int c = 0; c < NCONS; ++c) {
      uint64_t *f = reinterpret_cast<uint64_t *>(region(c) + G::kData);
      for (int s = 0; s < 2 * ST + XST + 2; ++s) mbar_init(&f[s], s < ST ? 32 : 1);
      stop[c] = 0;
      prog[c] = 0;
    }
    mbar_init_fence();
  }
  if (warp == 0) tmem_alloc(tmem_slot, kTmemCols);
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  const uint32_t tmem_base = *tmem_slot;
  // Programmatic dependent launch: the next grid in the stream may run its
  // prologue on SMs this grid's CTAs leave; this grid touches global memory
  // only after the previous grid has completed (everything above is on-chip)
  if (threadIdx.x == 0) asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  asm volatile("griddepcontrol.wait;\n" ::: "memory");

  // the job of global tile t (t increases along a warp's sequence)
  auto job_of = [&](int t, int &cursor) -> const TmemJob<F> * {
    if constexpr (BATCH) {
      while (cursor + 1 < n_jobs && jobs[cursor + 1].tile_base <= t) ++cursor;
      return &jobs[cursor];
    } else {
      return &job1;
    }
  };
  // a job's geometry, kept in registers while a warp stays on that job
  struct Geo {
    const TmemJob<F> *J;
    F *x, *scratch;
    int n, mt, inner, tpr, n_sys, tile_base, n_tiles, tma, grp, tail, chunks;
  };
  auto load_geo = [&](const TmemJob<F> *J, Geo &g) {
    g.J = J;
    g.x = J->x;
    g.scratch = J->scratch;
    g.n = J->n;
    g.mt = J->mt;
    g.inner = J->inner;
    g.tpr = J->tpr;
    g.n_sys = J->n_sys;
    g.tile_base = J->tile_base;
    g.n_tiles = J->n_tiles;
    g.tma = J->tma;
    g.grp = J->grp;
    g.tail = J->tail;
    g.chunks = J->chunks;
  };
  auto tile_coords = [&](const Geo &g, int tile, int &c0, int &c2) {
    if (CONTIG) {
      c0 = tile * TS;  // first line
      c2 = 0;
    } else {
      c2 = tile / g.tpr;  // run
      c0 = (tile - c2 * g.tpr) * TS;
    }
  };

  // ================================ producer ================================
  // The whole warp: lane 0 issues TMA tiles (arriving for all 32 lanes), or
  // all lanes copy elements of a misaligned grid.  full[] counts 32 arrivals.
  if (role == 1) {
    // read once: evict first -- except along x with dw2 in the buffer, where
    // the larger scratch round trip does better against normal-priority loads
    // streamed loads evict-first, except along x with factors in the buffer, where
    // they keep normal priority unless the launch capped its CTAs (flags bit 1)
    const uint64_t pol_in = (CONTIG && FM >= 1 && !(flags & 2)) ? l2_policy_normal()
                                                                 : l2_policy_first();
    int slot = 0, use = 0, cursor = 0, fenced = -1;
    Geo JG;
    load_geo(job_of(gw, cursor), JG);
    const F *arrs[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    for (int ti = 0; ti < my_tiles; ++ti) {
      const int t = gw + ti * tw;
      const TmemJob<F> *J = job_of(t, cursor);
      if (J != JG.J || ti == 0) {
        load_geo(J, JG);
        if (LD == 1 || !JG.tma)
#pragma unroll
          for (int q = 0; q < 6; ++q) arrs[q] = J->arr[q];
      }
      const bool tma = LD == 0 && JG.tma != 0;
      const bool maps_used = tma || (LD == 1 && J->grp > 0);
      if (BATCH && cursor != fenced) {  // a new grid: its maps, and the next grid's
        if (lane == 0) {
          if (maps_used)
            for (int q = 0; q < 6; ++q) {
              tensormap_acquire(&J->maps[q]);  // host-written: acquire once
              tensormap_prefetch(&J->maps[q]);
            }
          if (cursor + 1 < n_jobs && (jobs[cursor + 1].tma || jobs[cursor + 1].grp))
            for (int q = 0; q < 6; ++q) tensormap_prefetch(&jobs[cursor + 1].maps[q]);
        }
        fenced = cursor;
      }
      int c0, c2;
      tile_coords(JG, t - JG.tile_base, c0, c2);
      const int n = JG.n, mt = JG.mt, n_stages = mt / R, inner = JG.inner;
      for (int g = 0; g < n_stages; ++g) {
        // lane 0 waits for the slot (the others park in the shuffle, issuing
        // nothing) and reads the stop flag for the warp
        int go = 1;
        if (lane == 0) {
          go = (use == 0 || mbar_wait(&empty[slot], (unsigned)(use - 1) & 1u)) ? 1 : 0;
          if (go && stop[cons] != 0) go = 2;
        }
        go = __shfl_sync(0xffffffffu, go, 0);
        if (go != 1) {
          if (go == 0 && lane == 0) atomicOr(status_word, STATUS_TIMEOUT_BIT);
          return;
        }
        const int r_up = g * R;
        const int r_dn = 2 * mt - (g + 1) * R;  // lower half, virtual rows included
        F *dst = ring + slot * SE;
        bool by_groups = false;
        if constexpr (LD == 1)
          by_groups = JG.grp > 0 && (CONTIG ? (c0 / TS < JG.tail) : (c2 != JG.tail));
        if (LD == 1 && by_groups) {
          // One TMA box per residue class of the group view: along x the
          // lines c0 + k grp + sub (box {R + chunk, 16 / grp} at the aligned-
          // down first row), strided the rows whose global index G = c2 n + r
          // has G % grp == sub (box {16 + chunk, R / grp} of consecutive
          // groups).  Class sub lands at sub (16/grp) PL (x) or sub (R/grp) PS
          // (strided) in its tile; the forward warp reads it there.
          if (lane == 0) {
            const bool lower = r_dn < n;  // else all rows are virtual: not loaded
            const int gq = JG.grp, lgq = gq == 4 ? 2 : (gq == 2 ? 1 : 3);
            const int cpe = gq == 4 ? CP4 : CP2;  // class block (128-byte multiple)
            mbar_arrive_n(&full[slot], 31);
            // each box is rows/grp x pitch elements; grp of them per tile half
            constexpr unsigned kTileBytes = (unsigned)(G::kRows * G::kPitch * sizeof(F));
            mbar_expect_tx(&full[slot], (lower ? 12u : 6u) * kTileBytes);
#pragma unroll
            for (int q = 0; q < 6; ++q)
#pragma unroll
              for (int h = 0; h < 2; ++h) {
                if (h && !lower) continue;
                const CUtensorMap *map = &J->maps[h ? kMirror[q] : q];
                F *const tb = dst + (2 * q + h) * BOXL;
                const int r0 = h ? r_dn : r_up;
                for (int sub = 0; sub < gq; ++sub) {
                  if (CONTIG) {
                    const int sh = (sub * (n & (G::EPC - 1))) & (G::EPC - 1);
                    tma_load_2d_hint(tb + sub * cpe, map, &full[slot],
                                     sub * n + r0 - sh, c0 >> lgq, pol_in);
                  } else {
                    const long long G0 = (long long)c2 * n + r0;
                    const int rr0 = (sub - (int)(G0 & (gq - 1))) & (gq - 1);
                    const int sh = (sub * (inner & (G::EPC - 1))) & (G::EPC - 1);
                    tma_load_2d_hint(tb + sub * cpe, map, &full[slot],
                                     sub * inner + c0 - sh, (int)((G0 + rr0) >> lgq), pol_in);
                  }
                }
              }
          }
        } else if (LD == 1 && JG.chunks) {
          // 16-byte cp.async copies of the same windows as the bulk copies
          // below: every row (strided) or line's R rows (x), widened to the
          // 16-byte chunks that hold them.  Each lane keeps the same (window,
          // chunk) pairs for every tile half, so a copy costs the stage's row
          // offset and an add.  A chunk reaching past an array's end is read
          // only up to it (the rest zero-filled); windows of rows past n (the
          // lower half's virtual rows) and of lines past the grid are skipped.
          constexpr int NCH = (CONTIG ? PL : PS) / G::EPC;  // chunks per window
          constexpr int NW = CONTIG ? TS : R;                // windows per tile half
          constexpr int NP = NW * NCH;
          constexpr int KP = (NP + 31) / 32;
          const long long npts = (long long)n * JG.n_sys;
#pragma unroll
          for (int kp = 0; kp < KP; ++kp) {
            const int p = lane + 32 * kp;
            if (p >= NP) continue;
            const int w = p / NCH, j = p - (p / NCH) * NCH;
            const int doff = (CONTIG ? G::line_off(w) : w * PS) + j * G::EPC;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int r0 = h ? r_dn : r_up;
              long long off;
              bool ok;
              if (CONTIG) {
                off = (long long)(c0 + w) * n + r0;
                ok = c0 + w < JG.n_sys && r0 < n;
              } else {
                off = (long long)c2 * inner * n + (long long)(r0 + w) * inner + c0;
                ok = r0 + w < n;
              }
              const long long e = (off & ~(long long)(G::EPC - 1)) + j * G::EPC;
              const long long left = npts - e;
              const int bytes = !ok || left <= 0
                                    ? 0
                                    : (left >= G::EPC ? 16 : (int)(left * (long long)sizeof(F)));
              if (bytes == 0) continue;
#pragma unroll
              for (int q = 0; q < 6; ++q) {
                const int aq = h ? (q < 5 ? 4 - q : 5) : q;
                cp_async16_bytes(dst + (2 * q + h) * BOXL + doff, arrs[aq] + e, bytes);
              }
            }
          }
          cp_async_mbar_arrive(&full[slot]);
        } else if constexpr (LD == 1) {
          // Bulk copies of 16-byte aligned supersets.  Copy k of the stage:
          // tile bx = 2 q + half, then line (along x) or row (strided) `sub`.
          // Each lane arrives once with its own byte count, then issues its
          // copies; rows past n, lines past the grid and tiles past the run are
          // not fetched.  A window whose last 16-byte chunk would reach past
          // the array's end takes those few elements with plain loads (before
          // the arrival that publishes them), so nothing outside the arrays
          // is read.
          constexpr int NCP = CONTIG ? 12 * TS : 12 * R;  // copies per stage
          constexpr int KC = NCP / 32;
          static_assert(NCP % 32 == 0, "copies per lane");
          const long long npts = (long long)n * JG.n_sys;  // elements per array
          const F *srcs[KC];
          uint32_t dsts[KC];
          unsigned nbs[KC];
          unsigned mine = 0;
#pragma unroll
          for (int kk = 0; kk < KC; ++kk) {
            const int k = lane + 32 * kk;
            const int bx = CONTIG ? k / TS : k / R;
            const int sub = CONTIG ? k % TS : k % R;
            const int q = bx >> 1, h = bx & 1;
            // the array (mirrored for the lower half: ds<->dw, dl<->du), picked
            // by selects so that `arrs` stays in registers
            const int aq = h ? (q < 5 ? 4 - q : 5) : q;
            const F *src = arrs[0];
#pragma unroll
            for (int j = 1; j < 6; ++j)
              if (aq == j) src = arrs[j];
            long long off;
            int cnt;
            if (CONTIG) {
              const int line = c0 + sub;
              const int row0 = h ? r_dn : r_up;
              cnt = (line < JG.n_sys && row0 < n) ? min(R, n - row0) : 0;
              off = (long long)line * n + row0;
            } else {
              const int row = (h ? r_dn : r_up) + sub;
              cnt = row < n ? min(TS, inner - c0) : 0;
              off = (long long)c2 * inner * n + (long long)row * inner + c0;
            }
            F *const tdst = dst + bx * BOXL + (CONTIG ? G::line_off(sub) : sub * PS);
            nbs[kk] = 0;
            if (cnt > 0) {
              const long long first = off & ~(long long)(EPC - 1);
              const long long last = off + cnt;  // exclusive, <= npts
              long long end = (last + EPC - 1) & ~(long long)(EPC - 1);
              if (end > npts) {
                end = npts & ~(long long)(EPC - 1);
                for (long long e = end > off ? end : off; e < last; ++e) tdst[e - first] = src[e];
              }
              if (end > first) {
                nbs[kk] = (unsigned)((end - first) * (long long)sizeof(F));
                srcs[kk] = src + first;
                dsts[kk] = smem_u32(tdst);
                mine += nbs[kk];
              }
            }
          }
          mbar_expect_tx(&full[slot], mine);
#pragma unroll
          for (int kk = 0; kk < KC; ++kk)
            if (nbs[kk] != 0) bulk_load_smem_hint(dsts[kk], srcs[kk], nbs[kk], &full[slot], pol_in);
        } else if (tma) {
          if (lane == 0) {
            const bool lower = r_dn < n;  // else all rows are virtual: not loaded
            mbar_arrive_n(&full[slot], 31);  // for the lanes that copy nothing
            mbar_expect_tx(&full[slot], (lower ? 12u : 6u) * BOX * (unsigned)sizeof(F));
            // along x an even stage and the next one read the two 64-byte
            // halves of the same 128-byte line of every line (both tile
            // halves): with flags bit 2 the next stage's tiles are requested
            // into L2 now, so each line reaches DRAM as one burst
            const bool pre = CONTIG && (flags & 4) && (g & 1) == 0 && g + 1 < n_stages;
#pragma unroll
            for (int q = 0; q < 6; ++q) {
              if (CONTIG) {
                tma_load_2d_hint(dst + (2 * q) * BOX, &J->maps[q], &full[slot], r_up, c0, pol_in);
                if (pre) tma_prefetch_2d_hint(&J->maps[q], r_up + R, c0, pol_in);
                if (lower)
                  tma_load_2d_hint(dst + (2 * q + 1) * BOX, &J->maps[kMirror[q]], &full[slot],
                                   r_dn, c0, pol_in);
                if (pre && r_dn - R < n)
                  tma_prefetch_2d_hint(&J->maps[kMirror[q]], r_dn - R, c0, pol_in);
              } else {
                tma_load_3d_hint(dst + (2 * q) * BOX, &J->maps[q], &full[slot], c0, r_up, c2,
                                 pol_in);
                if (lower)
                  tma_load_3d_hint(dst + (2 * q + 1) * BOX, &J->maps[kMirror[q]], &full[slot],
                                   c0, r_dn, c2, pol_in);
              }
            }
          }
        } else {
          // the same tiles, element by element; rows past n and lines past the
          // grid read as zeros.  The 12 tiles unrolled: each one's array is
          // a register (no job-table load per element).  Along x a lane copies
          // row lane % R of lines lane / R + (32 / R) k; strided, line
          // lane % 16 at rows lane / 16 + 2 k.
          constexpr int K = BOX / 32;  // elements per lane per tile
#pragma unroll
          for (int bx = 0; bx < 12; ++bx) {
            const int q = bx >> 1, h = bx & 1;
            const F *const src = h ? arrs[kMirror[q]] : arrs[q];
            const int rbase = h ? r_dn : r_up;
            F *const tdst = dst + bx * BOX;
            if (CONTIG) {
              const int rr = lane % R;
              const int row = rbase + rr;
#pragma unroll 4
              for (int k = 0; k < K; ++k) {
                const int ls = lane / R + (32 / R) * k;
                const bool valid = row < n && c0 + ls < JG.n_sys;
                const int doff = ls * R + ((rr / EPC) ^ ((ls >> 1) & 3)) * EPC + rr % EPC;
                cp_async_zfill<sizeof(F)>(tdst + doff,
                                          valid ? src + (long long)(c0 + ls) * n + row : src,
                                          valid);
              }
            } else {
              const int ls = lane % TS;
              const bool lvalid = c0 + ls < inner;
              const F *const lp = src + (long long)c2 * inner * n + c0 + ls;
#pragma unroll 4
              for (int k = 0; k < K; ++k) {
                const int rr = lane / TS + 2 * k;
                const int row = rbase + rr;
                const bool valid = lvalid && row < n;
                cp_async_zfill<sizeof(F)>(tdst + rr * TS + ls,
                                          valid ? lp + (long long)row * inner : src, valid);
              }
            }
          }
          cp_async_mbar_arrive(&full[slot]);
        }
        if (++slot == ST) {
          slot = 0;
          ++use;
        }
      }
    }
    return;
  }

  const int sys = lane % TS;
  const int part = lane / TS;
  const uint32_t taddr = tmem_base + ((uint32_t)(cons * 32) << 16);

  if (role == 0) {
    // ============================ forward sweep ==============================
    // Tile ti stores stage g's factors in TMEM block g (even ti) or NB-1-g
    // (odd ti).  The back-substitution of the previous tile reads its blocks
    // in the order that frees exactly the ones this tile fills first, and
    // publishes its progress in prog[cons] = tile * 65536 + steps done: block
    // b of this tile is free once that tile has done b's share of its steps.
    // element offset, inside a stage, of this lane's r-th row (strided), or
    // of the 16-byte chunk holding its rows 2j and 2j+1 (along x: a line's
    // rows are contiguous, two to a chunk, so they are read in pairs)
    int ld[CONTIG ? R / 2 : R];
    if constexpr (CONTIG) {
      const int sw = (sys >> 1) & 3;  // 64-byte swizzle: 16-byte chunk ^= (line / 2) % 4
#pragma unroll
      for (int j = 0; j < R / 2; ++j) {
        const int e = part ? (R - 2 - 2 * j) : 2 * j;  // the pair's even row in the tile
        ld[j] = part * BOX + sys * R + ((e / EPC) ^ sw) * EPC + e % EPC;
      }
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) ld[r] = part * BOX + (part ? (R - 1 - r) : r) * TS + sys;
    }
    const uint64_t pol_x2 = l2_policy_last();  // read back soon: keep in L2
    int slot = 0, cursor = 0, n_prev = 0, seen = 0;
    unsigned phase = 0;
    Geo JG;
    load_geo(job_of(gw, cursor), JG);
    bool bad = false;
    int fail = 0;  // 0 fine, 1 a wait ran out, 2 stopped by another warp
    int ti = 0;
    for (; ti < my_tiles; ++ti) {
      const int t = gw + ti * tw;
      const TmemJob<F> *J = job_of(t, cursor);
      if (J != JG.J) load_geo(J, JG);
      const int tile = t - JG.tile_base;
      int c0, c2;
      tile_coords(JG, tile, c0, c2);
      const int n = JG.n, mt = JG.mt;
      const int n_stages = mt / R;
      const int nvp = part ? 2 * mt - n : 0;  // this half's virtual rows
      const int count = CONTIG ? min(TS, JG.n_sys - c0) : min(TS, JG.inner - c0);
      // this lane's scratch: row k at + k 16 PW (all factors: component c of
      // row k at + (3 k + c) 16, so that each component is one 128-byte line)
      F *const x2w = JG.scratch + (long long)tile * 2 * mt * TS * PW +
                     (FM == 2 ? part * mt * TS * PW + sys : (part * mt * TS + sys) * PW);
      const bool flip = (ti & 1) != 0;
      const int free_blocks = NB - n_prev;  // blocks the previous tile never used
      // bulk layout: where this lane's r-th row of a stage sits in its half's
      // tile.  The window of a line (x) or a row (strided) starts at the
      // 16-byte chunk holding its first element; the element's offset in that
      // chunk is the shift.  Stages start at multiples of R rows (R a multiple
      // of the chunk), so a tile's shifts repeat from stage to stage.
      int ldm[LD == 1 ? R : 1];
      bool by_groups = false;
      if constexpr (LD == 1)
        by_groups = JG.grp > 0 && (CONTIG ? (c0 / TS < JG.tail) : (c2 != JG.tail));
      if (LD == 1 && by_groups) {
        // the group view's classes (see the feeding warp)
        const int gq = JG.grp, lgq = gq == 4 ? 2 : (gq == 2 ? 1 : 3);
        const int cpe = gq == 4 ? CP4 : CP2;
        if constexpr (CONTIG) {
          const int sub = sys & (gq - 1), k = sys >> lgq;
          const int sh = (sub * (n & (G::EPC - 1))) & (G::EPC - 1);
          const int b = part * BOXL + sub * cpe + k * PL + sh;
#pragma unroll
          for (int r = 0; r < R; ++r) ldm[r] = b + (part ? (R - 1 - r) : r);
        } else {
          const int q0 = (int)(((long long)c2 * n) & (gq - 1));
          const int im = JG.inner & (G::EPC - 1);
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int rr = part ? (R - 1 - r) : r;
            const int sub = (q0 + rr) & (gq - 1);
            ldm[r] = part * BOXL + sub * cpe + (rr >> lgq) * PS + ((sub * im) & (G::EPC - 1)) +
                     sys;
          }
        }
      } else if constexpr (LD == 1) {
        if constexpr (CONTIG) {
          const int sh = (int)(((long long)(c0 + sys) * n) & (G::EPC - 1));
#pragma unroll
          for (int r = 0; r < R; ++r)
            ldm[r] = part * BOXL + G::line_off(sys) + sh + (part ? (R - 1 - r) : r);
        } else {
          const int s0 = (int)(((long long)c2 * JG.inner * n) & (G::EPC - 1));
          const int im = JG.inner & (G::EPC - 1);
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int rr = part ? (R - 1 - r) : r;
            ldm[r] = part * BOXL + rr * PS + ((s0 + rr * im) & (G::EPC - 1)) + sys;
          }
        }
      }
      Carry<F> c;
      c.zero();
      for (int g = 0; g < n_stages; ++g) {
        if (!__all_sync(0xffffffffu, mbar_wait(&full[slot], phase))) {
          fail = 1;
          break;
        }
        const F *v = ring + slot * SE;
        F a[R][6];
        if constexpr (LD == 1) {
#pragma unroll
          for (int r = 0; r < R; ++r)
#pragma unroll
            for (int q = 0; q < 6; ++q) a[r][q] = v[ldm[r] + q * 2 * BOXL];
        } else if constexpr (CONTIG) {
          // the lower half runs its tile backwards: the pair's odd row first
#pragma unroll
          for (int q = 0; q < 6; ++q)
#pragma unroll
            for (int j = 0; j < R / 2; ++j) {
              const V2 pv = *reinterpret_cast<const V2 *>(v + ld[j] + q * 2 * BOX);
              a[2 * j][q] = part ? pv.y : pv.x;
              a[2 * j + 1][q] = part ? pv.x : pv.y;
            }
        } else {
#pragma unroll
          for (int r = 0; r < R; ++r)
#pragma unroll
            for (int q = 0; q < 6; ++q) a[r][q] = v[ld[r] + q * 2 * BOX];
        }
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
        if (++slot == ST) {
          slot = 0;
          phase ^= 1u;
        }
        F u[R], w[R], y[R];
#pragma unroll
        for (int r = 0; r < R; ++r)
          fwd_row_lean(a[r][0], a[r][1], a[r][2], a[r][3], a[r][4], a[r][5], c, u[r], w[r],
                       y[r]);
        if constexpr (FM != 2) {  // du2 (and dw2, and x2) into TMEM
        constexpr int VPR = tmem_values_per_row<F, FM>();
        uint32_t tv[G::kCols];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          put_bits<F>(tv, r * CW * VPR, u[r]);
          if (VPR >= 2) put_bits<F>(tv, r * CW * VPR + CW, w[r]);
          if (VPR == 3) put_bits<F>(tv, r * CW * VPR + 2 * CW, y[r]);
        }
        // wait (lane 0, bounded) until the previous tile has read this block
        const int need = (ti - 1) * 65536 + max(0, g + 1 - free_blocks);
        int ok = 1;
        if (lane == 0 && seen < need) {
          seen = ld_acquire_shared(&prog[cons]);
          if (seen < need) {
            const unsigned long long t0 = global_ns();
            for (;;) {
              __nanosleep(32);
              seen = ld_acquire_shared(&prog[cons]);
              if (seen >= need) break;
              if (stop[cons] != 0) {
                ok = 2;
                break;
              }
              if (global_ns() - t0 > 2000000000ull) {
                ok = 0;
                break;
              }
            }
          }
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (ok != 1) {
          fail = ok == 0 ? 1 : 2;
          break;
        }
        tmem_fence_after_sync();
        const int blk = flip ? NB - 1 - g : g;
        if constexpr (G::kCols == 48)
          tmem_store48(taddr + (uint32_t)(blk * G::kCols), reinterpret_cast<uint32_t(&)[48]>(tv));
        else if constexpr (G::kCols == 32)
          tmem_store32(taddr + (uint32_t)(blk * G::kCols), reinterpret_cast<uint32_t(&)[32]>(tv));
        else
          tmem_store16(taddr + (uint32_t)(blk * G::kCols), reinterpret_cast<uint32_t(&)[16]>(tv));
        }
        F *const x2g = x2w + g * R * TS * PW;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          if constexpr (FM == 3) {
            // nothing leaves the SM: x2 went to TMEM with the factors
          } else if constexpr (FM == 2) {
            st_hint(x2g + (3 * r) * TS, u[r], pol_x2);
            st_hint(x2g + (3 * r + 1) * TS, w[r], pol_x2);
            st_hint(x2g + (3 * r + 2) * TS, y[r], pol_x2);
          } else if constexpr (FM == 1) {
            V2 pv;
            pv.x = w[r];
            pv.y = y[r];
            st_hint(reinterpret_cast<V2 *>(x2g + r * TS * 2), pv, pol_x2);
          } else {
            st_hint(x2g + r * TS, y[r], pol_x2);
          }
        }
      }
      n_prev = n_stages;
      if (fail) break;
      if (sys < count)
        bad |= !(isfinite(c.u1) && isfinite(c.u2) && isfinite(c.w1) && isfinite(c.w2) &&
                 isfinite(c.y1) && isfinite(c.y2));
      // hand the carries to the back-substitution warp; the x2 stores above
      // are read next by its bulk copies (async proxy)
      F *const h = hand + (ti & 1) * 6 * 32 + lane;
      h[0] = c.u1;
      h[32] = c.u2;
      h[64] = c.w1;
      h[96] = c.w2;
      h[128] = c.y1;
      h[160] = c.y2;
      fence_async_global();
      tmem_fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(&hfull[ti & 1]);
    }
    if (fail) {
      stop[cons] = 1;  // the producer issues nothing more
      // wake the back-substitution warp if it waits for this tile
      __syncwarp();
      if (lane == 0) mbar_arrive(&hfull[ti & 1]);
      // drain what may still land in the ring (bounded waits)
      for (int k = 0; k < ST; ++k) {
        if (!mbar_wait(&full[slot], phase)) break;
        if (++slot == ST) {
          slot = 0;
          phase ^= 1u;
        }
      }
      if (fail == 1 && lane == 0) atomicOr(status_word, STATUS_TIMEOUT_BIT);
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(status_word, STATUS_ZERO_PIVOT_BIT);
  } else {
    // ========================= back-substitution ============================
    // Along x the results of two steps leave together as one tile of 2R rows
    // (128-byte rows, 128-byte swizzle) per half, written two rows at a time
    // (st2 below; an odd step's offsets are an even step's ^ R: its rows are
    // the other R of the tile).  A last step without a partner uses R-row
    // tiles (64-byte swizzle, offsets st1).
    int st1[R], st2[R / 2];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (CONTIG) {
        const int rs = part ? r : (R - 1 - r);
        st1[r] = part * 2 * BOX + sys * R + ((rs / EPC) ^ ((sys >> 1) & 3)) * EPC + rs % EPC;
      } else {
        st1[r] = 0;
      }
    }
    // rows 2j and 2j+1 of a step share a 16-byte chunk of the 2R-row tile:
    // st2[j] is the chunk's even row (the upper half writes its rows downwards)
#pragma unroll
    for (int j = 0; j < R / 2; ++j) {
      if (CONTIG) {
        const int rr = part ? 2 * j : (2 * R - 2 - 2 * j);
        st2[j] = part * 2 * BOX + sys * 2 * R + ((rr / EPC) ^ (sys & 7)) * EPC + rr % EPC;
      } else {
        st2[j] = 0;
      }
    }
    const bool drop = (flags & 1) != 0;
    const uint64_t pol_out = l2_policy_first();  // written once
    const uint64_t pol_rb = l2_policy_first();   // read once (then dropped)
    int r_slot = 0, o_buf = 0, cursor = 0;
    unsigned r_phase = 0;
    Geo JG;
    load_geo(job_of(gw, cursor), JG);
    long long r_issued = 0, r_consumed = 0;
    int fail = 0;
    for (int ti = 0; ti < my_tiles && !fail; ++ti) {
      const int t = gw + ti * tw;
      const TmemJob<F> *J = job_of(t, cursor);
      if (J != JG.J) load_geo(J, JG);
      const int tile = t - JG.tile_base;
      int c0, c2;
      tile_coords(JG, tile, c0, c2);
      const int n = JG.n, mt = JG.mt, inner = JG.inner;
      const int n_stages = mt / R;
      const int count = CONTIG ? min(TS, JG.n_sys - c0) : min(TS, inner - c0);
      const bool active = sys < count;
      F *const x2t = JG.scratch + (long long)tile * 2 * mt * TS * PW;  // [2][m][16][PW]
      const bool flip = (ti & 1) != 0;

      // the forward sweep of this tile: factors in TMEM, x2 in the buffer
      if (!__all_sync(0xffffffffu, mbar_wait(&hfull[ti & 1], (unsigned)(ti >> 1) & 1u))) {
        fail = 1;
        break;
      }
      if (stop[cons] != 0) {
        fail = 2;
        break;
      }
      tmem_fence_after_sync();

      // read-back copies of x2 (most recent rows first)
      constexpr unsigned kBlock = (unsigned)(R * TS * PW * sizeof(F));  // one half, one stage
      int ri_slot = r_slot;
      auto rissue = [&](int s) {
        if (s >= n_stages) return;
        if (lane == 0) {
          const int k0 = mt - (s + 1) * R;
          F *dst = xr + ri_slot * XE;
          mbar_expect_tx(&rfull[ri_slot], 2u * kBlock);
          bulk_load_hint(dst, x2t + (long long)k0 * TS * PW, kBlock, &rfull[ri_slot], pol_rb);
          bulk_load_hint(dst + R * TS * PW, x2t + (long long)(mt + k0) * TS * PW, kBlock,
                         &rfull[ri_slot], pol_rb);
        }
        ++r_issued;
        if (++ri_slot == XST) ri_slot = 0;
      };
      if constexpr (FM != 3)  // factor mode 3 keeps x2 in TMEM: nothing to read back
        for (int s = 0; s < XST; ++s) rissue(s);

      // ---------------------------- interface -------------------------------
      const F *const h = hand + (ti & 1) * 6 * 32 + lane;
      Carry<F> c;
      c.u1 = h[0];
      c.u2 = h[32];
      c.w1 = h[64];
      c.w2 = h[96];
      c.y1 = h[128];
      c.y2 = h[160];
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

      // ---------------------------- backward --------------------------------
      // step s: elimination rows k in [m - (s+1) R, m - s R) of both halves
      for (int s = 0; s < n_stages; ++s) {
        const int g = n_stages - 1 - s;  // the forward stage being undone
        const int blk = flip ? NB - 1 - g : g;
        uint32_t tv[G::kCols];
        if constexpr (FM != 2) {
          if constexpr (G::kCols == 48)
            tmem_load48(taddr + (uint32_t)(blk * G::kCols), reinterpret_cast<uint32_t(&)[48]>(tv));
          else if constexpr (G::kCols == 32)
            tmem_load32(taddr + (uint32_t)(blk * G::kCols), reinterpret_cast<uint32_t(&)[32]>(tv));
          else
            tmem_load16(taddr + (uint32_t)(blk * G::kCols), reinterpret_cast<uint32_t(&)[16]>(tv));
          // the block is free for the next tile's forward sweep
          tmem_fence_before_sync();
          __syncwarp();
          if (lane == 0) st_release_shared(&prog[cons], ti * 65536 + s + 1);
        }
        if constexpr (FM != 3) {
          if (!__all_sync(0xffffffffu, mbar_wait(&rfull[r_slot], r_phase))) {
            fail = 1;
            break;
          }
        }
        const F *xsrc = xr + r_slot * XE +
                        (FM == 2 ? part * R * TS * PW + sys : (part * R * TS + sys) * PW);
        F xs[R], du[R], dw[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int j = R - 1 - r;  // row inside the stage block
          if constexpr (FM == 3) {
            du[r] = get_bits<F>(tv, j * CW * 3);
            dw[r] = get_bits<F>(tv, j * CW * 3 + CW);
            xs[r] = get_bits<F>(tv, j * CW * 3 + 2 * CW);
          } else if constexpr (FM == 2) {
            du[r] = xsrc[(3 * j) * TS];
            dw[r] = xsrc[(3 * j + 1) * TS];
            xs[r] = xsrc[(3 * j + 2) * TS];
          } else if constexpr (FM == 1) {
            const V2 pv = *reinterpret_cast<const V2 *>(xsrc + j * TS * 2);
            dw[r] = pv.x;
            xs[r] = pv.y;
            du[r] = get_bits<F>(tv, j * CW);
          } else {
            xs[r] = xsrc[j * TS];
            du[r] = get_bits<F>(tv, j * CW * 2);
            dw[r] = get_bits<F>(tv, j * CW * 2 + CW);
          }
        }
        if (CONTIG && (s & 1) == 0 && lane == 0) bulk_wait_read<1>();  // buffer o_buf is free
        fence_async_shared();
        __syncwarp();
        if constexpr (FM != 3) {
          ++r_consumed;
          rissue(s + XST);  // refills the slot just read (ri_slot == r_slot here)
          if (++r_slot == XST) {
            r_slot = 0;
            r_phase ^= 1u;
          }
        }
        // the stage's block of each half is dead: drop its 128-byte lines
        constexpr int kLines = (int)(kBlock / 128);
        for (int l = sys; drop && l < kLines; l += TS)
          discard_l2_line(reinterpret_cast<const unsigned char *>(
                              x2t + (long long)(part * mt + mt - (s + 1) * R) * TS * PW) +
                          l * 128);
        F xk[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          xk[r] = xs[r] - dw[r] * xb - du[r] * xa;
          xb = xa;
          xa = xk[r];
        }
        if (CONTIG && !JG.tma) {
          // misaligned grid (no TMA): the step's results go through the
          // shared tile and leave in runs of a line's R rows, R consecutive
          // lanes a run, instead of one scattered element per lane
          // (lane: row rr = lane % R of lines a + (32 / R) j, one pointer
          // step a line group; the rows of each half checked once)
          F *const ob = obuf;
#pragma unroll
          for (int r = 0; r < R; ++r) ob[st1[r]] = xk[r];
          __syncwarp();
          constexpr int LPI = 32 / R;  // lines a warp instruction writes
          const int a0 = lane / R, rr = lane % R;
          F *const xl = JG.x + (long long)(c0 + a0) * n;
          const long long lstep = (long long)LPI * n;
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int row = h ? (mt + s * R + rr) : (mt - (s + 1) * R + rr);
            if (row < n) {
#pragma unroll
              for (int j = 0; j < TS / LPI; ++j) {
                const int l = a0 + LPI * j;
                if (c0 + l < JG.n_sys)
                  xl[j * lstep + row] =
                      ob[h * 2 * BOX + l * R + ((rr / EPC) ^ ((l >> 1) & 3)) * EPC + rr % EPC];
              }
            }
          }
          __syncwarp();
        } else if (CONTIG) {
          F *const ob = obuf + o_buf * 4 * BOX;
          if ((s & 1) == 0 && s + 1 == n_stages) {  // a last step without a partner
#pragma unroll
            for (int r = 0; r < R; ++r) ob[st1[r]] = xk[r];
            fence_async_shared();
            __syncwarp();
            if (lane == 0) {
              tma_store_2d_hint(&J->maps[5], ob, mt - (s + 1) * R, c0, pol_out);
              if (mt + s * R < n)
                tma_store_2d_hint(&J->maps[5], ob + 2 * BOX, mt + s * R, c0, pol_out);
              bulk_commit();
            }
            // the next tile writes the other buffer: the wait before each
            // even step leaves one store group in flight, and that group may
            // still be reading this one
            o_buf ^= 1;
          } else {
            const int odd = (s & 1) ? R : 0;
#pragma unroll
            for (int j = 0; j < R / 2; ++j) {
              V2 pv;
              pv.x = part ? xk[2 * j] : xk[2 * j + 1];
              pv.y = part ? xk[2 * j + 1] : xk[2 * j];
              *reinterpret_cast<V2 *>(ob + (st2[j] ^ odd)) = pv;
            }
            if (odd) {  // steps s - 1 and s: rows [mt - (s+1) R, mt - (s-1) R) of each half
              fence_async_shared();
              __syncwarp();
              if (lane == 0) {
                tma_store_2d_hint(&J->maps[6], ob, mt - (s + 1) * R, c0, pol_out);
                if (mt + (s - 1) * R < n)
                  tma_store_2d_hint(&J->maps[6], ob + 2 * BOX, mt + (s - 1) * R, c0, pol_out);
                bulk_commit();
              }
              o_buf ^= 1;
            }
          }
        } else if (active) {
          // the upper half runs towards row 0, the lower half towards row n - 1
          const int row0 = part ? (mt + s * R) : (mt - 1 - s * R);
          const long long step = part ? (long long)inner : -(long long)inner;
          F *const p = JG.x + (long long)c2 * inner * n + c0 + sys + (long long)row0 * inner;
          if (part == 0 || mt + (s + 1) * R <= n) {
#pragma unroll
            for (int r = 0; r < R; ++r) st_hint(p + r * step, xk[r], pol_out);
          } else {  // the lower half's last stages end in virtual rows
#pragma unroll
            for (int r = 0; r < R; ++r)
              if (row0 + r < n) st_hint(p + r * step, xk[r], pol_out);
          }
        }
      }
      if (lane == 0) st_release_shared(&prog[cons], (ti + 1) * 65536);
    }
    if (fail) {
      stop[cons] = 1;
      // drain the read-back copies in flight (bounded waits)
      for (; r_consumed < r_issued; ++r_consumed) {
        if (!mbar_wait(&rfull[r_slot], r_phase)) break;
        if (++r_slot == XST) {
          r_slot = 0;
          r_phase ^= 1u;
        }
      }
      if (fail == 1 && lane == 0) atomicOr(status_word, STATUS_TIMEOUT_BIT);
    }
    if (CONTIG && lane == 0) bulk_wait<0>();
  }

  // the forward and back-substitution warps are done with Tensor Memory:
  // warp 0 frees it
  tmem_fence_before_sync();
  asm volatile("bar.sync 1, %0;\n" ::"n"(64 * NCONS) : "memory");
  tmem_fence_after_sync();
  if (warp == 0) tmem_dealloc(tmem_base, kTmemCols);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
template <typename F>
bool encode(CUtensorMap *m, const F *ptr, const Lines &L, bool contig, int R,
            bool wide = false) {
  auto fn = tensor_map_encoder();
  if (fn == nullptr) return false;
  const CUtensorMapDataType dt =
      sizeof(F) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  CUresult r;
  if (contig) {
    const cuuint64_t dims[2] = {(cuuint64_t)L.n, (cuuint64_t)L.n_sys};
    const cuuint64_t strides[1] = {(cuuint64_t)L.n * sizeof(F)};
    const cuuint32_t box[2] = {(cuuint32_t)(wide ? 2 * R : R), (cuuint32_t)TS};
    const cuuint32_t es[2] = {1, 1};
    r = fn(m, dt, 2, const_cast<F *>(ptr), dims, strides, box, es,
           CU_TENSOR_MAP_INTERLEAVE_NONE,
           wide ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
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

// Is this line set one the kernel takes (apart from the buffer)?  Also gives
// whether it needs the dw2-in-buffer mode.
template <typename F>
bool shape_ok(const Lines &L, bool contig, int &fmode) {
  if (contig ? L.inner != 1 : L.inner <= 1) return false;
  const long long R =
      contig ? tmem_rows_per_stage<F, true>() : tmem_rows_per_stage<F, false>();
  const long long mt = split_row<F>(L, contig);
  if (L.n - mt < 2) return false;  // two real rows per half
  const long long stages = mt / R;
  // all three values fit 10 stages, but with all 10 in use the next tile's
  // forward sweep waits for every block in turn (160^3 FP64: 1-6% slower than
  // factor mode 0); at 8 stages it gains (128^3 FP64: 11-14%; FP32 along x
  // 1-3% up to 256 rows).  FP32 along y and z, where x2 costs only 4 B/pt,
  // measured 5-12% slower at 6-7 stages (192^3, 224^3): there up to 4 stages.
  const long long cap_all =
      (sizeof(F) == 4 && !contig) ? 4 : kTmemCols / tmem_cols_per_stage<F, 3>() - 2;
  const long long cap_both = kTmemCols / tmem_cols_per_stage<F, 0>();
  const long long cap_du = kTmemCols / tmem_cols_per_stage<F, 1>();
  // PENTA_TMEM_FM3=0: short lines too send x2 through the buffer (measurement)
  static const bool fm3_off = [] {
    const char *e = std::getenv("PENTA_TMEM_FM3");
    return e != nullptr && e[0] == '0';
  }();
  fmode = stages > cap_du ? 2 : stages > cap_both ? 1 : (stages <= cap_all && !fm3_off) ? 3 : 0;
  // every global offset is formed in 64 bits; line, run and tile indices (and
  // the TMA coordinates made of them) must stay below 2^31
  if (L.n_sys >= (1LL << 31) - TS || tile_count(L, contig) >= (1LL << 31)) return false;
  return true;
}

// Bulk-copy loads apply when every array starts on a 16-byte boundary (any
// row stride).
template <typename F> bool bulk_ok(const SolveArgs<F> &a) {
  const void *ptrs[6] = {a.ds, a.dl, a.d, a.du, a.dw, a.x};
  for (const void *p : ptrs)
    if (reinterpret_cast<uintptr_t>(p) % 16 != 0) return false;
  return true;
}

// TMA applies when the row stride and every array are 16-byte aligned.
template <typename F> bool tma_ok(const SolveArgs<F> &a, bool contig) {
  if (tensor_map_encoder() == nullptr) return false;
  if (contig ? (a.L.n * sizeof(F)) % 16 != 0 : (a.L.inner * sizeof(F)) % 16 != 0) return false;
  const void *ptrs[6] = {a.ds, a.dl, a.d, a.du, a.dw, a.x};
  for (const void *p : ptrs)
    if (reinterpret_cast<uintptr_t>(p) % 16 != 0) return false;
  return true;
}

template <typename F> size_t job_scratch_bytes(const Lines &L, bool contig, int fmode) {
  return (size_t)tile_count(L, contig) * 2 * (size_t)split_row<F>(L, contig) * TS *
         (fmode == 2 ? 3 : fmode == 1 ? 2 : fmode == 3 ? 0 : 1) * sizeof(F);
}

// The pitched layout filled by 16-byte cp.async copies: the default for
// misaligned rows or runs whose arrays start on 16-byte boundaries, unless
// PENTA_TMEM_LOADS names another loader.
template <typename F> bool chunk_loads(const SolveArgs<F> &a) {
  const char *e = std::getenv("PENTA_TMEM_LOADS");
  if (e != nullptr && (!std::strcmp(e, "bulk") || !std::strcmp(e, "group") ||
                       !std::strcmp(e, "element")))
    return false;
  return bulk_ok<F>(a);
}

// The group view of a grid whose rows (x) or runs (strided) are not 16-byte
// aligned: `grp` consecutive lines (x) or rows (strided) form a 16-byte
// periodic group, so maps over {grp * stride, groups} are valid tensor maps.
// Returns grp, or 0 when the view does not apply (or bulk copies are forced).
template <typename F> int group_size(const SolveArgs<F> &a, bool contig) {
  const char *e = std::getenv("PENTA_TMEM_LOADS");
  if (e == nullptr || std::strcmp(e, "group") != 0) return 0;
  if (!bulk_ok<F>(a) || tma_ok<F>(a, contig) || tensor_map_encoder() == nullptr) return 0;
  const long long m = contig ? a.L.n : a.L.inner;
  const long long bytes = m * (long long)sizeof(F);
  const int g = bytes % 16 == 0 ? 1 : (bytes % 8 == 0 ? 2 : (bytes % 4 == 0 ? 4 : 8));
  if (g > 4 || g * m >= (1LL << 31)) return 0;
  const long long groups = contig ? a.L.n_sys / g : a.L.n * (a.L.n_sys / a.L.inner) / g;
  if (groups < 1 || groups >= (1LL << 31)) return 0;
  return g;
}

template <typename F>
bool encode_groups(CUtensorMap *m, const F *ptr, const Lines &L, bool contig, int g, int R) {
  auto fn = tensor_map_encoder();
  if (fn == nullptr) return false;
  constexpr int EPC = 16 / (int)sizeof(F);
  const CUtensorMapDataType dt =
      sizeof(F) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const long long stride = contig ? L.n : L.inner;
  const long long groups = contig ? L.n_sys / g : L.n * (L.n_sys / L.inner) / g;
  const cuuint64_t dims[2] = {(cuuint64_t)(g * stride), (cuuint64_t)groups};
  const cuuint64_t strides[1] = {(cuuint64_t)(g * stride) * sizeof(F)};
  const cuuint32_t box[2] = {(cuuint32_t)(contig ? R + EPC : TS + EPC),
                             (cuuint32_t)(contig ? TS / g : R / g)};
  const cuuint32_t es[2] = {1, 1};
  return fn(m, dt, 2, const_cast<F *>(ptr), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            contig ? CU_TENSOR_MAP_L2_PROMOTION_L2_256B : CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <typename F>
bool fill_job(TmemJob<F> &J, const SolveArgs<F> &a, bool contig, F *scratch, int tile_base,
              int loads = 0) {
  std::memset(&J, 0, sizeof(J));
  const int R = contig ? tmem_rows_per_stage<F, true>() : tmem_rows_per_stage<F, false>();
  const F *ptrs[6] = {a.ds, a.dl, a.d, a.du, a.dw, a.x};
  J.tma = tma_ok<F>(a, contig) ? 1 : 0;
  J.bulk = bulk_ok<F>(a) ? 1 : 0;
  for (int q = 0; q < 6; ++q) {
    J.arr[q] = ptrs[q];
    if (J.tma && !encode<F>(&J.maps[q], ptrs[q], a.L, contig, R)) J.tma = 0;
  }
  if (J.tma && contig && !encode<F>(&J.maps[6], a.x, a.L, contig, R, true)) J.tma = 0;
  J.grp = 0;
  J.tail = contig ? 0x7fffffff : -1;
  J.chunks = 0;
  if (loads == 1 && chunk_loads<F>(a)) {
    J.chunks = 1;
  } else if (loads == 1) {  // pitched layout: the group view where it applies
    const int g = group_size<F>(a, contig);
    bool ok = g > 0;
    for (int q = 0; ok && q < 6; ++q) ok = encode_groups<F>(&J.maps[q], ptrs[q], a.L, contig, g, R);
    if (ok) {
      J.grp = g;
      if (contig) {
        if (a.L.n_sys % g != 0) J.tail = (int)(a.L.n_sys / g * g / TS);
      } else {
        const long long outer = a.L.n_sys / a.L.inner;
        if ((a.L.n * outer) % g != 0) J.tail = (int)(outer - 1);
      }
    }
  }
  J.x = a.x;
  J.scratch = scratch;
  J.n = (int)a.L.n;
  J.mt = (int)split_row<F>(a.L, contig);
  J.inner = (int)a.L.inner;
  J.tpr = contig ? 1 : (int)((a.L.inner + TS - 1) / TS);
  J.n_sys = (int)a.L.n_sys;
  J.n_tiles = (int)tile_count(a.L, contig);
  J.tile_base = tile_base;
  return true;
}

template <typename F, bool CONTIG, int FM, int ST, int XST, int LD, bool BATCH>
cudaError_t tmem_launch_raw(const TmemJob<F> &job1, const TmemJob<F> *jobs, int n_jobs,
                            int total_tiles, int flags, int sm_count, int *status,
                            cudaStream_t stream) {
  using G = TmemGeom<F, CONTIG, FM, ST, XST, LD>;
  auto kern = tmem_thomas_kernel<F, CONTIG, FM, ST, XST, LD, BATCH>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)G::kSmem);
  if (err != cudaSuccess) return err;
  const int need = (total_tiles + NCONS - 1) / NCONS;
  const int grid = need < sm_count ? need : sm_count;
  if (grid <= 0) return cudaSuccess;
  // launched with programmatic stream serialization (see griddepcontrol in the
  // kernel): at most one CTA per SM, all resident at once, so an early
  // dependent only takes SMs this grid has left
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(96 * NCONS);
  cfg.dynamicSmemBytes = G::kSmem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  err = cudaLaunchKernelEx(&cfg, kern, job1, jobs, n_jobs, total_tiles, flags, status);
  if (err != cudaSuccess) return err;
  return cudaGetLastError();
}

template <typename F, bool CONTIG, int FM, int ST, int XST, int LD> int tmem_occ() {
  using G = TmemGeom<F, CONTIG, FM, ST, XST, LD>;
  auto kern = tmem_thomas_kernel<F, CONTIG, FM, ST, XST, LD, false>;
  int blocks = 0;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)G::kSmem) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, 96 * NCONS, G::kSmem) !=
          cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return blocks;
}

}  // namespace

// (type, contiguous, factor mode, forward stages, read-back stages, loads);
// for each (type, layout, mode, loads) the first variant is the default.
// Batched launches use the default variants.  Along x in FP64 two forward
// stages beat three: fewer 64-byte requests in flight per line keep HBM row
// hits up (measured at 256^3 and 512^3); FP32 along x, with 16 rows a stage,
// and the strided directions want three.  Strided FP64 with both factors in
// TMEM keeps four read-back stages: the autotuner times three ~1% faster on
// back-to-back solves of one direction at 256^3 (y 153.5 / z 156.0 against
// 155.5 / 157.4 us), but in the ADI loop (x, y, z launches overlapping
// through dependent launches) the y solve measured 0.167 ms with three
// against 0.157-0.158 ms with four.  The bulk-load variants (loads = 1)
// have wider stages, so some take fewer of them to fit shared memory.
#define PENTA_TMEM_CONFIGS(X)   \
  X(double, true, 0, 2, 4, 0)   \
  X(double, true, 0, 3, 4, 0)   \
  X(double, true, 0, 3, 3, 0)   \
  X(double, false, 0, 3, 4, 0)  \
  X(double, false, 0, 3, 3, 0)  \
  X(double, false, 0, 2, 4, 0)  \
  X(double, true, 1, 2, 3, 0)   \
  X(double, true, 1, 3, 2, 0)   \
  X(double, false, 1, 3, 4, 0)  \
  X(double, true, 2, 2, 2, 0)   \
  X(double, false, 2, 3, 2, 0)  \
  X(float, true, 0, 3, 4, 0)    \
  X(float, true, 0, 2, 4, 0)    \
  X(float, false, 0, 3, 4, 0)   \
  X(float, false, 0, 4, 3, 0)   \
  X(float, true, 1, 2, 3, 0)    \
  X(float, true, 1, 3, 2, 0)    \
  X(float, false, 1, 3, 4, 0)   \
  X(float, true, 2, 2, 2, 0)    \
  X(float, false, 2, 3, 2, 0)   \
  X(double, true, 0, 2, 4, 1)   \
  X(double, false, 0, 3, 3, 1)  \
  X(double, true, 1, 2, 2, 1)   \
  X(double, false, 1, 2, 4, 1)  \
  X(double, true, 2, 2, 1, 1)   \
  X(double, false, 2, 2, 2, 1)  \
  X(float, true, 0, 2, 4, 1)    \
  X(float, false, 0, 2, 4, 1)   \
  X(float, true, 1, 2, 2, 1)    \
  X(float, false, 1, 2, 4, 1)   \
  X(float, true, 2, 2, 1, 1)    \
  X(float, false, 2, 2, 2, 1)   \
  X(double, true, 3, 2, 1, 0)   \
  X(double, true, 3, 3, 1, 0)   \
  X(double, false, 3, 3, 1, 0)  \
  X(double, false, 3, 2, 1, 0)  \
  X(float, true, 3, 3, 1, 0)    \
  X(float, true, 3, 2, 1, 0)    \
  X(float, false, 3, 3, 1, 0)   \
  X(float, false, 3, 4, 1, 0)   \
  X(double, true, 3, 2, 1, 1)   \
  X(double, false, 3, 3, 1, 1)  \
  X(float, true, 3, 2, 1, 1)    \
  X(float, false, 3, 2, 1, 1)

template <typename F> const std::vector<TmemConfig> &tmem_configs() {
  static const std::vector<TmemConfig> v = [] {
    std::vector<TmemConfig> out;
#define PENTA_X(FT_, C_, W_, ST_, XST_, LD_)                                             \
  if (std::is_same<F, FT_>::value)                                                       \
    out.push_back(TmemConfig{C_, W_, ST_, XST_, TmemGeom<FT_, C_, W_, ST_, XST_, LD_>::R, \
                             TmemGeom<FT_, C_, W_, ST_, XST_, LD_>::kSmem, LD_});
    PENTA_TMEM_CONFIGS(PENTA_X)
#undef PENTA_X
    return out;
  }();
  return v;
}

template <typename F> int tmem_occupancy(const TmemConfig &c) {
#define PENTA_X(FT_, C_, W_, ST_, XST_, LD_)                                             \
  if (std::is_same<F, FT_>::value && c.contig == C_ && c.fmode == W_ && c.stages == ST_ && \
      c.xstages == XST_ && c.loads == LD_)                                               \
    return tmem_occ<FT_, C_, W_, ST_, XST_, LD_>();
  PENTA_TMEM_CONFIGS(PENTA_X)
#undef PENTA_X
  return 0;
}

template <typename F> bool tmem_shape(const Lines &L, bool contig, int &fmode) {
  return shape_ok<F>(L, contig, fmode);
}

template <typename F> size_t tmem_scratch_bytes(const Lines &L, bool contig, int fmode) {
  return job_scratch_bytes<F>(L, contig, fmode);
}

// Which stage layout a grid's loads use.  0: TMA tiles for aligned rows or
// runs; element copies (cp.async, 8 or 4 bytes) for misaligned ones whose
// arrays do not start on 16-byte boundaries, or with
// PENTA_TMEM_LOADS=element.  1, the pitched layout (one 16-byte chunk wider
// per row or line): by default for misaligned rows or runs, filled by
// 16-byte cp.async copies of the aligned superset of each row or line
// (chunk_loads; 255^3 FP64 x 229, y 177, z 183 us against 284 / 237 / 241
// with element copies -- a quarter to a half of their copy instructions).
// For measurement: PENTA_TMEM_LOADS=group fills it with TMA boxes of the
// group view (group_size), =bulk with one cp.async.bulk per row or line (any
// grid).  Both measured slower than element copies (255^3 FP64: x 354 / 736
// us, y 271 / 388 us): every misaligned 128-byte row spans two or three L2
// lines, the group boxes along x re-read their overlap chunk (1.5x DRAM reads
// under evict-first loads), and each cp.async.bulk is a TMA request of 80-144
// bytes, of which the TMA unit takes about one per 18 cycles per SM.
template <typename F> int tmem_loads(const SolveArgs<F> &a, bool contig) {
  const char *e = std::getenv("PENTA_TMEM_LOADS");
  if (e != nullptr && !std::strcmp(e, "bulk")) return bulk_ok<F>(a) ? 1 : 0;
  if (e != nullptr && !std::strcmp(e, "group")) return group_size<F>(a, contig) > 0 ? 1 : 0;
  if (e != nullptr && !std::strcmp(e, "element")) return 0;
  return (chunk_loads<F>(a) && !tma_ok<F>(a, contig)) ? 1 : 0;
}

template <typename F> const char *tmem_loader(const SolveArgs<F> &a, bool contig) {
  if (tmem_loads<F>(a, contig) != 1) return "";
  if (chunk_loads<F>(a)) return " chunk";
  return group_size<F>(a, contig) > 0 ? " grp" : " bulk";
}

template <typename F>
bool tmem_supported(const SolveArgs<F> &a, bool contig, size_t usable_buf, int &fmode) {
  if (!tmem_shape<F>(a.L, contig, fmode)) return false;
  // factor mode 3 keeps everything on chip: it needs no buffer at all
  if (fmode != 3 && (a.scratch == nullptr || reinterpret_cast<uintptr_t>(a.scratch) % 16 != 0 ||
                     tmem_scratch_bytes<F>(a.L, contig, fmode) > usable_buf))
    return false;
  const void *ptrs[6] = {a.ds, a.dl, a.d, a.du, a.dw, a.x};
  for (const void *p : ptrs)  // element alignment (TMA needs 16 bytes; see tma_ok)
    if (reinterpret_cast<uintptr_t>(p) % sizeof(F) != 0) return false;
  return true;
}

// CTAs for an FP64 launch with dw2 in the buffer (factor mode 1) and many tiles
// per lane quarter: each quarter keeps about one tile of (dw2, x2) pairs live in
// L2 (written by the forward sweep, read back by the substitution), and once all
// quarters' live scratch outgrows about half the L2 -- the rest holding the
// streamed arrays -- it spills to HBM (at 512^3 FP64 the x solve moved 1.36x its
// algorithmic bytes with all 148 SMs).  At 512^3 FP64 (131 KB a tile, 28 tiles
// a quarter) 96 CTAs beat 148 by 5-7% along y and z (74 lose 13%); along x,
// with evict-first loads, 111 CTAs beat 148 by 5%.  With few tiles a quarter the
// lost parallelism costs more than the spill (FP32 1024 x 128 x 128, under two
// tiles a quarter: 20-40% slower capped), so the cap needs 8 tiles a quarter;
// FP32 and factor mode 2 (n = 1024 FP64: no gain) keep the full grid.
template <typename F>
int scratch_grid_cap(const SolveArgs<F> &a, const TmemConfig &c, long long tiles,
                     int sm_count) {
  if (sizeof(F) != 8 || c.fmode != 1 || tiles < 8LL * NCONS * sm_count) return sm_count;
  const long long tile_bytes =
      2 * split_row<F>(a.L, c.contig) * TS * 2 * (long long)sizeof(F);
  const long long budget = c.contig ? (58ll << 20) : (50ll << 20);
  const long long cap = budget / (NCONS * tile_bytes);
  const int floor_ctas = 2 * sm_count / 3;
  return cap >= sm_count ? sm_count : (cap < floor_ctas ? floor_ctas : (int)cap);
}

// flags bit 2: along x, an even stage prefetches the next stage's tiles into
// L2.  It pays only where the launch caps its CTAs to keep the (dw2, x2)
// scratch in L2 (FP64 512^3 along x: 1.61 against 1.65 ms); elsewhere it cost
// 0.5-3.5% (256^3, FP32, and the batched launches of uneven grids).
// PENTA_TMEM_XPREFETCH=0 turns it off, =1 on for every x launch (measurement).
int x_prefetch_flag(bool contig, bool capped) {
  static const int mode = [] {
    const char *e = std::getenv("PENTA_TMEM_XPREFETCH");
    return e == nullptr ? -1 : (e[0] == '0' ? 0 : 1);
  }();
  if (!contig || mode == 0) return 0;
  return (mode == 1 || capped) ? 4 : 0;
}

template <typename F>
cudaError_t launch_tmem(const SolveArgs<F> &a, const TmemConfig &c, int sm_count,
                        cudaStream_t stream) {
  TmemJob<F> J;
  if (!fill_job<F>(J, a, c.contig, static_cast<F *>(a.scratch), 0, c.loads))
    return cudaErrorInvalidValue;
  if (c.loads == 1 && !J.bulk) return cudaErrorInvalidValue;  // bulk loads need aligned arrays
  int flags = ((reinterpret_cast<uintptr_t>(a.scratch) % 128 == 0) ? 1 : 0);
  const int capped = scratch_grid_cap<F>(a, c, J.n_tiles, sm_count);
  flags |= x_prefetch_flag(c.contig, capped < sm_count);
  // streamed loads evict-first when the grid is capped, and for FP32 along x with
  // dw2 in the buffer (1024 x 128 x 128: 118 against 129 us with normal priority)
  if (capped < sm_count || (sizeof(F) == 4 && c.contig && c.fmode == 1)) flags |= 2;
  sm_count = capped;
#define PENTA_X(FT_, C_, W_, ST_, XST_, LD_)                                              \
  if (std::is_same<F, FT_>::value && c.contig == C_ && c.fmode == W_ && c.stages == ST_ &&  \
      c.xstages == XST_ && c.loads == LD_)                                                \
    return tmem_launch_raw<FT_, C_, W_, ST_, XST_, LD_, false>(                           \
        reinterpret_cast<const TmemJob<FT_> &>(J), nullptr, 1, J.n_tiles, flags, sm_count, \
        a.status, stream);
  PENTA_TMEM_CONFIGS(PENTA_X)
#undef PENTA_X
  return cudaErrorInvalidConfiguration;
}

// ---- batched launches -------------------------------------------------------
template <typename F> size_t tmem_job_bytes() { return sizeof(TmemJob<F>); }

template <typename F>
bool tmem_fill_jobs(const SolveArgs<F> *grids, int count, bool contig, int fmode, int loads,
                    unsigned char *device_base, void *host_jobs, size_t *scratch_offsets,
                    int *total_tiles) {
  TmemJob<F> *J = static_cast<TmemJob<F> *>(host_jobs);
  long long tiles = 0;
  for (int i = 0; i < count; ++i) {
    F *scratch = reinterpret_cast<F *>(device_base + scratch_offsets[i]);
    if (!fill_job<F>(J[i], grids[i], contig, scratch, (int)tiles, loads)) return false;
    tiles += J[i].n_tiles;
    if (tiles >= (1LL << 31)) return false;  // tile indices of one launch are 32-bit
  }
  *total_tiles = (int)tiles;
  (void)fmode;
  return true;
}

template <typename F>
cudaError_t launch_tmem_batch(const void *device_jobs, int n_jobs, int total_tiles, bool contig,
                              int fmode, int loads, bool discard, int sm_count, int *status,
                              cudaStream_t stream) {
  TmemJob<F> none;
  std::memset(&none, 0, sizeof(none));
  const TmemJob<F> *jobs = static_cast<const TmemJob<F> *>(device_jobs);
  // the load policy of single-grid launches (launch_tmem) on an uncapped grid:
  // evict-first streamed loads for FP32 along x with dw2 in the buffer
  const int flags = (discard ? 1 : 0) | ((sizeof(F) == 4 && contig && fmode == 1) ? 2 : 0) |
                    x_prefetch_flag(contig, false);
  // the default variant of each (layout, factor mode, loads)
  const std::vector<TmemConfig> &all = tmem_configs<F>();
  for (const TmemConfig &c : all) {
    if (c.contig != contig || c.fmode != fmode || c.loads != loads) continue;
#define PENTA_X(FT_, C_, W_, ST_, XST_, LD_)                                              \
  if (std::is_same<F, FT_>::value && c.contig == C_ && c.fmode == W_ && c.stages == ST_ &&  \
      c.xstages == XST_ && c.loads == LD_)                                                \
    return tmem_launch_raw<FT_, C_, W_, ST_, XST_, LD_, true>(                            \
        reinterpret_cast<const TmemJob<FT_> &>(none),                                     \
        reinterpret_cast<const TmemJob<FT_> *>(jobs), n_jobs, total_tiles, flags, sm_count, \
        status, stream);
    PENTA_TMEM_CONFIGS(PENTA_X)
#undef PENTA_X
  }
  return cudaErrorInvalidConfiguration;
}

template const std::vector<TmemConfig> &tmem_configs<double>();
template const std::vector<TmemConfig> &tmem_configs<float>();
template int tmem_occupancy<double>(const TmemConfig &);
template int tmem_occupancy<float>(const TmemConfig &);
template bool tmem_shape<double>(const Lines &, bool, int &);
template bool tmem_shape<float>(const Lines &, bool, int &);
template size_t tmem_scratch_bytes<double>(const Lines &, bool, int);
template size_t tmem_scratch_bytes<float>(const Lines &, bool, int);
template bool tmem_supported<double>(const SolveArgs<double> &, bool, size_t, int &);
template bool tmem_supported<float>(const SolveArgs<float> &, bool, size_t, int &);
template cudaError_t launch_tmem<double>(const SolveArgs<double> &, const TmemConfig &, int,
                                         cudaStream_t);
template cudaError_t launch_tmem<float>(const SolveArgs<float> &, const TmemConfig &, int,
                                        cudaStream_t);
template size_t tmem_job_bytes<double>();
template size_t tmem_job_bytes<float>();
template bool tmem_fill_jobs<double>(const SolveArgs<double> *, int, bool, int, int,
                                     unsigned char *, void *, size_t *, int *);
template bool tmem_fill_jobs<float>(const SolveArgs<float> *, int, bool, int, int,
                                    unsigned char *, void *, size_t *, int *);
template const char *tmem_loader<double>(const SolveArgs<double> &, bool);
template const char *tmem_loader<float>(const SolveArgs<float> &, bool);
template cudaError_t launch_tmem_batch<double>(const void *, int, int, bool, int, int, bool,
                                               int, int *, cudaStream_t);
template cudaError_t launch_tmem_batch<float>(const void *, int, int, bool, int, int, bool, int,
                                              int *, cudaStream_t);
template int tmem_loads<double>(const SolveArgs<double> &, bool);
template int tmem_loads<float>(const SolveArgs<float> &, bool);

}  // namespace penta
