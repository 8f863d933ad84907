// tma_kernels.cu -- the on-chip Thomas kernel for the strided (y, z)
// directions, fed by TMA.
//
// Same algorithm as tiled_kernels.cu with P = 2 (each of S = 16 systems per
// warp split at row m = ceil(n/2), upper half eliminated downwards, lower half
// upwards on the mirrored band, 4x4 interface solve by warp shuffles), with
// three changes that cut the instructions a warp spends per row and the shared
// memory it needs per system:
//
//  * Loads: one lane issues, per ring stage, 12 tensor-tile copies
//    (cp.async.bulk.tensor.3d: 6 arrays x 2 halves, 16 systems x R rows each)
//    that complete on one mbarrier.  The lower half's tiles are taken from the
//    mirrored arrays (dw, du, d, dl, ds, rhs), so every lane runs the same
//    downward recurrence without selects.  Each wait on an mbarrier is bounded;
//    a wait that runs out raises STATUS_TIMEOUT_BIT and the kernel returns.
//  * The forward-substituted right-hand side x2 is written in place into x
//    (the right-hand side of that row has just been consumed) and read back,
//    most recently written first, in the backward sweep through a small
//    cp.async ring.  It makes an L2 round trip instead of occupying shared
//    memory; the final solution overwrites the same lines, so HBM still sees
//    one write per point.  Shared memory per system is 16 B/row (du2, dw2).
//  * Stages of R rows are unrolled, with the first-row couplings zeroed in
//    shared memory once per tile rather than masked per row.
//
// Tensor view: the array as a 3-D tensor {inner, n, outer} (element strides
// 1, inner, inner*n), tile {16, R, 1} at (system offset in the run, first row,
// run).  TMA requires a 16-byte aligned base, inner * sizeof(F) a multiple of
// 16 and a 16-byte aligned innermost coordinate (the system offset is a
// multiple of 16); the host checks all three and otherwise uses the cp.async
// kernel.  Rows outside [0, n) read as zeros (never consumed).
#include <cstdlib>

#include "penta_internal.hpp"
#include "tma_device.cuh"

namespace penta {
namespace {

constexpr int TS = 16;                 // systems per warp


// SCR = false: du2, dw2 in shared memory, x2 written in place into x.
// SCR = true:  du2 in shared memory, (dw2, x2) pairs in the caller's scratch
//              buffer ([tile][row][16 systems][2]), one vector store per row.
template <typename F, int R, int STAGES, int XST, bool SCR>
struct TmaGeom {
  static constexpr int SE = 6 * 2 * R * TS;            // ring stage (elements)
  static constexpr int FW = SCR ? TS : 2 * TS;          // factor row (elements)
  static constexpr int XE = R * 32 * (SCR ? 2 : 1);     // read-back stage
  // Rounded up to 1 KB so that every co-resident CTA's window (and with it
  // each 128-byte aligned TMA destination) starts aligned.
  static size_t smem_bytes(long long n) {
    const size_t b = (size_t)((long long)STAGES * SE + n * FW + (long long)XST * XE) *
                         sizeof(F) +
                     2 * STAGES * sizeof(uint64_t);
    return (b + 1023) & ~size_t(1023);
  }
};


// Warp 0 computes (lanes 0..15: upper halves of 16 systems, 16..31: lower
// halves); lane 0 of warp 1 is the producer.
template <typename F, int R, int STAGES, int XST, bool SCR>
__global__ void __launch_bounds__(64, 1)
tma_strided_kernel(const __grid_constant__ TmaMaps maps, F *__restrict__ x,
                   F *__restrict__ scratch, int n, int inner, int tiles_per_run,
                   int n_tiles, int *__restrict__ status_word) {
  using G = TmaGeom<F, R, STAGES, XST, SCR>;
  using V2 = typename Vec2<F>::T;
  constexpr int SE = G::SE, XE = G::XE, FW = G::FW;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  F *const ring = reinterpret_cast<F *>(smem_raw);
  F *const fac = ring + STAGES * SE;          // [n][FW]
  F *const xr = fac + n * FW;                 // [XST][R][32](x2 or (dw2,x2))
  uint64_t *const full = reinterpret_cast<uint64_t *>(xr + XST * XE);
  uint64_t *const empty = full + STAGES;

  const int warp = threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  // TMA writes shared memory at 128-byte aligned addresses only; refuse to
  // run (and report) rather than issue a misaligned copy.
  if ((smem_u32(smem_raw) & 127u) != 0u) {
    if (threadIdx.x == 0 && blockIdx.x == 0) atomicOr(status_word, STATUS_TIMEOUT_BIT);
    return;
  }
  const int mt = (n + 1) / 2;
  const int mb = n - mt;
  const int n_stages = (mt + R - 1) / R;
  const int my_first = blockIdx.x;
  const int my_tiles =
      (my_first < n_tiles) ? (n_tiles - 1 - my_first) / (int)gridDim.x + 1 : 0;
  const int total = my_tiles * n_stages;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();

  // ------------------------------- producer --------------------------------
  if (warp == 1) {
    if (lane != 0) return;
    constexpr unsigned kStageBytes = 12u * R * TS * sizeof(F);
    // the lower half reads the mirrored band: ds<-dw, dl<-du, d, du<-dl,
    // dw<-ds, rhs
    constexpr int kMirror[6] = {4, 3, 2, 1, 0, 5};
    int slot = 0, use = 0, g = 0, ti = 0;
    int run = my_first / tiles_per_run;
    int j0 = (my_first - run * tiles_per_run) * TS;
    for (int gs = 0; gs < total; ++gs) {
      if (use > 0 && !mbar_wait(&empty[slot], (unsigned)(use - 1) & 1u)) {
        atomicOr(status_word, STATUS_TIMEOUT_BIT);
        return;
      }
      F *dst = ring + slot * SE;
      mbar_expect_tx(&full[slot], kStageBytes);
      const int r_up = g * R;            // upper half: rows r_up ..
      const int r_dn = n - (g + 1) * R;  // lower half: rows r_dn ..
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        tma_load_3d(dst + (q * 2 + 0) * R * TS, &maps.m[q], &full[slot], j0, r_up, run);
        tma_load_3d(dst + (q * 2 + 1) * R * TS, &maps.m[kMirror[q]], &full[slot], j0,
                    r_dn, run);
      }
      if (++slot == STAGES) { slot = 0; ++use; }
      if (++g == n_stages) {
        g = 0;
        if (++ti < my_tiles) {
          const int tile = my_first + ti * (int)gridDim.x;
          run = tile / tiles_per_run;
          j0 = (tile - run * tiles_per_run) * TS;
        }
      }
    }
    return;
  }

  // ------------------------------- consumer --------------------------------
  const int sys = lane % TS;
  const int part = lane / TS;
  const int my_rows = part ? mb : mt;
  const int fstep = part ? -FW : FW;       // factor row step (elements)
  const int sstep = part ? -2 * TS : 2 * TS;  // scratch row step (elements)
  int slot = 0;
  unsigned phase = 0;
  bool bad = false, timed_out = false;
  for (int ti = 0; ti < my_tiles; ++ti) {
    const int tile = my_first + ti * (int)gridDim.x;
    const int run = tile / tiles_per_run;
    const int j0 = (tile - run * tiles_per_run) * TS;
    const bool active = j0 + sys < inner;
    const int xstep = part ? -inner : inner;  // element offset per row
    const int row0 = part ? (n - 1) : 0;       // first row in elimination order
    int xo = run * inner * n + j0 + sys + row0 * inner;
    // (dw2, x2) of this lane's rows: [row][16][2] inside the tile's region
    F *const sg = SCR ? scratch + (long long)tile * n * 2 * TS : nullptr;
    int so = (row0 * TS + sys) * 2;

    Carry<F> c;
    c.zero();
    F *fp = fac + row0 * FW + sys;             // du2 fp[0] (, dw2 fp[TS])
    for (int g = 0; g < n_stages; ++g) {
      if (!mbar_wait(&full[slot], phase)) { timed_out = true; break; }
      F *v = ring + slot * SE + part * R * TS + sys + (part ? (R - 1) * TS : 0);
      const int vs = part ? -TS : TS;
      if (g == 0) {  // couplings that leave the line: ds' rows 0,1, dl' row 0
        v[0] = F(0);
        v[vs] = F(0);
        v[2 * R * TS] = F(0);
        // order these generic writes before the slot's next TMA refill
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      }
      // Whole stage into registers, then hand the slot back to the producer
      // before computing: no load waits behind a store, and the refill starts
      // one stage earlier.
      F a[R][6];
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int q = 0; q < 6; ++q) a[r][q] = v[r * vs + q * 2 * R * TS];
      {
        // The refill is an async-proxy write: order these generic-proxy reads
        // before it, or a refill can land under a load still in flight.
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[slot]);
      }
      if (++slot == STAGES) { slot = 0; phase ^= 1u; }
      if (active) {
        const int rows = min(R, my_rows - g * R);
        const Carry<F> c0 = c;
        F u[R], vv[R], y[R];
#pragma unroll
        for (int r = 0; r < R; ++r)
          fwd_row_lean(a[r][0], a[r][1], a[r][2], a[r][3], a[r][4], a[r][5], c,
                       u[r], vv[r], y[r]);
        auto put = [&](int r) {
          fp[r * fstep] = u[r];
          if constexpr (SCR) {
            V2 pv;
            pv.x = vv[r];
            pv.y = y[r];
            *reinterpret_cast<V2 *>(sg + so + r * sstep) = pv;
          } else {
            fp[r * fstep + TS] = vv[r];
            x[xo + r * xstep] = y[r];
          }
        };
        if (rows == R) {
#pragma unroll
          for (int r = 0; r < R; ++r) put(r);
          fp += R * fstep;
          xo += R * xstep;
          so += R * sstep;
        } else {
          // partial last stage: keep the rows that exist and rebuild the
          // carries from them (rows past the line were computed on filler)
          Carry<F> cr = c0;
#pragma unroll
          for (int r = 0; r < R; ++r) {
            if (r < rows) {
              put(r);
              cr.u2 = cr.u1; cr.u1 = u[r];
              cr.w2 = cr.w1; cr.w1 = vv[r];
              cr.y2 = cr.y1; cr.y1 = y[r];
            }
          }
          c = cr;
          if (rows > 0) {
            fp += rows * fstep;
            xo += rows * xstep;
            so += rows * sstep;
          }
        }
      }
    }
    if (timed_out) break;
    bad |= !(isfinite(c.u1) && isfinite(c.u2) && isfinite(c.w1) &&
             isfinite(c.w2) && isfinite(c.y1) && isfinite(c.y2));

    // ---- interface ---------------------------------------------------------
    const F pu1 = __shfl_xor_sync(0xffffffffu, c.u1, TS);
    const F pu2 = __shfl_xor_sync(0xffffffffu, c.u2, TS);
    const F pw1 = __shfl_xor_sync(0xffffffffu, c.w1, TS);
    const F pw2 = __shfl_xor_sync(0xffffffffu, c.w2, TS);
    const F py1 = __shfl_xor_sync(0xffffffffu, c.y1, TS);
    const F py2 = __shfl_xor_sync(0xffffffffu, c.y2, TS);
    F u0, u1, u2, u3;
    if (part == 0)
      solve_interface(c.u2, c.w2, c.y2, c.u1, c.w1, c.y1, pu1, pw1, py1, pu2,
                      pw2, py2, u0, u1, u2, u3);
    else
      solve_interface(pu2, pw2, py2, pu1, pw1, py1, c.u1, c.w1, c.y1, c.u2,
                      c.w2, c.y2, u0, u1, u2, u3);
    // The solution just beyond this half's last row: x(K+1), x(K+2).
    F xa = part ? u1 : u2;
    F xb = part ? u0 : u3;

    // ---- backward over all rows k = K .. 0 ---------------------------------
    // x2 (and dw2 when SCR) of row k come back through a cp.async ring; each
    // lane reads only what it wrote.
    __threadfence_block();
    const int xo_end = xo;                     // one row past row K
    const int so_end = so;
    const F *fb = fp - fstep;                  // factors of row K
    auto xissue = [&](int s) {
      if (s < n_stages && active) {
        F *dst = xr + (s % XST) * XE + lane * (SCR ? 2 : 1);
        if constexpr (SCR) {
          int o = so_end - (1 + s * R) * sstep;
#pragma unroll
          for (int r = 0; r < R; ++r) {
            if (s * R + r < my_rows) {
              if constexpr (sizeof(F) == 8) {
                cp_async_ca<16>(dst + r * 64, sg + o);
              } else {
                cp_async_ca<2 * sizeof(F)>(dst + r * 64, sg + o);
              }
            }
            o -= sstep;
          }
        } else {
          int o = xo_end - (1 + s * R) * xstep;
#pragma unroll
          for (int r = 0; r < R; ++r) {
            if (s * R + r < my_rows) cp_async_ca<sizeof(F)>(dst + r * 32, x + o);
            o -= xstep;
          }
        }
      }
      cp_async_commit();
    };
    for (int s = 0; s < XST - 1; ++s) xissue(s);
    int xw = xo_end - xstep;                   // output offset of row K
    for (int s = 0; s < n_stages; ++s) {
      cp_async_wait<XST - 2>();                // stage s has landed
      F xs[R], du[R], dw[R];
      if constexpr (SCR) {
        const V2 *src = reinterpret_cast<const V2 *>(xr + (s % XST) * XE) + lane;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const V2 pv = src[r * 32];
          dw[r] = pv.x;
          xs[r] = pv.y;
          du[r] = fb[-r * fstep];
        }
      } else {
        const F *src = xr + (s % XST) * XE + lane;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          xs[r] = src[r * 32];
          du[r] = fb[-r * fstep];
          dw[r] = fb[-r * fstep + TS];
        }
      }
      xissue(s + XST - 1);                     // refills the slot of stage s-1
      if constexpr (SCR) {
        // The (dw2, x2) lines of stage s are dead once they sit in shared
        // memory: drop them from L2 so they are never written back to HBM.
        // Each lane of a half drops one of the half's 2 x R lines; a line
        // holds 8 lanes' values, so every lane's copy must have landed first.
        __syncwarp();
        if (active) {
          // a scratch row (16 pairs) is LPR 128-byte lines; lane sys drops
          // line h of the stage's r-th row
          constexpr int LPR = sizeof(F) / 4;
          const int r = sys / LPR, h = sys % LPR;
          const int k = s * R + r;             // k-th row back from row K
          if (r < R && k < my_rows) {
            const int row = part ? (mt + k) : (mt - 1 - k);
            const F *line = sg + row * TS * 2 + h * (128 / (int)sizeof(F));
            asm volatile("discard.global.L2 [%0], 128;\n" ::"l"(line) : "memory");
          }
        }
      }
      if (active) {
        const int rows = min(R, my_rows - s * R);
        F xk[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          xk[r] = xs[r] - du[r] * xa - dw[r] * xb;
          xb = xa;
          xa = xk[r];
        }
        if (rows == R) {
#pragma unroll
          for (int r = 0; r < R; ++r) x[xw - r * xstep] = xk[r];
          xw -= R * xstep;
          fb -= R * fstep;
        } else {
#pragma unroll
          for (int r = 0; r < R; ++r)
            if (r < rows) x[xw - r * xstep] = xk[r];
        }
      }
    }
    cp_async_wait<0>();
    __syncwarp();
  }

  if (timed_out) {
    // give copies that may still be in flight a bounded chance to land
    for (int s = 0; s < STAGES; ++s) {
      mbar_wait(&full[slot], phase);
      if (++slot == STAGES) { slot = 0; phase ^= 1u; }
    }
    if (lane == 0) atomicOr(status_word, STATUS_TIMEOUT_BIT);
    return;
  }
  if (__any_sync(0xffffffffu, bad) && lane == 0)
    atomicOr(status_word, STATUS_ZERO_PIVOT_BIT);
}

// ---------------------------------------------------------------------------
// The contiguous (x) direction.  A tile is 16 consecutive lines, i.e. one
// contiguous block of 16 x n elements.  Tensor view {n, n_sys}; each stage
// loads tiles of {R rows, 16 systems} with the 64-byte swizzle (R * sizeof(F)
// = 64): system s's row r lands at byte s*64 + ((r / EPC) ^ ((s >> 1) & 3))*16
// + (r % EPC)*sizeof(F), EPC = 16 / sizeof(F), which spreads one row of 16
// systems over the banks (two-way at most).  du2 stays in shared memory in a
// system-major layout with an odd pitch (n + 1) -- conflict-free for one row
// of 16 systems and for one system's consecutive rows -- and after the
// backward sweep holds the solution, which leaves through a coalesced
// copy-out.  (dw2, x2) go through the caller's buffer as in the strided
// scratch variant.  Requires n * sizeof(F) to be a multiple of 16.
// ---------------------------------------------------------------------------
template <typename F, int STAGES, int XST>
struct TmaContigGeom {
  static constexpr int R = 64 / sizeof(F);       // rows per box (64 bytes)
  static constexpr int EPC = 16 / sizeof(F);     // elements per 16-byte chunk
  static constexpr int BOX = R * TS;             // elements per box
  static constexpr int SE = 12 * BOX;            // ring stage
  static constexpr int XE = R * 32 * 2;          // read-back stage
  static size_t smem_bytes(long long n) {
    const size_t b = (size_t)((long long)STAGES * SE + TS * (n + 1) + (long long)XST * XE) *
                         sizeof(F) +
                     2 * STAGES * sizeof(uint64_t);
    return ((b + 1023) & ~size_t(1023)) + 1024;  // + slack for 1 KB alignment
  }
};


template <typename F, int STAGES, int XST>
__global__ void __launch_bounds__(64, 1)
tma_contig_kernel(const __grid_constant__ TmaMaps maps, F *__restrict__ x,
                  F *__restrict__ scratch, int n, int n_sys, int n_tiles,
                  int *__restrict__ status_word) {
  using G = TmaContigGeom<F, STAGES, XST>;
  using V2 = typename Vec2<F>::T;
  constexpr int R = G::R, EPC = G::EPC, BOX = G::BOX, SE = G::SE, XE = G::XE;
  constexpr int ROWE = 64 / sizeof(F);            // elements per 64-byte box row
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // swizzled boxes need a 1 KB aligned destination; the launch requests 1 KB
  // of slack for this
  unsigned char *const base = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  F *const ring = reinterpret_cast<F *>(base);
  F *const fac = ring + STAGES * SE;              // [16][n + 1]: du2, then x
  F *const xr = fac + TS * (n + 1);               // [XST][R][32](dw2, x2)
  uint64_t *const full = reinterpret_cast<uint64_t *>(xr + XST * XE);
  uint64_t *const empty = full + STAGES;

  const int warp = threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  const int mt = (n + 1) / 2;
  const int mb = n - mt;
  const int n_stages = (mt + R - 1) / R;
  const int my_first = blockIdx.x;
  const int my_tiles =
      (my_first < n_tiles) ? (n_tiles - 1 - my_first) / (int)gridDim.x + 1 : 0;
  const int total = my_tiles * n_stages;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();

  if (warp == 1) {  // ------------------------------ producer ----------------
    if (lane != 0) return;
    constexpr unsigned kStageBytes = 12u * BOX * sizeof(F);
    constexpr int kMirror[6] = {4, 3, 2, 1, 0, 5};
    int slot = 0, use = 0, g = 0, ti = 0;
    int s0 = my_first * TS;
    for (int gs = 0; gs < total; ++gs) {
      if (use > 0 && !mbar_wait(&empty[slot], (unsigned)(use - 1) & 1u)) {
        atomicOr(status_word, STATUS_TIMEOUT_BIT);
        return;
      }
      F *dst = ring + slot * SE;
      mbar_expect_tx(&full[slot], kStageBytes);
      const int r_up = g * R, r_dn = n - (g + 1) * R;
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        tma_load_2d(dst + (q * 2 + 0) * BOX, &maps.m[q], &full[slot], r_up, s0);
        tma_load_2d(dst + (q * 2 + 1) * BOX, &maps.m[kMirror[q]], &full[slot], r_dn, s0);
      }
      if (++slot == STAGES) { slot = 0; ++use; }
      if (++g == n_stages) {
        g = 0;
        if (++ti < my_tiles) s0 = (my_first + ti * (int)gridDim.x) * TS;
      }
    }
    return;
  }

  // -------------------------------- consumer --------------------------------
  const int sys = lane % TS;
  const int part = lane / TS;
  const int my_rows = part ? mb : mt;
  // element offset, inside a box, of this lane's r-th row in elimination order
  int off[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int rb = part ? (R - 1 - r) : r;
    off[r] = sys * ROWE + (((rb / EPC) ^ ((sys >> 1) & 3)) * EPC) + (rb % EPC);
  }
  const int fpitch = n + 1;
  const int fstep = part ? -1 : 1;
  const int sstep = part ? -2 * TS : 2 * TS;
  int slot = 0;
  unsigned phase = 0;
  bool bad = false, timed_out = false;
  for (int ti = 0; ti < my_tiles; ++ti) {
    const int tile = my_first + ti * (int)gridDim.x;
    const int s0 = tile * TS;
    const int count = min(TS, n_sys - s0);
    const bool active = sys < count;
    const int row0 = part ? (n - 1) : 0;
    F *const sg = scratch + (long long)tile * n * 2 * TS;
    int so = (row0 * TS + sys) * 2;
    F *fp = fac + sys * fpitch + row0;

    Carry<F> c;
    c.zero();
    for (int g = 0; g < n_stages; ++g) {
      if (!mbar_wait(&full[slot], phase)) { timed_out = true; break; }
      const F *v = ring + slot * SE + part * BOX;
      F a[R][6];
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int q = 0; q < 6; ++q) a[r][q] = v[q * 2 * BOX + off[r]];
      if (g == 0) {  // couplings that leave the line: ds' rows 0,1, dl' row 0
        a[0][0] = F(0);
        a[1][0] = F(0);
        a[0][1] = F(0);
      }
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[slot]);
      if (++slot == STAGES) { slot = 0; phase ^= 1u; }
      if (active) {
        const int rows = min(R, my_rows - g * R);
        const Carry<F> c0 = c;
        F u[R], vv[R], y[R];
#pragma unroll
        for (int r = 0; r < R; ++r)
          fwd_row_lean(a[r][0], a[r][1], a[r][2], a[r][3], a[r][4], a[r][5], c,
                       u[r], vv[r], y[r]);
        auto put = [&](int r) {
          fp[r * fstep] = u[r];
          V2 pv;
          pv.x = vv[r];
          pv.y = y[r];
          *reinterpret_cast<V2 *>(sg + so + r * sstep) = pv;
        };
        if (rows == R) {
#pragma unroll
          for (int r = 0; r < R; ++r) put(r);
          fp += R * fstep;
          so += R * sstep;
        } else {
          Carry<F> cr = c0;
#pragma unroll
          for (int r = 0; r < R; ++r) {
            if (r < rows) {
              put(r);
              cr.u2 = cr.u1; cr.u1 = u[r];
              cr.w2 = cr.w1; cr.w1 = vv[r];
              cr.y2 = cr.y1; cr.y1 = y[r];
            }
          }
          c = cr;
          if (rows > 0) {
            fp += rows * fstep;
            so += rows * sstep;
          }
        }
      }
    }
    if (timed_out) break;
    bad |= !(isfinite(c.u1) && isfinite(c.u2) && isfinite(c.w1) &&
             isfinite(c.w2) && isfinite(c.y1) && isfinite(c.y2));

    const F pu1 = __shfl_xor_sync(0xffffffffu, c.u1, TS);
    const F pu2 = __shfl_xor_sync(0xffffffffu, c.u2, TS);
    const F pw1 = __shfl_xor_sync(0xffffffffu, c.w1, TS);
    const F pw2 = __shfl_xor_sync(0xffffffffu, c.w2, TS);
    const F py1 = __shfl_xor_sync(0xffffffffu, c.y1, TS);
    const F py2 = __shfl_xor_sync(0xffffffffu, c.y2, TS);
    F u0, u1, u2, u3;
    if (part == 0)
      solve_interface(c.u2, c.w2, c.y2, c.u1, c.w1, c.y1, pu1, pw1, py1, pu2,
                      pw2, py2, u0, u1, u2, u3);
    else
      solve_interface(pu2, pw2, py2, pu1, pw1, py1, c.u1, c.w1, c.y1, c.u2,
                      c.w2, c.y2, u0, u1, u2, u3);
    F xa = part ? u1 : u2;  // x(K+1)
    F xb = part ? u0 : u3;  // x(K+2)

    // ---- backward over k = K .. 0; x(k) replaces du2(k) in shared memory ---
    __threadfence_block();
    const int so_end = so;
    F *fb = fp - fstep;                        // row K
    auto xissue = [&](int s) {
      if (s < n_stages && active) {
        F *dst = xr + (s % XST) * XE + lane * 2;
        int o = so_end - (1 + s * R) * sstep;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          if (s * R + r < my_rows) cp_async_ca<2 * sizeof(F)>(dst + r * 64, sg + o);
          o -= sstep;
        }
      }
      cp_async_commit();
    };
    for (int s = 0; s < XST - 1; ++s) xissue(s);
    for (int s = 0; s < n_stages; ++s) {
      cp_async_wait<XST - 2>();
      const V2 *src = reinterpret_cast<const V2 *>(xr + (s % XST) * XE) + lane;
      F xs[R], du[R], dw[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const V2 pv = src[r * 32];
        dw[r] = pv.x;
        xs[r] = pv.y;
        du[r] = fb[-r * fstep];
      }
      xissue(s + XST - 1);
      __syncwarp();  // every lane's copies of stage s have landed
      if (active) {  // drop the dead (dw2, x2) lines from L2
        constexpr int LPR = sizeof(F) / 4;  // 128-byte lines per scratch row
        const int r = sys / LPR, h = sys % LPR;
        const int k = s * R + r;
        if (r < R && k < my_rows) {
          const int row = part ? (mt + k) : (mt - 1 - k);
          const F *line = sg + row * TS * 2 + h * (128 / (int)sizeof(F));
          asm volatile("discard.global.L2 [%0], 128;\n" ::"l"(line) : "memory");
        }
      }
      if (active) {
        const int rows = min(R, my_rows - s * R);
        F xk[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          xk[r] = xs[r] - du[r] * xa - dw[r] * xb;
          xb = xa;
          xa = xk[r];
        }
#pragma unroll
        for (int r = 0; r < R; ++r)
          if (r < rows) fb[-r * fstep] = xk[r];
        if (rows == R) fb -= R * fstep;
      }
    }
    cp_async_wait<0>();
    __syncwarp();
    // coalesced copy-out of the tile's solution
    for (int sy = 0; sy < count; ++sy) {
      F *dst = x + (long long)(s0 + sy) * n;
      const F *src = fac + sy * fpitch;
      for (int row = lane; row < n; row += 32) dst[row] = src[row];
    }
    __syncwarp();
  }

  if (timed_out) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_wait(&full[slot], phase);
      if (++slot == STAGES) { slot = 0; phase ^= 1u; }
    }
    if (lane == 0) atomicOr(status_word, STATUS_TIMEOUT_BIT);
    return;
  }
  if (__any_sync(0xffffffffu, bad) && lane == 0)
    atomicOr(status_word, STATUS_ZERO_PIVOT_BIT);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() { return tensor_map_encoder(); }

template <typename F>
bool encode_map(CUtensorMap *m, const F *ptr, const Lines &L, int R) {
  auto fn = encode_fn();
  if (fn == nullptr) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)L.inner, (cuuint64_t)L.n,
                              (cuuint64_t)(L.n_sys / L.inner)};
  const cuuint64_t strides[2] = {(cuuint64_t)L.inner * sizeof(F),
                                 (cuuint64_t)L.inner * L.n * sizeof(F)};
  const cuuint32_t box[3] = {(cuuint32_t)TS, (cuuint32_t)R, 1};
  const cuuint32_t es[3] = {1, 1, 1};
  CUresult r = fn(m,
                  sizeof(F) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                  3, const_cast<F *>(ptr), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <typename F, int R, int ST, int XST, bool SCR>
cudaError_t tma_launch(const SolveArgs<F> &a, int grid, cudaStream_t stream) {
  using G = TmaGeom<F, R, ST, XST, SCR>;
  TmaMaps maps;
  const F *ptrs[6] = {a.ds, a.dl, a.d, a.du, a.dw, a.x};
  for (int q = 0; q < 6; ++q)
    if (!encode_map<F>(&maps.m[q], ptrs[q], a.L, R)) return cudaErrorInvalidValue;
  auto kern = tma_strided_kernel<F, R, ST, XST, SCR>;
  const size_t smem = G::smem_bytes(a.L.n);
  cudaError_t err = cudaFuncSetAttribute(
      kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  const int inner = (int)a.L.inner, n = (int)a.L.n;
  const int tiles_per_run = (inner + TS - 1) / TS;
  const int n_tiles = (int)(a.L.n_sys / a.L.inner) * tiles_per_run;
  if (grid <= 0 || grid > n_tiles) grid = n_tiles;
  kern<<<grid, 64, smem, stream>>>(maps, a.x, static_cast<F *>(a.scratch), n,
                                   inner, tiles_per_run, n_tiles, a.status);
  return cudaGetLastError();
}


template <typename F>
bool encode_map_contig(CUtensorMap *m, const F *ptr, const Lines &L) {
  auto fn = encode_fn();
  if (fn == nullptr) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)L.n, (cuuint64_t)L.n_sys};
  const cuuint64_t strides[1] = {(cuuint64_t)L.n * sizeof(F)};
  const cuuint32_t box[2] = {(cuuint32_t)(64 / sizeof(F)), (cuuint32_t)TS};
  const cuuint32_t es[2] = {1, 1};
  CUresult r = fn(m,
                  sizeof(F) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                  2, const_cast<F *>(ptr), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <typename F, int ST, int XST>
cudaError_t tma_contig_launch(const SolveArgs<F> &a, int grid, cudaStream_t stream) {
  using G = TmaContigGeom<F, ST, XST>;
  TmaMaps maps;
  const F *ptrs[6] = {a.ds, a.dl, a.d, a.du, a.dw, a.x};
  for (int q = 0; q < 6; ++q)
    if (!encode_map_contig<F>(&maps.m[q], ptrs[q], a.L)) return cudaErrorInvalidValue;
  auto kern = tma_contig_kernel<F, ST, XST>;
  const size_t smem = G::smem_bytes(a.L.n);
  cudaError_t err = cudaFuncSetAttribute(
      kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  const int n = (int)a.L.n, n_sys = (int)a.L.n_sys;
  const int n_tiles = (n_sys + TS - 1) / TS;
  if (grid <= 0 || grid > n_tiles) grid = n_tiles;
  kern<<<grid, 64, smem, stream>>>(maps, a.x, static_cast<F *>(a.scratch), n,
                                   n_sys, n_tiles, a.status);
  return cudaGetLastError();
}

template <typename F, int ST, int XST> int tma_contig_occ(long long n) {
  using G = TmaContigGeom<F, ST, XST>;
  auto kern = tma_contig_kernel<F, ST, XST>;
  const size_t smem = G::smem_bytes(n);
  int blocks = 0;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, 64, smem) !=
          cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return blocks;
}

template <typename F, int R, int ST, int XST, bool SCR> int tma_occ(long long n) {
  using G = TmaGeom<F, R, ST, XST, SCR>;
  auto kern = tma_strided_kernel<F, R, ST, XST, SCR>;
  const size_t smem = G::smem_bytes(n);
  int blocks = 0;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, 64, smem) !=
          cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return blocks;
}

}  // namespace

#define PENTA_TMA_CONFIGS(X) \
  X(double, 8, 3, 6, false)  \
  X(double, 8, 2, 4, true)   \
  X(double, 8, 3, 4, true)   \
  X(double, 4, 4, 6, true)   \
  X(float, 8, 3, 4, false)   \
  X(float, 8, 3, 4, true)    \
  X(float, 8, 4, 6, true)

template <typename F> const std::vector<TmaConfig> &tma_configs() {
  static const std::vector<TmaConfig> v = [] {
    std::vector<TmaConfig> out;
#define PENTA_X(FT_, R_, ST_, XST_, SCR_) \
  if (std::is_same<F, FT_>::value) out.push_back(TmaConfig{R_, ST_, XST_, SCR_});
    PENTA_TMA_CONFIGS(PENTA_X)
#undef PENTA_X
    return out;
  }();
  return v;
}

template <typename F> size_t tma_smem_bytes(const TmaConfig &c, long long n) {
  const long long fw = c.scratch ? TS : 2 * TS;
  const long long xe = (long long)c.R * 32 * (c.scratch ? 2 : 1);
  const size_t b = (size_t)((long long)c.stages * 6 * 2 * c.R * TS + n * fw +
                            (long long)c.xstages * xe) *
                       sizeof(F) +
                   2 * c.stages * sizeof(uint64_t);
  return (b + 1023) & ~size_t(1023);
}

template <typename F> int tma_occupancy(const TmaConfig &c, long long n) {
#define PENTA_X(FT_, R_, ST_, XST_, SCR_)                                 \
  if (std::is_same<F, FT_>::value && c.R == R_ && c.stages == ST_ &&      \
      c.xstages == XST_ && c.scratch == SCR_)                             \
    return tma_occ<FT_, R_, ST_, XST_, SCR_>(n);
  PENTA_TMA_CONFIGS(PENTA_X)
#undef PENTA_X
  return 0;
}

template <typename F>
bool tma_supported(const SolveArgs<F> &a) {
  if (encode_fn() == nullptr) return false;
  if (a.L.inner == 1) return false;                        // strided only
  if ((a.L.inner * sizeof(F)) % 16 != 0) return false;     // row stride
  if (a.L.n * a.L.n_sys >= (1LL << 31)) return false;
  if (a.L.inner > 0xffffffffLL || a.L.n_sys / a.L.inner > 0xffffffffLL) return false;
  const void *ptrs[6] = {a.ds, a.dl, a.d, a.du, a.dw, a.x};
  for (const void *p : ptrs)
    if (reinterpret_cast<uintptr_t>(p) % 16 != 0) return false;
  return true;
}

template <typename F>
cudaError_t launch_tma(const SolveArgs<F> &a, const TmaConfig &c, int grid,
                       cudaStream_t stream) {
#define PENTA_X(FT_, R_, ST_, XST_, SCR_)                                 \
  if (std::is_same<F, FT_>::value && c.R == R_ && c.stages == ST_ &&      \
      c.xstages == XST_ && c.scratch == SCR_)                             \
    return tma_launch<FT_, R_, ST_, XST_, SCR_>(                          \
        reinterpret_cast<const SolveArgs<FT_> &>(a), grid, stream);
  PENTA_TMA_CONFIGS(PENTA_X)
#undef PENTA_X
  return cudaErrorInvalidConfiguration;
}

template const std::vector<TmaConfig> &tma_configs<double>();
template const std::vector<TmaConfig> &tma_configs<float>();
template size_t tma_smem_bytes<double>(const TmaConfig &, long long);
template size_t tma_smem_bytes<float>(const TmaConfig &, long long);
template int tma_occupancy<double>(const TmaConfig &, long long);
template int tma_occupancy<float>(const TmaConfig &, long long);
template bool tma_supported<double>(const SolveArgs<double> &);
template bool tma_supported<float>(const SolveArgs<float> &);
template cudaError_t launch_tma<double>(const SolveArgs<double> &,
                                        const TmaConfig &, int, cudaStream_t);
template cudaError_t launch_tma<float>(const SolveArgs<float> &,
                                       const TmaConfig &, int, cudaStream_t);

#define PENTA_TMA_CONTIG_CONFIGS(X) \
  X(double, 3, 4)                   \
  X(double, 2, 4)                   \
  X(double, 4, 4)                   \
  X(float, 3, 4)                    \
  X(float, 2, 4)

template <typename F> const std::vector<TmaConfig> &tma_contig_configs() {
  static const std::vector<TmaConfig> v = [] {
    std::vector<TmaConfig> out;
#define PENTA_X(FT_, ST_, XST_) \
  if (std::is_same<F, FT_>::value) out.push_back(TmaConfig{64 / (int)sizeof(FT_), ST_, XST_, true});
    PENTA_TMA_CONTIG_CONFIGS(PENTA_X)
#undef PENTA_X
    return out;
  }();
  return v;
}

template <typename F> size_t tma_contig_smem_bytes(const TmaConfig &c, long long n) {
  const long long R = 64 / sizeof(F);
  const size_t b = (size_t)((long long)c.stages * 12 * R * TS + TS * (n + 1) +
                            (long long)c.xstages * R * 64) *
                       sizeof(F) +
                   2 * c.stages * sizeof(uint64_t);
  return ((b + 1023) & ~size_t(1023)) + 1024;
}

template <typename F> int tma_contig_occupancy(const TmaConfig &c, long long n) {
#define PENTA_X(FT_, ST_, XST_)                                                  \
  if (std::is_same<F, FT_>::value && c.stages == ST_ && c.xstages == XST_)       \
    return tma_contig_occ<FT_, ST_, XST_>(n);
  PENTA_TMA_CONTIG_CONFIGS(PENTA_X)
#undef PENTA_X
  return 0;
}

template <typename F> bool tma_contig_supported(const SolveArgs<F> &a) {
  if (encode_fn() == nullptr) return false;
  if (a.L.inner != 1) return false;
  if ((a.L.n * sizeof(F)) % 16 != 0) return false;
  if (a.L.n * a.L.n_sys >= (1LL << 31)) return false;
  // 128-byte aligned: the kernel drops whole 128-byte lines of it from L2
  if (a.scratch == nullptr || reinterpret_cast<uintptr_t>(a.scratch) % 128 != 0)
    return false;
  const void *ptrs[6] = {a.ds, a.dl, a.d, a.du, a.dw, a.x};
  for (const void *p : ptrs)
    if (reinterpret_cast<uintptr_t>(p) % 16 != 0) return false;
  return true;
}

template <typename F>
cudaError_t launch_tma_contig(const SolveArgs<F> &a, const TmaConfig &c, int grid,
                              cudaStream_t stream) {
#define PENTA_X(FT_, ST_, XST_)                                                  \
  if (std::is_same<F, FT_>::value && c.stages == ST_ && c.xstages == XST_)       \
    return tma_contig_launch<FT_, ST_, XST_>(                                    \
        reinterpret_cast<const SolveArgs<FT_> &>(a), grid, stream);
  PENTA_TMA_CONTIG_CONFIGS(PENTA_X)
#undef PENTA_X
  return cudaErrorInvalidConfiguration;
}

template const std::vector<TmaConfig> &tma_contig_configs<double>();
template const std::vector<TmaConfig> &tma_contig_configs<float>();
template size_t tma_contig_smem_bytes<double>(const TmaConfig &, long long);
template size_t tma_contig_smem_bytes<float>(const TmaConfig &, long long);
template int tma_contig_occupancy<double>(const TmaConfig &, long long);
template int tma_contig_occupancy<float>(const TmaConfig &, long long);
template bool tma_contig_supported<double>(const SolveArgs<double> &);
template bool tma_contig_supported<float>(const SolveArgs<float> &);
template cudaError_t launch_tma_contig<double>(const SolveArgs<double> &,
                                               const TmaConfig &, int, cudaStream_t);
template cudaError_t launch_tma_contig<float>(const SolveArgs<float> &,
                                              const TmaConfig &, int, cudaStream_t);

}  // namespace penta
