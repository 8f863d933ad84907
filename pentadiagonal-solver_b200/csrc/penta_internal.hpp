// penta_internal.hpp -- interfaces between the host dispatcher (C++) and the
// kernel launchers (CUDA).  Nothing here crosses the library boundary.
#pragma once
#include <cuda_runtime_api.h>
#include <cstddef>
#include <string>
#include <type_traits>
#include <vector>

#include "pentad_common.hpp"
#include "pentadsolver_handle.hpp"
#include "penta_lines.h"

namespace penta {

// penta_api.cpp: the rules every entry point applies, for entry points
// defined elsewhere.  check_shape: the shape checks (pure host code; the
// reference's limits, overflow-safe).  bind_handle: resolve a handle (NULL:
// the current device's default context), bind it to the current device on
// first use, refuse a handle bound to another device, and give the address of
// its status word.
pentadStatus_t check_shape(const int *dims, int ndim, int solvedim, Lines &L, const char **why);
pentadStatus_t bind_handle(pentadsolver_handle_t h, int **status, const char **why);

template <typename F> struct SolveArgs {
  const F *ds, *dl, *d, *du, *dw;
  F *x;
  Lines L;
  void *scratch;         // caller's buffer (may be null when unused)
  size_t scratch_bytes;  // its size
  int *status;           // device word that kernels OR status bits into
};

// A compiled variant of the tiled Thomas kernel.
struct TiledConfig {
  int S;       // systems per CTA
  int P;       // partitions (threads) per system: 1 or 2
  bool contig; // contiguous (x) layout
  int R;       // rows per ring slot
  int stages;  // ring slots
};

// thomas_kernels.cu
template <typename F>
cudaError_t launch_thomas_global(const SolveArgs<F> &a, cudaStream_t stream);

// tiled_kernels.cu (on-chip Thomas, one warp per CTA; S = 32 / P)
template <typename F> const std::vector<TiledConfig> &tiled2_configs();
template <typename F> size_t tiled2_smem_bytes(const TiledConfig &cfg, long long n);
template <typename F> int tiled2_occupancy(const TiledConfig &cfg, long long n);
template <typename F>
cudaError_t launch_tiled2(const SolveArgs<F> &a, const TiledConfig &cfg,
                          int grid, cudaStream_t stream);

// A compiled variant of the TMA-fed strided kernel (tma_kernels.cu).
struct TmaConfig {
  int R;         // rows per ring stage
  int stages;    // ring stages
  int xstages;   // stages of the read-back ring
  bool scratch;  // (dw2, x2) in the caller's buffer instead of smem / x
};

// Bytes of caller buffer the scratch variant of the TMA kernel uses.
template <typename F> inline size_t tma_scratch_bytes(const Lines &L) {
  const long long tiles = (L.n_sys / L.inner) * ((L.inner + 15) / 16);
  return (size_t)tiles * (size_t)L.n * 32 * sizeof(F);
}
template <typename F> const std::vector<TmaConfig> &tma_configs();
template <typename F> size_t tma_smem_bytes(const TmaConfig &c, long long n);
template <typename F> int tma_occupancy(const TmaConfig &c, long long n);
template <typename F> bool tma_supported(const SolveArgs<F> &a);
template <typename F>
cudaError_t launch_tma(const SolveArgs<F> &a, const TmaConfig &c, int grid,
                       cudaStream_t stream);

// The TMA-fed contiguous (x) kernel (always keeps (dw2, x2) in the buffer).
template <typename F> const std::vector<TmaConfig> &tma_contig_configs();
template <typename F> size_t tma_contig_smem_bytes(const TmaConfig &c, long long n);
template <typename F> int tma_contig_occupancy(const TmaConfig &c, long long n);
template <typename F> bool tma_contig_supported(const SolveArgs<F> &a);
template <typename F>
cudaError_t launch_tma_contig(const SolveArgs<F> &a, const TmaConfig &c, int grid,
                              cudaStream_t stream);
// Bytes of caller buffer the contiguous TMA kernel uses.
template <typename F> inline size_t tma_contig_scratch_bytes(const Lines &L) {
  return (size_t)((L.n_sys + 15) / 16) * (size_t)L.n * 32 * sizeof(F);
}

// tmem_kernels.cu: the Thomas kernel with its factors in Tensor Memory (all
// directions; n <= 512 in FP64, n <= 1024 in FP32; x2 -- and dw2 for the
// longer lines -- go through the caller's buffer).  One grid per launch, or
// many grids of one direction and precision in one batched launch.
struct TmemConfig {
  bool contig;   // along x (rows contiguous) or strided
  int fmode;     // factors in TMEM: 0 du2 and dw2, 1 du2 (dw2 in the buffer), 2 none
  int stages;    // forward ring stages per consumer warp
  int xstages;   // read-back stages per consumer warp
  int R;         // rows per stage
  size_t smem;   // dynamic shared memory per CTA
  int loads;     // 0: TMA tiles / element copies; 1: pitched (group-view TMA, bulk copies)
};
template <typename F> const std::vector<TmemConfig> &tmem_configs();
template <typename F> int tmem_occupancy(const TmemConfig &c);
// A line set the kernel takes; `fmode` tells which factor mode it needs.
template <typename F> bool tmem_shape(const Lines &L, bool contig, int &fmode);
template <typename F> size_t tmem_scratch_bytes(const Lines &L, bool contig, int fmode);
template <typename F>
bool tmem_supported(const SolveArgs<F> &a, bool contig, size_t usable_buf, int &fmode);
// The stage layout (TmemConfig::loads) a grid's loads take.
template <typename F> int tmem_loads(const SolveArgs<F> &a, bool contig);
// " grp", " bulk", " chunk" or "" -- which loader fills the stages (variant names)
template <typename F> const char *tmem_loader(const SolveArgs<F> &a, bool contig);
template <typename F>
cudaError_t launch_tmem(const SolveArgs<F> &a, const TmemConfig &c, int sm_count,
                        cudaStream_t stream);
// Batched: the job table (tmem_job_bytes() per grid) is filled on the host
// and copied to device memory by the caller; grid i's scratch starts at
// device_base + scratch_offsets[i] (128-byte aligned for L2 discards).
template <typename F> size_t tmem_job_bytes();
template <typename F>
bool tmem_fill_jobs(const SolveArgs<F> *grids, int count, bool contig, int fmode, int loads,
                    unsigned char *device_base, void *host_jobs, size_t *scratch_offsets,
                    int *total_tiles);
template <typename F>
cudaError_t launch_tmem_batch(const void *device_jobs, int n_jobs, int total_tiles, bool contig,
                              int fmode, int loads, bool discard, int sm_count, int *status,
                              cudaStream_t stream);

// shared_fact_kernels.cu: shared factorisation (line 0's coefficients for
// every line).  The Tensor-Memory kernel needs no buffer (it caches its table
// at the end of the buffer when there is one); the per-line fallback needs
// sf_lines_scratch_bytes.
template <typename F>
bool sf_tmem_supported(const SolveArgs<F> &a, bool contig, int smem_optin);
template <typename F> int sf_tmem_occupancy(bool contig);
template <typename F>
cudaError_t launch_sf_tmem(const SolveArgs<F> &a, bool contig, int sm_count,
                           size_t usable_buf, cudaStream_t stream);
template <typename F> size_t sf_lines_scratch_bytes(const Lines &L);
template <typename F> cudaError_t launch_sf_lines(const SolveArgs<F> &a, cudaStream_t stream);

// refine_kernels.cu: FP64 residual and correction steps of mixed-precision
// refinement over one grid (passed by value) or a device table of grids.
struct RefineGrid {
  const double *ds, *dl, *d, *du, *dw;  // the FP64 problem
  double *x;                            // the iterate (the caller's x)
  double *b;                            // the saved right-hand side
  float *s_ds, *s_dl, *s_d, *s_du, *s_dw;  // FP32 coefficient copies
  float *r;                             // FP32 right-hand side / correction
  float *q;                             // FP32 residual / correction of a one-step solve
  double *est;                          // [max|last correction|, max|x|]
  long long n_points;
  int n, inner;                         // line length, row stride
  int chunk_base;                       // first CTA of this grid in a table launch
  int pad_;
};
enum class RefineStep {
  PrepareCast, Prepare, Lift, Residual, Correct,
  // one refinement step without an FP64 copy of the first iterate or of b:
  // r = fl32(x) (b stays in x), the sweep leaves x0 in r, q = fl32(x - A x0),
  // the sweep leaves d in q, x = x0 + d
  FirstCast, First, Residual1, Correct1
};
int refine_chunks(long long n_points);
cudaError_t launch_refine_step(RefineStep step, const RefineGrid &one, const RefineGrid *table,
                               int count, int total_chunks, cudaStream_t stream);

// slab_kernels.cu: the segment copies of the slab-decomposed ADI (pack: the
// z-slab's blocks for every destination rank into one buffer; unpack: back).
cudaError_t launch_slab_copy(int elem_bytes, const void *src, void *dst, int nx, int ny,
                             int nz_local, int parts, bool to_packed, int sm_count,
                             cudaStream_t stream);

// penta_tune.cpp: the process-wide tuning table (an autotuner's measured
// choices per shape class; read from PENTA_TUNING_CACHE on first use).
struct TuneChoice {
  std::string spec;  // pentadsolver_set_tuning string ("" = automatic)
  std::string algo;  // kernel family ("thomas-pcr", ...; "" = automatic)
  int lanes = 0;     // PCR lanes (0 = automatic)
  int ctas = 0;      // a plan's CTA count (0 = every SM)
  double ms = 0.0;   // the measured time
};
std::string tune_key(const std::string &gpu, const char *kind, size_t elem, int dir,
                     long long n, long long lines);
bool tune_lookup(const std::string &key, TuneChoice &out);
bool tune_table_empty();
void tune_store(const std::string &key, const TuneChoice &c);
bool tune_load(const char *path);
bool tune_save(const char *path);
void tune_clear();
std::string tune_format(const TuneChoice &c);  // "spec\talgo\tlanes\tctas\tms"

// penta_status.cu: status words, one slot per handle or plan in a fixed
// device array (slot 0: the handle-less calls).  Addresses are taken with
// `device` current.
constexpr int kStatusSlots = 4096;
int *status_word(int device, int slot);
int *device_status_word(int device);  // slot 0
int status_slot_acquire();            // a free slot, or 0 when none is left
void status_slot_release(int slot, int device);  // clears the word (synchronous)
// *bits = atomicExch(word, 0) on `stream`, then synchronises `stream`.
cudaError_t status_take(int device, int slot, cudaStream_t stream, int *bits);
// A kernel whose one wait never completes: raises STATUS_TIMEOUT_BIT in
// *status after `limit_ns`.
cudaError_t launch_bounded_wait_selftest(unsigned long long limit_ns, int *status,
                                         cudaStream_t stream);

// Bytes of caller scratch the global-scratch kernel needs.
template <typename F> inline size_t thomas_global_scratch(const Lines &L) {
  return (size_t)3 * (size_t)L.n * (size_t)L.n_sys * sizeof(F);
}

}  // namespace penta
