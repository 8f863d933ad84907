/*
 * pentadsolver_ext.h -- extension C ABI of the B200 pentadiagonal solver.
 *
 * These entry points have no counterpart in the reference's API; they add
 * what its void, default-stream interface cannot express: an explicit CUDA
 * stream (passed as void*, i.e. a cudaStream_t), a returned pentadStatus_t,
 * the buffer size the caller actually passed, per-handle algorithm selection
 * and the record of what ran.  Everything is plain C: pointers and sizes.
 *
 * Array conventions are those of pentadsolver.hpp.
 */
#ifndef PENTADSOLVER_EXT_H_INCLUDED
#define PENTADSOLVER_EXT_H_INCLUDED

#include "pentad_common.hpp"
#include "pentadsolver_handle.hpp"

#include <stddef.h>

/* Scratch bytes a solve of this shape may use, for element size 8 (double)
 * or 4 (float).  The same value the reference-named sizing functions return. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_buffer_size_ex(
    pentadsolver_handle_t handle, int elem_bytes, const int *t_dims,
    int t_ndim, int t_solvedim, size_t *bytes);

/* Solve on `stream`.  `t_buffer_bytes` is the size of t_buffer; the call
 * returns PENTAD_STATUS_INVALID_VALUE instead of overrunning it.  Launch
 * failures return PENTAD_STATUS_EXECUTION_FAILED.  Asynchronous: pivot
 * problems are reported later by pentadsolver_status_check. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_D_gpsv_batch_ex(
    pentadsolver_handle_t handle, const double *ds, const double *dl,
    const double *d, const double *du, const double *dw, double *x,
    const int *t_dims, int t_ndim, int t_solvedim, void *t_buffer,
    size_t t_buffer_bytes, void *stream);
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_S_gpsv_batch_ex(
    pentadsolver_handle_t handle, const float *ds, const float *dl,
    const float *d, const float *du, const float *dw, float *x,
    const int *t_dims, int t_ndim, int t_solvedim, void *t_buffer,
    size_t t_buffer_bytes, void *stream);

/* Read and clear the status bits raised by this handle's solves (bit 0: a
 * pivot was zero or not finite; bit 1: a wait inside a kernel ran out), then
 * synchronise `stream`.  The read and the clear are one atomic exchange on the
 * device, issued on `stream`: a bit raised by a kernel on another stream is
 * either returned now or kept for the next check.  Every created handle has a
 * status word of its own (a slot of a fixed device array, so nothing is
 * allocated); the NULL handle's word is shared by all handle-less calls on
 * the device, and so is it for handles created after the array's 4095 slots
 * are taken.  Returns PENTAD_STATUS_ZERO_PIVOT when bit 0 was set, and
 * PENTAD_STATUS_INVALID_VALUE when the handle is bound to another device
 * than the current one. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_status_check(pentadsolver_handle_t handle,
                                                  void *stream, int *bits);

/* Test of the bounded waits every kernel uses: launches on `stream` a kernel
 * whose one mbarrier wait can never complete; the wait gives up after
 * `limit_us` microseconds (1 .. 1,000,000) and raises bit 1 in the handle's
 * status word, as a solve does when one of its waits runs out.  The device
 * stays usable; pentadsolver_status_check then reports the bit. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_selftest_bounded_wait(
    pentadsolver_handle_t handle, unsigned limit_us, void *stream);

/* Per-handle algorithm choice for one direction (0 = x, 1 = middle, 2 =
 * outermost): "naive", "transpose", "thomas-pcr", "shared-fact", "auto", or
 * NULL to clear.  Environment selectors (PENTA_XALGO ...) still win, as in the
 * reference.  `pcr_lanes` (0 = automatic) plays PENTA_PCR_LANES's role. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_set_algo(pentadsolver_handle_t handle,
                                              int dir, const char *algo,
                                              int pcr_lanes);

/* Kernel choice within a family for one direction of this handle, as an
 * autotuner sets it: "auto" (or NULL), "no-tmem" (skip the Tensor-Memory
 * kernel), "no-tma" (no TMA kernel at all), "tmem=ST,XST" (its variant with
 * ST forward and XST read-back stages), "tma=R,ST,XST,SCR" (the older TMA
 * kernel's variant).  When set, it replaces the PENTA_NO_TMEM / PENTA_NO_TMA /
 * PENTA_TMEM_VARIANT / PENTA_TMA_VARIANT environment variables for this
 * handle and direction. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_set_tuning(pentadsolver_handle_t handle,
                                                           int dir, const char *spec);

/* Kernel family the handle's last solve along `dir` launched, and the exact
 * variant (e.g. "thomas-pcr:tiled S16 P2 R1 x8"). */
EXTERN_C PENTAD_API const char *pentadsolver_kernel_that_ran_ex(
    pentadsolver_handle_t handle, int dir);
EXTERN_C PENTAD_API const char *pentadsolver_variant_that_ran(pentadsolver_handle_t handle,
                                                   int dir);

EXTERN_C PENTAD_API const char *pentadsolver_status_string(pentadStatus_t status);

/* ---- Plans: many grids in one persistent launch ---------------------------
 * No counterpart in the reference.  A plan solves a fixed set of grids (any
 * mix of shapes, one precision, one solvedim) with one launch of the batched
 * Tensor-Memory kernel; grids that kernel does not take (lines too short or
 * too long) are solved one by one inside the same execute.  Creating a plan
 * writes its job table into the caller's buffer with a copy that returns
 * when done and waits for no other stream, so the buffer must not be in use
 * by queued work; executing it launches kernels on `stream` only, so an
 * execute can be captured into a CUDA graph and replayed.  The grids' arrays and the buffer
 * must stay valid and unmoved for the plan's lifetime; their contents may
 * change between executes (x is solved in place each time). */
typedef struct pentadsolver_grid {
  const void *ds, *dl, *d, *du, *dw; /* prod(dims) elements each, dims[0] contiguous */
  void *x;                           /* right-hand side in, solution out */
  int ndim;
  int dims[PENTAD_MAXDIM];
} pentadsolver_grid_t;
typedef struct pentadsolver_plan_s *pentadsolver_plan_t;

EXTERN_C PENTAD_API pentadStatus_t pentadsolver_plan_buffer_size(
    pentadsolver_handle_t handle, int elem_bytes, int count, const pentadsolver_grid_t *grids,
    int solvedim, size_t *bytes);
/* `ctas` = 0 uses every SM; fewer leaves SMs to concurrent work. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_plan_create(
    pentadsolver_handle_t handle, int elem_bytes, int count, const pentadsolver_grid_t *grids,
    int solvedim, void *buffer, size_t buffer_bytes, int ctas, pentadsolver_plan_t *plan);
/* The same with the job table and the scratch in separate memory: plans
 * that never run at the same time (e.g. the x, y and z plans of one ADI
 * iteration on one stream) may share one scratch region. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_plan_sizes(
    pentadsolver_handle_t handle, int elem_bytes, int count, const pentadsolver_grid_t *grids,
    int solvedim, size_t *table_bytes, size_t *scratch_bytes);
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_plan_create_split(
    pentadsolver_handle_t handle, int elem_bytes, int count, const pentadsolver_grid_t *grids,
    int solvedim, void *table, size_t table_bytes, void *scratch, size_t scratch_bytes,
    int ctas, pentadsolver_plan_t *plan);
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_plan_execute(pentadsolver_plan_t plan,
                                                              void *stream);
/* As pentadsolver_plan_execute.  With PENTADSOLVER_PLAN_REUSE_FP32 in `flags`
 * a refinement plan keeps the FP32 copies of the coefficients that an earlier
 * execute of this plan made, instead of casting them again: the caller
 * vouches that the grids' coefficients have not changed since (an ADI loop's
 * fixed coefficients).  The first execute, and any after one whose cast
 * did not launch, casts anyway.  Ignored by plans without refinement; other bits are invalid.
 * In a captured execute the choice is made at capture. */
#define PENTADSOLVER_PLAN_REUSE_FP32 1
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_plan_execute_ex(pentadsolver_plan_t plan,
                                                                 void *stream, int flags);
EXTERN_C PENTAD_API const char *pentadsolver_plan_describe(pentadsolver_plan_t plan);
/* Times `reps` executes of the plan with each of several CTA counts (all SMs,
 * 90%, 75%, 50%), keeps the fastest for this plan and records it in the
 * tuning table for plans of its class (see pentadsolver_tuning_key).  The
 * executes solve the grids in place again and again.  Synchronises `stream`. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_autotune_plan(pentadsolver_plan_t plan,
                                                              int reps, void *stream,
                                                              int *best_ctas);
/* As pentadsolver_status_check, for the kernels of this plan's executes: every
 * plan reports into a status word of its own. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_plan_status_check(pentadsolver_plan_t plan,
                                                                  void *stream, int *bits);
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_plan_destroy(pentadsolver_plan_t plan);

/* ---- Mixed precision: FP32 sweeps, FP64 residual and correction -----------
 * No counterpart in the reference.  Solves the FP64 system with FP32 sweeps
 * (the library's FP32 kernels on FP32 copies of the coefficients) and `steps`
 * rounds of iterative refinement: r = b - A x in FP64, an FP32 sweep of r,
 * x += d in FP64.  With `reuse_fp32_coefficients` the copies already in the
 * buffer (from an earlier call with the same coefficients) are used as they
 * are.  The buffer's first 16 bytes receive (max|last correction|, max|x|)
 * of the last step, an estimate of the remaining forward error
 * (pentadsolver_refine_estimate reads them; zeros when steps = 0).  With
 * steps <= 1 the first iterate stays in FP32 and b in x until the result is
 * written (no FP64 copies of either): fewer bytes, the same values. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_refine_buffer_size(
    pentadsolver_handle_t handle, const int *t_dims, int t_ndim, int t_solvedim, size_t *bytes);
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_D_gpsv_batch_refine(
    pentadsolver_handle_t handle, const double *ds, const double *dl, const double *d,
    const double *du, const double *dw, double *x, const int *t_dims, int t_ndim,
    int t_solvedim, int steps, int reuse_fp32_coefficients, void *t_buffer,
    size_t t_buffer_bytes, void *stream);
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_refine_estimate(const void *t_buffer,
                                                                 void *stream, double *out);
/* The same for a set of FP64 grids as one plan (executed with
 * pentadsolver_plan_execute): one batched FP32 launch per sweep plus one
 * launch per FP64 step; pentadsolver_plan_estimates gives (max|d|, max|x|)
 * per grid. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_refine_plan_buffer_size(
    pentadsolver_handle_t handle, int count, const pentadsolver_grid_t *grids, int solvedim,
    size_t *bytes);
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_refine_plan_create(
    pentadsolver_handle_t handle, int count, const pentadsolver_grid_t *grids, int solvedim,
    int steps, void *buffer, size_t buffer_bytes, int ctas, pentadsolver_plan_t *plan);
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_plan_estimates(pentadsolver_plan_t plan,
                                                               void *stream, double *out);

/* ---- Autotuning ----------------------------------------------------------
 * No counterpart in the reference (whose selection is the fixed heuristic of
 * src/cuda/singlenode/pentad_cuda.cu:1143-1174 plus PENTA_PCR_LANES).  A
 * process-wide tuning table maps a shape class to the kernel choice that
 * measured fastest; the class key is
 *     <GPU name>|<solve, plan or refine>|<f64 or f32>|<x or yz>|n<N>|l<L>
 * with N the line length (a plan: its longest) and L the number of lines (a
 * plan: all of them), each rounded up to a power of two.  The automatic
 * selection of every handle consults it for shapes that neither environment
 * selectors nor the handle's own choices fix, and plan creation with ctas = 0
 * takes its CTA count from it -- so a caller of the reference's interface
 * gets tuned kernels without code changes.  On first use the table is read
 * from the file named by PENTA_TUNING_CACHE when that variable is set; files
 * hold one entry per line, "key<TAB>spec<TAB>algo<TAB>lanes<TAB>ctas<TAB>ms"
 * (spec as pentadsolver_set_tuning takes it, "auto" for none). */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_tuning_load(const char *path);
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_tuning_save(const char *path);
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_tuning_clear(void);
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_tuning_set(const char *key, const char *spec,
                                                           const char *algo, int lanes,
                                                           int ctas, double ms);
/* The entry for `key` as "spec<TAB>algo<TAB>lanes<TAB>ctas<TAB>ms";
 * PENTAD_STATUS_INVALID_VALUE when there is none or `len` is too small. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_tuning_lookup(const char *key, char *out,
                                                              size_t len);
/* The key of a shape (`kind` "solve", "plan" or "refine"; for plans the
 * grid's own line length and lines); `gpu_name` NULL: the current device. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_tuning_key(const char *gpu_name,
                                                           const char *kind, int elem_bytes,
                                                           const int *t_dims, int t_ndim,
                                                           int t_solvedim, char *out,
                                                           size_t len);
/* Times, on the caller's problem and stream, each candidate kernel choice --
 * the Tensor-Memory kernel's ring variants, the older TMA kernels, the
 * cp.async kernel with two lanes or one lane per line -- `reps` solves each,
 * records the fastest in the tuning table for this shape's class, and writes
 * a report (one line per distinct kernel variant, fastest first:
 * "label<TAB>spec<TAB>algo<TAB>lanes<TAB>variant<TAB>ms") when `report` is
 * not NULL.  The trial solves overwrite x; `x_save` (device memory of x's
 * size, or NULL) keeps it and puts it back at the end.  Synchronises
 * `stream`. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_autotune_solve(
    pentadsolver_handle_t handle, int elem_bytes, const void *ds, const void *dl,
    const void *d, const void *du, const void *dw, void *x, void *x_save, const int *t_dims,
    int t_ndim, int t_solvedim, void *t_buffer, size_t t_buffer_bytes, int reps, void *stream,
    char *report, size_t report_len);

/* ---- ADI iterations as one CUDA graph --------------------------------------
 * The loop of the reference's ADI application (apps/adi_cuda.cu:167-176: one
 * pentadsolver_gpsv_batch call per direction and step) captured once:
 * `iterations` steps of x, then y, then z solves of one grid in place (through
 * pentadsolver_{D,S}_gpsv_batch_ex with `handle`, so its algorithm choices --
 * shared factorisation with its table cached across steps, for instance --
 * hold), replayed with one call.  `t_buffer` is the x direction's
 * reference-sized buffer (pentadsolver_buffer_size_ex with solvedim 0); an
 * eager warm-up before capture solves a copy of x kept in its unused tail, so
 * x is untouched until the first replay and nothing is allocated.  Creation
 * synchronises the device.  The arrays and the buffer must stay valid while
 * the graph lives. */
typedef struct pentadsolver_adi_s *pentadsolver_adi_t;
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_adi_create(
    pentadsolver_handle_t handle, int elem_bytes, const void *ds, const void *dl, const void *d,
    const void *du, const void *dw, void *x, const int *t_dims, int t_ndim, int iterations,
    void *t_buffer, size_t t_buffer_bytes, pentadsolver_adi_t *adi);
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_adi_replay(pentadsolver_adi_t adi, void *stream);
EXTERN_C PENTAD_API int pentadsolver_adi_launches(pentadsolver_adi_t adi);
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_adi_destroy(pentadsolver_adi_t adi);

/* ---- Serving handle: a continuous-batching request loop -------------------
 * No counterpart in the reference.  Requests -- one FP64 grid (the caller's
 * device arrays; x is the right-hand side in and the solution out) and a
 * solve direction, with the forward-error tolerance the caller needs -- are
 * submitted as they arrive; pentadsolver_server_progress completes finished
 * batches and launches new ones: the queued requests sharing the oldest
 * one's solve direction and precision class, as one plan (one persistent
 * launch), on the next of `n_streams` streams, while fewer than
 * `max_in_flight` batches run -- so batches overlap and late arrivals join the
 * next batch as memory frees.  All batch memory comes from `arena` (device
 * memory, 256-byte aligned, the HBM budget); a batch that does not fit is
 * shortened, and a request that alone exceeds the arena completes at once
 * with PENTADSOLVER_SERVER_REJECTED_BIT.  Under PENTADSOLVER_SERVE_MIXED,
 * requests with tol >= 1e-10 take FP32 sweeps + `refine_steps` FP64
 * refinement steps along a direction where pentadsolver_server_calibrate
 * measured that form faster than plain FP64 (everywhere if not measured);
 * PENTADSOLVER_SERVE_SEQUENTIAL solves one request at a time (the baseline).
 * Completed requests are read with pentadsolver_server_poll, each with the
 * status bits of its batch (as pentadsolver_status_check reports them).
 * The server's streams are non-blocking: work that writes a request's arrays
 * must have completed before the progress call that launches it.  At most
 * min(n_streams, max_in_flight) batches run at once, one per stream.
 * Not thread-safe: drive one server from one thread. */
typedef struct pentadsolver_server_s *pentadsolver_server_t;
#define PENTADSOLVER_SERVE_FP64 0
#define PENTADSOLVER_SERVE_MIXED 1
#define PENTADSOLVER_SERVE_SEQUENTIAL 2
#define PENTADSOLVER_SERVER_REJECTED_BIT (1 << 30)
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_server_create(
    pentadsolver_handle_t handle, void *arena, size_t arena_bytes, int policy, int n_streams,
    int max_batch, int max_in_flight, int refine_steps, pentadsolver_server_t *server);
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_server_submit(pentadsolver_server_t server,
                                                              const pentadsolver_grid_t *grid,
                                                              int solvedim, double tol,
                                                              unsigned long long *id);
/* wait = 0: complete what has finished and launch what fits, then return;
 * wait = 1: run until every submitted request has completed. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_server_progress(pentadsolver_server_t server,
                                                                int wait);
/* Up to `capacity` completed requests: their ids and status bits. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_server_poll(pentadsolver_server_t server,
                                                            unsigned long long *ids,
                                                            int *bits, int capacity, int *n);
/* out[0..count): queued, in flight, arena bytes used, arena peak, arena size,
 * batches launched. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_server_stats(pentadsolver_server_t server,
                                                             size_t *out, int count);
/* Times a plain FP64 plan and a refinement plan of `sample` along each solve
 * direction (`reps` executes each, the sample's x overwritten; arena memory,
 * nothing in flight) and keeps, per direction, whether the refined form was
 * faster; ms[2d], ms[2d + 1] receive the two times when ms is not NULL. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_server_calibrate(pentadsolver_server_t server,
                                                                 const pentadsolver_grid_t *sample,
                                                                 int reps, double *ms);
/* Waits for the batches in flight, then frees the server (not the arena). */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_server_destroy(pentadsolver_server_t server);

/* ---- Slab decomposition over several GPUs ----------------------------------
 * The multi-GPU form of the ADI sweep.  The reference distributes one solve
 * direction over MPI ranks and exchanges a reduced system through host memory
 * (src/cuda/mpi/pentad_cuda.cu:929-955, :529-555); here a grid of
 * nx x ny x nz points (x contiguous) is split into `parts` slabs along z, one
 * per GPU: x and y lines lie inside a slab and are solved in place, and one
 * all-to-all of equal blocks turns the z slabs into y slabs (rank r: y in
 * [r ny/parts, (r+1) ny/parts), all z, as [z][y][x]) in which z lines are
 * local, and back.  These two kernels are the data movement around that
 * exchange: pack gathers, for every destination rank r, the rank's block
 * send[r][zl][yl][x] = zslab[zl][r ny/parts + yl][x] (the all-to-all's
 * receive buffer is then the y slab itself); unpack scatters what the way
 * back receives, recv[r][zl][yl][x], into the z slab.  nz_local is the slab's
 * own z extent; ny must be a multiple of parts.  Asynchronous on `stream`. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_slab_pack(int elem_bytes, const void *zslab,
                                                          void *send, int nx, int ny,
                                                          int nz_local, int parts, void *stream);
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_slab_unpack(int elem_bytes, const void *recv,
                                                            void *zslab, int nx, int ny,
                                                            int nz_local, int parts,
                                                            void *stream);

/* No counterpart in the reference.  An FP64 solve that allocates nothing and
 * takes no scratch buffer, for callers that cannot call cudaMalloc around a
 * solve: applications whose device memory is all owned by their own pool,
 * solve loops where cudaMalloc/cudaFree would synchronise the device, and code
 * written against the reference's CPU interface that passes no t_buffer.  It
 * runs the global-scratch Thomas kernel with its scratch in a fixed device
 * array of PENTADSOLVER_NOALLOC_MAX_BYTES that the library carries on every
 * GPU that loads it, until the process exits.  Limits and rules:
 *   - the grid may have at most PENTADSOLVER_NOALLOC_MAX_BYTES / 24 points
 *     (699,050; e.g. 88^3); larger grids return PENTAD_STATUS_INVALID_VALUE
 *     and a message on stderr, before any device work;
 *   - all calls on a device share the array: calls that may overlap on the
 *     GPU (unordered streams, several host threads) race and corrupt each
 *     other's results; nothing needs clearing between ordered calls;
 *   - the first call on each device takes the array's device address
 *     (cudaGetSymbolAddress) with that device current, so make that first
 *     call before any stream capture on the device.
 * Asynchronous on `stream` (a cudaStream_t, or NULL for the legacy default
 * stream).  `handle` (NULL: the current device's default context) receives
 * the status bits, read by pentadsolver_status_check; arguments and shape
 * rules otherwise as pentadsolver_D_gpsv_batch. */
#define PENTADSOLVER_NOALLOC_MAX_BYTES (16u * 1024u * 1024u)
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_D_gpsv_batch_noalloc(
    pentadsolver_handle_t handle, const double *ds, const double *dl,
    const double *d, const double *du, const double *dw, double *x,
    const int *t_dims, int t_ndim, int t_solvedim, void *stream);

#endif /* PENTADSOLVER_EXT_H_INCLUDED */
