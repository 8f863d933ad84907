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

/* Synchronise `stream`, then read and clear the device status bits raised by
 * the solves issued so far on the current device (bit 0: a pivot was zero or
 * not finite).  Returns PENTAD_STATUS_ZERO_PIVOT when bit 0 was set. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_status_check(pentadsolver_handle_t handle,
                                                  void *stream, int *bits);

/* Per-handle algorithm choice for one direction (0 = x, 1 = middle, 2 =
 * outermost): "naive", "transpose", "thomas-pcr", "shared-fact", "auto", or
 * NULL to clear.  Environment selectors (PENTA_XALGO ...) still win, as in the
 * reference.  `pcr_lanes` (0 = automatic) plays PENTA_PCR_LANES's role. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_set_algo(pentadsolver_handle_t handle,
                                              int dir, const char *algo,
                                              int pcr_lanes);

/* Kernel family the handle's last solve along `dir` launched, and the exact
 * variant (e.g. "thomas-pcr:tiled S16 P2 R1 x8"). */
EXTERN_C PENTAD_API const char *pentadsolver_kernel_that_ran_ex(
    pentadsolver_handle_t handle, int dir);
EXTERN_C PENTAD_API const char *pentadsolver_variant_that_ran(pentadsolver_handle_t handle,
                                                   int dir);

EXTERN_C PENTAD_API const char *pentadsolver_status_string(pentadStatus_t status);

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
 * stream); arguments otherwise as pentadsolver_D_gpsv_batch. */
#define PENTADSOLVER_NOALLOC_MAX_BYTES (16u * 1024u * 1024u)
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_D_gpsv_batch_noalloc(
    pentadsolver_handle_t handle, const double *ds, const double *dl,
    const double *d, const double *du, const double *dw, double *x,
    const int *t_dims, int t_ndim, int t_solvedim, void *stream);

#endif /* PENTADSOLVER_EXT_H_INCLUDED */
