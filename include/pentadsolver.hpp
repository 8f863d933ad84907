/*
 * pentadsolver.hpp -- drop-in public API of the B200 pentadiagonal solver.
 *
 * Every declaration below has the name, signature and meaning of the
 * reference's include/pentadsolver.hpp, so apps/adi_cuda.cu, the verifiers and
 * the reference's GPU tests compile and link against this library unchanged.
 * Each entry point names the reference declaration it replaces.
 *
 * Contract (reference include/pentadsolver.hpp:88-131):
 *   - ds, dl, d, du, dw, x are dense device arrays of the grid t_dims[0..t_ndim)
 *     with t_dims[0] contiguous; the systems are the lines along t_solvedim.
 *   - Row i: ds[i] x[i-2] + dl[i] x[i-1] + d[i] x[i] + du[i] x[i+1]
 *            + dw[i] x[i+2] = b[i].  Couplings that leave the line (ds at rows
 *     0,1; dl at row 0; du at row n-1; dw at rows n-2,n-1) are ignored
 *     whatever they hold.  No pivoting: the matrix must be safely factorable
 *     (diagonal dominance is sufficient).
 *   - x holds the right-hand side on entry and the solution on exit.
 *   - t_buffer is caller-allocated device memory of at least
 *     pentadsolver_*_gpsv_batch_buffer_size_ext() bytes.  The solve path
 *     allocates nothing.
 *   - The call is asynchronous on the legacy default stream; synchronise
 *     before reading x.  Invalid arguments and launch failures are reported
 *     on stderr (the reference's behaviour, pentad_cuda.cu:1534-1539); the
 *     `_ex` entry points of pentadsolver_ext.h return a status instead.
 *   - Algorithm selection: PENTA_XALGO, PENTA_YALGO, PENTA_ZALGO, PENTA_YZALGO
 *     (values naive | transpose | thomas-pcr | shared-fact | auto) and
 *     PENTA_PCR_LANES, read on every call as in the reference.
 */
#ifndef PENTADSOLVER_HPP_INCLUDED
#define PENTADSOLVER_HPP_INCLUDED

#include "pentadsolver_handle.hpp"

#include <stddef.h>

#ifdef __cplusplus
#define EXTERN_C extern "C"
#define PENTAD_NODISCARD [[nodiscard]]
#else
#define EXTERN_C
#define PENTAD_NODISCARD
#endif

#ifndef PENTAD_API
#if defined(__GNUC__)
#define PENTAD_API __attribute__((visibility("default")))
#else
#define PENTAD_API
#endif
#endif

/* Context functions.  Replaces include/pentadsolver.hpp:36-41.  The MPI
 * arguments are accepted and ignored (one GPU, no communicator). */
EXTERN_C PENTAD_API
void pentadsolver_create(pentadsolver_handle_t *handle, void *communicator,
                         int ndims, const int *num_procs);

EXTERN_C PENTAD_API
void pentadsolver_destroy(pentadsolver_handle_t *handle);

/* Scratch size in bytes.  Replaces include/pentadsolver.hpp:64-73 (which the
 * reference declares but, defining it with a non-const x, never exports as a
 * C symbol; here it is exported). */
EXTERN_C PENTAD_NODISCARD PENTAD_API
size_t pentadsolver_D_gpsv_batch_buffer_size_ext(
    pentadsolver_handle_t handle, const double *ds, const double *dl,
    const double *d, const double *du, const double *dw, const double *x,
    const int *t_dims, int t_ndim, int t_solvedim);
EXTERN_C PENTAD_NODISCARD PENTAD_API
size_t pentadsolver_S_gpsv_batch_buffer_size_ext(
    pentadsolver_handle_t handle, const float *ds, const float *dl,
    const float *d, const float *du, const float *dw, const float *x,
    const int *t_dims, int t_ndim, int t_solvedim);

#ifdef __cplusplus
/* Replaces include/pentadsolver.hpp:76-83. */
PENTAD_NODISCARD PENTAD_API size_t pentadsolver_gpsv_batch_buffer_size_ext(
    pentadsolver_handle_t handle, const double *ds, const double *dl,
    const double *d, const double *du, const double *dw, const double *x,
    const int *t_dims, int t_ndim, int t_solvedim);
PENTAD_NODISCARD PENTAD_API size_t pentadsolver_gpsv_batch_buffer_size_ext(
    pentadsolver_handle_t handle, const float *ds, const float *dl,
    const float *d, const float *du, const float *dw, const float *x,
    const int *t_dims, int t_ndim, int t_solvedim);
#endif

/* Batched solve.  Replaces include/pentadsolver.hpp:107-118. */
EXTERN_C PENTAD_API
void pentadsolver_D_gpsv_batch(pentadsolver_handle_t handle, const double *ds,
                               const double *dl, const double *d,
                               const double *du, const double *dw, double *x,
                               const int *t_dims, int t_ndim, int t_solvedim,
                               void *t_buffer);

EXTERN_C PENTAD_API
void pentadsolver_S_gpsv_batch(pentadsolver_handle_t handle, const float *ds,
                               const float *dl, const float *d, const float *du,
                               const float *dw, float *x, const int *t_dims,
                               int t_ndim, int t_solvedim, void *t_buffer);

#ifdef __cplusplus
/* Replaces include/pentadsolver.hpp:120-131. */
PENTAD_API void pentadsolver_gpsv_batch(pentadsolver_handle_t handle, const double *ds,
                             const double *dl, const double *d,
                             const double *du, const double *dw, double *x,
                             const int *t_dims, int t_ndim, int t_solvedim,
                             void *t_buffer);

PENTAD_API void pentadsolver_gpsv_batch(pentadsolver_handle_t handle, const float *ds,
                             const float *dl, const float *d, const float *du,
                             const float *dw, float *x, const int *t_dims,
                             int t_ndim, int t_solvedim, void *t_buffer);
#endif

/* Name of the kernel family the most recent solve along each direction
 * launched: dir 0 = x (solvedim 0), 2 = outermost, 1 = any middle dimension.
 * One of "naive", "transpose", "thomas-pcr", "shared-fact", or "none" before
 * any solve.  Replaces the reference's extra export
 * src/cuda/singlenode/pentad_cuda.cu:1159-1161, which apps/adi_cuda.cu
 * declares itself and uses to pick its traffic model. */
EXTERN_C PENTAD_API const char *pentadsolver_kernel_that_ran(int dir);

#endif /* PENTADSOLVER_HPP_INCLUDED */
