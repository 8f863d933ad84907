/*
 * pentadsolver_cuda.hpp -- the two-buffer form of the API.
 *
 * Mirrors the reference's include/pentadsolver_cuda.hpp:36-142 (written for its
 * MPI-CUDA backend): sizing reports a host and a device workspace and the
 * solve takes both buffers.  On one GPU the host workspace is always 0 bytes
 * and is ignored.  As in the reference this header shares its include guard
 * with pentadsolver.hpp, so a translation unit includes one or the other.
 *
 * The reference gives the two forms the same C names with different
 * parameter lists, which one shared library cannot export at once.  The
 * library therefore exports the two-buffer entry points under the
 * `_two_buffer` names below, and this header maps the reference's names onto
 * them with inline wrappers, so callers compile unchanged.
 */
#ifndef PENTADSOLVER_HPP_INCLUDED
#define PENTADSOLVER_HPP_INCLUDED

#include "pentadsolver_handle.hpp"

#include <stddef.h>

#ifdef __cplusplus
#define EXTERN_C extern "C"
#define PENTAD_INLINE inline
#else
#define EXTERN_C
#define PENTAD_INLINE static inline
#endif

#ifndef PENTAD_API
#if defined(__GNUC__)
#define PENTAD_API __attribute__((visibility("default")))
#else
#define PENTAD_API
#endif
#endif

/* Replaces include/pentadsolver_cuda.hpp:36-41. */
EXTERN_C PENTAD_API
void pentadsolver_create(pentadsolver_handle_t *handle, void *communicator,
                         int ndims, const int *num_procs);
EXTERN_C PENTAD_API
void pentadsolver_destroy(pentadsolver_handle_t *handle);

/* Exported two-buffer entry points. */
EXTERN_C PENTAD_API
void pentadsolver_D_gpsv_batch_buffer_size_two_buffer(
    pentadsolver_handle_t handle, const double *ds, const double *dl,
    const double *d, const double *du, const double *dw, const double *x,
    const int *t_dims, int t_ndim, int t_solvedim,
    size_t *t_workspace_in_bytes_host, size_t *t_workspace_in_bytes_device);
EXTERN_C PENTAD_API
void pentadsolver_S_gpsv_batch_buffer_size_two_buffer(
    pentadsolver_handle_t handle, const float *ds, const float *dl,
    const float *d, const float *du, const float *dw, const float *x,
    const int *t_dims, int t_ndim, int t_solvedim,
    size_t *t_workspace_in_bytes_host, size_t *t_workspace_in_bytes_device);
EXTERN_C PENTAD_API
void pentadsolver_D_gpsv_batch_two_buffer(
    pentadsolver_handle_t handle, const double *ds, const double *dl,
    const double *d, const double *du, const double *dw, double *x,
    const int *t_dims, int t_ndim, int t_solvedim, void *t_buffer_h,
    void *t_buffer_d);
EXTERN_C PENTAD_API
void pentadsolver_S_gpsv_batch_two_buffer(
    pentadsolver_handle_t handle, const float *ds, const float *dl,
    const float *d, const float *du, const float *dw, float *x,
    const int *t_dims, int t_ndim, int t_solvedim, void *t_buffer_h,
    void *t_buffer_d);

/* Replaces include/pentadsolver_cuda.hpp:67-78. */
PENTAD_INLINE void pentadsolver_D_gpsv_batch_buffer_size_ext(
    pentadsolver_handle_t handle, const double *ds, const double *dl,
    const double *d, const double *du, const double *dw, const double *x,
    const int *t_dims, int t_ndim, int t_solvedim,
    size_t *t_workspace_in_bytes_host, size_t *t_workspace_in_bytes_device) {
  pentadsolver_D_gpsv_batch_buffer_size_two_buffer(
      handle, ds, dl, d, du, dw, x, t_dims, t_ndim, t_solvedim,
      t_workspace_in_bytes_host, t_workspace_in_bytes_device);
}
PENTAD_INLINE void pentadsolver_S_gpsv_batch_buffer_size_ext(
    pentadsolver_handle_t handle, const float *ds, const float *dl,
    const float *d, const float *du, const float *dw, const float *x,
    const int *t_dims, int t_ndim, int t_solvedim,
    size_t *t_workspace_in_bytes_host, size_t *t_workspace_in_bytes_device) {
  pentadsolver_S_gpsv_batch_buffer_size_two_buffer(
      handle, ds, dl, d, du, dw, x, t_dims, t_ndim, t_solvedim,
      t_workspace_in_bytes_host, t_workspace_in_bytes_device);
}

/* Replaces include/pentadsolver_cuda.hpp:116-128. */
PENTAD_INLINE void pentadsolver_D_gpsv_batch(
    pentadsolver_handle_t handle, const double *ds, const double *dl,
    const double *d, const double *du, const double *dw, double *x,
    const int *t_dims, int t_ndim, int t_solvedim, void *t_buffer_h,
    void *t_buffer_d) {
  pentadsolver_D_gpsv_batch_two_buffer(handle, ds, dl, d, du, dw, x, t_dims,
                                       t_ndim, t_solvedim, t_buffer_h,
                                       t_buffer_d);
}
PENTAD_INLINE void pentadsolver_S_gpsv_batch(
    pentadsolver_handle_t handle, const float *ds, const float *dl,
    const float *d, const float *du, const float *dw, float *x,
    const int *t_dims, int t_ndim, int t_solvedim, void *t_buffer_h,
    void *t_buffer_d) {
  pentadsolver_S_gpsv_batch_two_buffer(handle, ds, dl, d, du, dw, x, t_dims,
                                       t_ndim, t_solvedim, t_buffer_h,
                                       t_buffer_d);
}

#ifdef __cplusplus
/* Replaces include/pentadsolver_cuda.hpp:80-90 and :130-141. */
inline void pentadsolver_gpsv_batch_buffer_size_ext(
    pentadsolver_handle_t handle, const double *ds, const double *dl,
    const double *d, const double *du, const double *dw, const double *x,
    const int *t_dims, int t_ndim, int t_solvedim,
    size_t *t_workspace_in_bytes_host, size_t *t_workspace_in_bytes_device) {
  pentadsolver_D_gpsv_batch_buffer_size_two_buffer(
      handle, ds, dl, d, du, dw, x, t_dims, t_ndim, t_solvedim,
      t_workspace_in_bytes_host, t_workspace_in_bytes_device);
}
inline void pentadsolver_gpsv_batch_buffer_size_ext(
    pentadsolver_handle_t handle, const float *ds, const float *dl,
    const float *d, const float *du, const float *dw, const float *x,
    const int *t_dims, int t_ndim, int t_solvedim,
    size_t *t_workspace_in_bytes_host, size_t *t_workspace_in_bytes_device) {
  pentadsolver_S_gpsv_batch_buffer_size_two_buffer(
      handle, ds, dl, d, du, dw, x, t_dims, t_ndim, t_solvedim,
      t_workspace_in_bytes_host, t_workspace_in_bytes_device);
}
inline void pentadsolver_gpsv_batch(pentadsolver_handle_t handle,
                                    const double *ds, const double *dl,
                                    const double *d, const double *du,
                                    const double *dw, double *x,
                                    const int *t_dims, int t_ndim,
                                    int t_solvedim, void *t_buffer_h,
                                    void *t_buffer_d) {
  pentadsolver_D_gpsv_batch_two_buffer(handle, ds, dl, d, du, dw, x, t_dims,
                                       t_ndim, t_solvedim, t_buffer_h,
                                       t_buffer_d);
}
inline void pentadsolver_gpsv_batch(pentadsolver_handle_t handle,
                                    const float *ds, const float *dl,
                                    const float *d, const float *du,
                                    const float *dw, float *x,
                                    const int *t_dims, int t_ndim,
                                    int t_solvedim, void *t_buffer_h,
                                    void *t_buffer_d) {
  pentadsolver_S_gpsv_batch_two_buffer(handle, ds, dl, d, du, dw, x, t_dims,
                                       t_ndim, t_solvedim, t_buffer_h,
                                       t_buffer_d);
}
#endif

EXTERN_C PENTAD_API const char *pentadsolver_kernel_that_ran(int dir);

#endif /* PENTADSOLVER_HPP_INCLUDED */
