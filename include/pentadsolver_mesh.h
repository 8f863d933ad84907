/*
 * pentadsolver_mesh.h -- test grids: fixture files and the random benchmark mesh.
 *
 * The reference keeps these in header-only C++ test utilities, not in its
 * library; here they are part of the C ABI so that its tests and benchmarks
 * have a counterpart without linking C++ templates:
 *
 *   pentadsolver_fixture_info / _read   replace Mesh<Float>(file)
 *                                       (include/util/mesh.hpp:51-80) and
 *                                       DeviceMesh<Float>(file)'s host half
 *                                       (include/util/device_mesh.hpp:35-50);
 *   pentadsolver_*_fixture_write        writes that text format (the one
 *                                       test/gen_testcases.py:50-79 emits) or
 *                                       a binary form of the same content;
 *   pentadsolver_*_mesh_random          replaces Mesh<Float>(solve_dim, dims)
 *                                       (mesh.hpp:85-124) plus DeviceMesh's
 *                                       upload (device_mesh.hpp:52-65): the
 *                                       same grid, generated on the GPU.
 *
 * Arrays are ordered as everywhere in this library: dims[0] is the contiguous
 * axis, prod(dims) elements per array.
 */
#ifndef PENTADSOLVER_MESH_H_INCLUDED
#define PENTADSOLVER_MESH_H_INCLUDED

#include "pentad_common.hpp"

/* Fixture file formats (the `format` argument and result). */
#define PENTADSOLVER_FIXTURE_TEXT 0        /* the reference's text format */
#define PENTADSOLVER_FIXTURE_BINARY_F64 8  /* binary, FP64 arrays */
#define PENTADSOLVER_FIXTURE_BINARY_F32 4  /* binary, FP32 arrays */

/*
 * Text format (reference): whitespace-separated tokens
 *     ndims solvedim
 *     dims[0] ... dims[ndims-1]
 *     ds... dl... d... du... dw... x... u... u_float...
 * each array prod(dims) values, one line per array; u is the FP64 solution,
 * u_float the FP32 one.  Values are parsed in the "C" locale.
 *
 * Binary format (this library; little-endian):
 *     char[8] "PENTAFX1"; uint32 elem_bytes (8 or 4); uint32 ndims;
 *     uint32 solvedim; uint32 has_u; uint32 dims[ndims]; zero padding to a
 *     multiple of 8 bytes; then ds, dl, d, du, dw, x and, when has_u, u --
 *     prod(dims) elements of elem_bytes each.
 */

/* Header of a fixture file.  `dims` receives up to PENTAD_MAXDIM extents;
 * `format` one of PENTADSOLVER_FIXTURE_*.  INVALID_VALUE for a file that is
 * missing, malformed or of more than PENTAD_MAXDIM dimensions. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_fixture_info(const char *path, int *ndims,
                                                             int *solvedim, int *dims,
                                                             int *format);

/* Read the arrays of a fixture file into host arrays of prod(dims) elements.
 * From a text file the FP64 reader takes u from the FP64 solution line and the
 * FP32 reader from the FP32 line, parsing every value at its own precision,
 * as Mesh<double> and Mesh<float> do.  A binary file must hold the reader's
 * precision.  `u` may be NULL (not read); asking for u from a binary file
 * written without it returns PENTAD_STATUS_INVALID_VALUE.  Unlike the
 * reference, a short or malformed file is an error rather than zeros; a call
 * that fails writes nothing. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_D_fixture_read(
    const char *path, double *ds, double *dl, double *d, double *du, double *dw, double *x,
    double *u);
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_S_fixture_read(
    const char *path, float *ds, float *dl, float *d, float *du, float *dw, float *x,
    float *u);

/* Write a fixture file in `format` (text, or binary at the writer's own
 * precision).  Text values are written with enough digits to read back
 * bit-exactly at the writer's precision (17 significant digits FP64, 9 FP32);
 * the text u_float line is u rounded to FP32.  `u` may be NULL: the text
 * solution lines are then zeros and a binary file has no u. */
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_D_fixture_write(
    const char *path, int format, int ndims, int solvedim, const int *dims,
    const double *ds, const double *dl, const double *d, const double *du,
    const double *dw, const double *x, const double *u);
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_S_fixture_write(
    const char *path, int format, int ndims, int solvedim, const int *dims, const float *ds,
    const float *dl, const float *d, const float *du, const float *dw, const float *x,
    const float *u);

/* The random grid of Mesh<Float>(solvedim, dims) as the reference builds it
 * with `n_threads` OpenMP threads (thread t seeds std::mt19937_64 with t; the
 * grid depends on the count), written into DEVICE arrays of prod(dims)
 * elements on `stream` (a cudaStream_t; NULL = legacy default stream).
 * Bit-identical to the reference's host arrays for the same n_threads.  One
 * launch; asynchronous.  1 <= n_threads <= PENTADSOLVER_MESH_MAX_THREADS. */
#define PENTADSOLVER_MESH_MAX_THREADS 65536
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_D_mesh_random(
    const int *dims, int ndims, int solvedim, int n_threads, double *ds, double *dl,
    double *d, double *du, double *dw, double *x, void *stream);
EXTERN_C PENTAD_API pentadStatus_t pentadsolver_S_mesh_random(
    const int *dims, int ndims, int solvedim, int n_threads, float *ds, float *dl, float *d,
    float *du, float *dw, float *x, void *stream);

#endif /* PENTADSOLVER_MESH_H_INCLUDED */
