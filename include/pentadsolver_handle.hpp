/*
 * pentadsolver_handle.hpp -- the library context type.
 *
 * Same type as the reference's single-node build
 * (include/pentadsolver_handle.hpp:4-5): an opaque pointer.  Here it points to
 * a real per-handle context (device properties, the record of the kernels that
 * ran, the autotuner's cache); a null or never-created handle is accepted and
 * means the process-wide default context of the current device, because the
 * reference's CPU apps pass a value-initialised handle without creating it.
 */
#ifndef PENTADSOLVER_HANDLE_HPP_INCLUDED
#define PENTADSOLVER_HANDLE_HPP_INCLUDED

#ifdef __cplusplus
using pentadsolver_handle_t = void *;
#else
typedef void *pentadsolver_handle_t;
#endif

#endif /* PENTADSOLVER_HANDLE_HPP_INCLUDED */
