/*
 * pentad_common.hpp -- status codes shared by the C ABI.
 *
 * The enumerators and their values are those of the reference's
 * include/pentad_common.hpp:26-37 (a copy of the cuSPARSE status enum), kept
 * identical so code that switches on them keeps working.  The reference
 * defines the enum but returns it from nothing; here the `_ex` entry points of
 * pentadsolver_ext.h return it.
 */
#ifndef PENTAD_COMMON_H__
#define PENTAD_COMMON_H__

#ifdef __cplusplus
#define EXTERN_C extern "C"
#else
#define EXTERN_C
#endif

#ifndef PENTAD_API
#if defined(__GNUC__)
#define PENTAD_API __attribute__((visibility("default")))
#else
#define PENTAD_API
#endif
#endif

/* Largest t_ndim the library accepts (the reference fixes 3; any rank works
 * here because every solve reduces to (rows, row stride, systems)). */
#define PENTAD_MAXDIM 8

typedef enum {
  PENTAD_STATUS_SUCCESS = 0,
  PENTAD_STATUS_NOT_INITIALIZED = 1,
  PENTAD_STATUS_ALLOC_FAILED = 2,
  PENTAD_STATUS_INVALID_VALUE = 3,
  PENTAD_STATUS_ARCH_MISMATCH = 4,
  PENTAD_STATUS_MAPPING_ERROR = 5,
  PENTAD_STATUS_EXECUTION_FAILED = 6,
  PENTAD_STATUS_INTERNAL_ERROR = 7,
  PENTAD_STATUS_MATRIX_TYPE_NOT_SUPPORTED = 8,
  PENTAD_STATUS_ZERO_PIVOT = 9
} pentadStatus_t;

#endif /* PENTAD_COMMON_H__ */
