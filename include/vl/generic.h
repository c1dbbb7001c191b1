/* vl/generic.h -- runtime services of the GPU drop-in library.
 *
 * The subset of the reference's vl/generic.h that programs using the GMM and
 * Fisher-vector API link against: data-type codes, allocation, error state,
 * thread-count state, printf hook and timing.  Signatures and constants match
 * the reference (line numbers cite vl/generic.h of VLFeat 0.9.21). */
#ifndef VL_GENERIC_H
#define VL_GENERIC_H

#include "host.h"
#include "random.h"

/* Data types, vl/generic.h:35-46. */
#define VL_TYPE_FLOAT   1
#define VL_TYPE_DOUBLE  2
#define VL_TYPE_INT8    3
#define VL_TYPE_UINT8   4
#define VL_TYPE_INT16   5
#define VL_TYPE_UINT16  6
#define VL_TYPE_INT32   7
#define VL_TYPE_UINT32  8
#define VL_TYPE_INT64   9
#define VL_TYPE_UINT64  10
typedef vl_uint32 vl_type;

/* Size in bytes of one element of a data type (vl/generic.h:84-98). */
VL_INLINE vl_size vl_get_type_size(vl_type type)
{
  switch (type) {
    case VL_TYPE_DOUBLE: case VL_TYPE_INT64: case VL_TYPE_UINT64: return 8;
    case VL_TYPE_FLOAT: case VL_TYPE_INT32: case VL_TYPE_UINT32: return 4;
    case VL_TYPE_INT16: case VL_TYPE_UINT16: return 2;
    case VL_TYPE_INT8: case VL_TYPE_UINT8: return 1;
    default: return 0;
  }
}

/* Error codes and last-error state, vl/generic.h:122-132.  The GPU library
 * records CUDA and argument failures here instead of aborting. */
#define VL_ERR_OK       0
#define VL_ERR_OVERFLOW 1
#define VL_ERR_ALLOC    2
#define VL_ERR_BAD_ARG  3
#define VL_ERR_IO       4
#define VL_ERR_EOF      5
VL_EXPORT int vl_get_last_error(void);
VL_EXPORT char const *vl_get_last_error_message(void);
VL_EXPORT int vl_set_last_error(int error, char const *errorMessage, ...);

/* Library information and CPU switches, vl/generic.h:102-116.  The SIMD
 * switch and the thread count are recorded for API compatibility; the GPU
 * kernels do not read them. */
VL_EXPORT char const *vl_get_version_string(void);
VL_EXPORT void vl_set_simd_enabled(vl_bool x);
VL_EXPORT vl_bool vl_get_simd_enabled(void);

/* CPU features, read with cpuid as the reference reads them
 * (vl/generic.h:104-108, vl/host.c:446-466).  With SIMD enabled, the kernels
 * that restate a SIMD routine of the reference use the summation order of the
 * variant the reference would pick (AVX, else SSE2, else scalar). */
VL_EXPORT vl_bool vl_cpu_has_avx(void);
VL_EXPORT vl_bool vl_cpu_has_sse3(void);
VL_EXPORT vl_bool vl_cpu_has_sse2(void);

/* The calling thread's random number generator (vl/generic.h:110). */
VL_EXPORT VlRand *vl_get_rand(void);
VL_EXPORT vl_size vl_get_max_threads(void);
VL_EXPORT void vl_set_num_threads(vl_size n);
VL_EXPORT vl_size vl_get_thread_limit(void);

/* Memory, vl/generic.h:143-147. */
VL_EXPORT void *vl_malloc(size_t n);
VL_EXPORT void *vl_realloc(void *ptr, size_t n);
VL_EXPORT void *vl_calloc(size_t n, size_t size);
VL_EXPORT void *vl_memalign(size_t n, size_t size);
VL_EXPORT void vl_free(void *ptr);

/* printf hook, vl/generic.h:154-168. */
typedef int (*printf_func_t)(char const *format, ...);
VL_EXPORT void vl_set_printf_func(printf_func_t printf_func);
VL_EXPORT printf_func_t vl_get_printf_func(void);
#define VL_PRINTF (*vl_get_printf_func())
#define VL_PRINT (*vl_get_printf_func())

/* Timing, vl/generic.h:204-206. */
VL_EXPORT void vl_tic(void);
VL_EXPORT double vl_toc(void);
VL_EXPORT double vl_get_cpu_time(void);

#define VL_MIN(x, y) (((x) < (y)) ? (x) : (y))
#define VL_MAX(x, y) (((x) > (y)) ? (x) : (y))

#endif /* VL_GENERIC_H */
