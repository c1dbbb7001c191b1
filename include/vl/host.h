/* vl/host.h -- basic types and export macro of the GPU drop-in for VLFeat's
 * GMM / Fisher-vector C API.
 *
 * Declares the same integer types and export convention as the reference's
 * vl/host.h:314-394 so that a program compiled against either header set
 * links against either library (same sizes, same C linkage).  64-bit only. */
#ifndef VL_HOST_H
#define VL_HOST_H

#include <stddef.h>

#ifdef __cplusplus
#  define VL_EXPORT extern "C" __attribute__((visibility("default")))
#else
#  define VL_EXPORT __attribute__((visibility("default"))) extern
#endif
#define VL_INLINE static __inline__

typedef long long          vl_int64;   /* vl/host.h:376 */
typedef int                vl_int32;
typedef short              vl_int16;
typedef char               vl_int8;
typedef long long unsigned vl_uint64;  /* vl/host.h:381 */
typedef int unsigned       vl_uint32;
typedef short unsigned     vl_uint16;
typedef char unsigned      vl_uint8;
typedef int                vl_int;
typedef unsigned int       vl_uint;
typedef int                vl_bool;    /* vl/host.h:389 */
typedef vl_int64           vl_intptr;
typedef vl_uint64          vl_uintptr;
typedef vl_uint64          vl_size;    /* vl/host.h:392 */
typedef vl_int64           vl_index;
typedef vl_uint64          vl_uindex;

#define VL_TRUE 1
#define VL_FALSE 0

#endif /* VL_HOST_H */
