/* vl/vlad.h -- VLAD encoding, GPU drop-in.
 *
 * Same flags and entry point as the reference's vl/vlad.h:23-50.  enc
 * receives numClusters x dimension elements of dataType (component-major),
 * written to caller-owned host memory.  data: numData rows of dimension
 * elements; assignments: numData rows of numClusters weights (hard or soft);
 * only positive weights contribute (vl/vlad.c:182).  The result is bit-equal
 * to the reference's CPU code for the same inputs.  On a CUDA or argument
 * error the function leaves enc unspecified and records the error with
 * vl_set_last_error. */
#ifndef VL_VLAD_H
#define VL_VLAD_H

#include "generic.h"

/* vl/vlad.h:23-26 */
#define VL_VLAD_FLAG_NORMALIZE_COMPONENTS (0x1 << 0)
#define VL_VLAD_FLAG_SQUARE_ROOT          (0x1 << 1)
#define VL_VLAD_FLAG_UNNORMALIZED         (0x1 << 2)
#define VL_VLAD_FLAG_NORMALIZE_MASS       (0x1 << 3)

/* vl/vlad.h:45-50 */
VL_EXPORT void vl_vlad_encode(void *enc, vl_type dataType,
                              void const *means, vl_size dimension, vl_size numClusters,
                              void const *data, vl_size numData,
                              void const *assignments, int flags);

#endif /* VL_VLAD_H */
