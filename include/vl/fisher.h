/* vl/fisher.h -- Fisher-vector encoding, GPU drop-in.
 *
 * Same flags and entry point as the reference's vl/fisher.h:23-54.  The
 * encoding [u_1..u_K | v_1..v_K] (2*D*K elements of dataType) is written to
 * caller-owned host memory; the return value is the number of (descriptor,
 * component) terms with posterior >= 1e-6 (vl/fisher.c:440-441).  On a CUDA or
 * argument error the function returns 0 and records the error with
 * vl_set_last_error. */
#ifndef VL_FISHER_H
#define VL_FISHER_H

#include "generic.h"

#define VL_FISHER_FLAG_SQUARE_ROOT (0x1 << 0)
#define VL_FISHER_FLAG_NORMALIZED  (0x1 << 1)
#define VL_FISHER_FLAG_IMPROVED    (VL_FISHER_FLAG_NORMALIZED | VL_FISHER_FLAG_SQUARE_ROOT)
#define VL_FISHER_FLAG_FAST        (0x1 << 2)

/* vl/fisher.h:48-54 */
VL_EXPORT vl_size vl_fisher_encode(void *enc, vl_type dataType,
                                   void const *means, vl_size dimension, vl_size numClusters,
                                   void const *covariances, void const *priors,
                                   void const *data, vl_size numData, int flags);

#endif /* VL_FISHER_H */
