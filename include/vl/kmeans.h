/* vl/kmeans.h -- only the opaque k-means handle that the GMM API mentions
 * (vl_gmm_set_kmeans_init_object, vl/gmm.h:123).  The GPU drop-in does not
 * implement k-means; the handle is stored and returned unchanged. */
#ifndef VL_KMEANS_H
#define VL_KMEANS_H
#include "generic.h"
struct _VlKMeans;
typedef struct _VlKMeans VlKMeans;
#endif
