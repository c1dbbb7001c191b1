/* vl/kmeans.h -- only the opaque k-means handle that the GMM API mentions
 * (vl_gmm_set_kmeans_init_object, vl/gmm.h:122; vl_gmm_get_kmeans_init_object,
 * vl/gmm.h:144).  The GPU drop-in creates and owns the k-means object of the
 * KMeans initialisation itself, with the settings of vl/gmm.c:1336-1356 (ANN
 * refinement over one kd-tree, random-selection seeding, 5 iterations,
 * max(numData/4, 10) comparisons); a handle from another library is refused. */
#ifndef VL_KMEANS_H
#define VL_KMEANS_H
#include "generic.h"
struct _VlKMeans;
typedef struct _VlKMeans VlKMeans;
#endif
