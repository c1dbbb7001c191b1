/* vl/gmm.h -- diagonal-covariance Gaussian mixture models, GPU drop-in.
 *
 * Same C API as the reference's vl/gmm.h (VLFeat 0.9.21); each declaration
 * cites the reference declaration it replaces.  Parameters, posteriors and
 * the returned pointers live in host memory exactly as in the reference
 * (getters return borrowed pointers, setters copy in); the E-step, M-step and
 * restarts run on the GPU.  Errors (bad type, CUDA failure, unsupported
 * initialisation) are reported through vl_set_last_error with a NaN
 * log-likelihood instead of the reference's abort(). */
#ifndef VL_GMM_H
#define VL_GMM_H

#include "kmeans.h"

/* vl/gmm.h:21-26 */
typedef enum _VlGMMInitialization {
  VlGMMKMeans,
  VlGMMRand,
  VlGMMCustom
} VlGMMInitialization;

struct _VlGMM;
typedef struct _VlGMM VlGMM;

/* Create and destroy, vl/gmm.h:40-44. */
VL_EXPORT VlGMM *vl_gmm_new(vl_type dataType, vl_size dimension, vl_size numComponents);
VL_EXPORT VlGMM *vl_gmm_new_copy(VlGMM const *gmm);
VL_EXPORT void vl_gmm_delete(VlGMM *self);
VL_EXPORT void vl_gmm_reset(VlGMM *self);

/* Clustering, vl/gmm.h:49-53 (initialisation + EM). */
VL_EXPORT double vl_gmm_cluster(VlGMM *self, void const *data, vl_size numData);

/* Fine-grained processing, vl/gmm.h:59-77. */
VL_EXPORT void vl_gmm_init_with_rand_data(VlGMM *self, void const *data, vl_size numData);
VL_EXPORT void vl_gmm_init_with_kmeans(VlGMM *self, void const *data, vl_size numData,
                                       VlKMeans *kmeansInit);
VL_EXPORT double vl_gmm_em(VlGMM *self, void const *data, vl_size numData);

/* Parameter setters, vl/gmm.h:79-92. */
VL_EXPORT void vl_gmm_set_means(VlGMM *self, void const *means);
VL_EXPORT void vl_gmm_set_covariances(VlGMM *self, void const *covariances);
VL_EXPORT void vl_gmm_set_priors(VlGMM *self, void const *priors);

/* Stand-alone E-step, vl/gmm.h:94-112: posteriors[k + i*K], returns the
 * data log-likelihood sum_i log p(x_i). */
VL_EXPORT double vl_get_gmm_data_posteriors_f(float *posteriors, vl_size numClusters,
                                              vl_size numData, float const *priors,
                                              float const *means, vl_size dimension,
                                              float const *covariances, float const *data);
VL_EXPORT double vl_get_gmm_data_posteriors_d(double *posteriors, vl_size numClusters,
                                              vl_size numData, double const *priors,
                                              double const *means, vl_size dimension,
                                              double const *covariances, double const *data);

/* Option setters, vl/gmm.h:117-124. */
VL_EXPORT void vl_gmm_set_num_repetitions(VlGMM *self, vl_size numRepetitions);
VL_EXPORT void vl_gmm_set_max_num_iterations(VlGMM *self, vl_size maxNumIterations);
VL_EXPORT void vl_gmm_set_verbosity(VlGMM *self, int verbosity);
VL_EXPORT void vl_gmm_set_initialization(VlGMM *self, VlGMMInitialization init);
VL_EXPORT void vl_gmm_set_kmeans_init_object(VlGMM *self, VlKMeans *kmeans);
VL_EXPORT void vl_gmm_set_covariance_lower_bounds(VlGMM *self, double const *bounds);
VL_EXPORT void vl_gmm_set_covariance_lower_bound(VlGMM *self, double bound);

/* Getters, vl/gmm.h:129-145. */
VL_EXPORT void const *vl_gmm_get_means(VlGMM const *self);
VL_EXPORT void const *vl_gmm_get_covariances(VlGMM const *self);
VL_EXPORT void const *vl_gmm_get_priors(VlGMM const *self);
VL_EXPORT void const *vl_gmm_get_posteriors(VlGMM const *self);
VL_EXPORT vl_type vl_gmm_get_data_type(VlGMM const *self);
VL_EXPORT vl_size vl_gmm_get_dimension(VlGMM const *self);
VL_EXPORT vl_size vl_gmm_get_num_repetitions(VlGMM const *self);
VL_EXPORT vl_size vl_gmm_get_num_data(VlGMM const *self);
VL_EXPORT vl_size vl_gmm_get_num_clusters(VlGMM const *self);
VL_EXPORT double vl_gmm_get_loglikelihood(VlGMM const *self);
VL_EXPORT int vl_gmm_get_verbosity(VlGMM const *self);
VL_EXPORT vl_size vl_gmm_get_max_num_iterations(VlGMM const *self);
VL_EXPORT VlGMMInitialization vl_gmm_get_initialization(VlGMM const *self);
VL_EXPORT VlKMeans *vl_gmm_get_kmeans_init_object(VlGMM const *self);
VL_EXPORT double const *vl_gmm_get_covariance_lower_bounds(VlGMM const *self);

#endif /* VL_GMM_H */
