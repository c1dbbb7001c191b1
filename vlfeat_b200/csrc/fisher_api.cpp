// Fisher-vector encoding entry points: VLFeat's vl_fisher_encode
// (vl/fisher.c:548-579, host pointers) and the device / batched extensions.
#include <cmath>
#include <vector>

#include "engine.h"

extern "C" {
#include "vl/fisher.h"
#include "vlb200.h"
}

using vlb::i64;

namespace {

template <typename F>
auto guarded(F &&f, decltype(f()) sentinel) -> decltype(f()) {
  try {
    return f();
  } catch (const vlb::Error &e) {
    vl_set_last_error(e.code, "%s", e.what());
  } catch (const std::exception &e) {
    vl_set_last_error(VL_ERR_ALLOC, "%s", e.what());
  }
  return sentinel;
}

// Runs the batched encoder on device data with the selected arithmetic.
template <typename T>
void encode_batch(T *enc, const vlb::DevModel<T> &m, const T *X, const i64 *h_offsets,
                  i64 numImages, int flags, int precision, unsigned long long *nterms,
                  cudaStream_t s) {
  if constexpr (sizeof(T) == 4) {
    if (precision != VLB200_PREC_EXACT && vlb::tc_fv_supported_padded(m.K, m.D)) {
      vlb::tc_fisher_batch(X, h_offsets, numImages, m, enc, nterms, flags, precision, s);
      vlb::note_precision(precision);
      return;
    }
  }
  const bool router = sizeof(T) == 4 && precision == VLB200_PREC_BF16_ROUTER;
  vlb::exact_fisher_batch<T>(X, h_offsets, numImages, m, enc, nterms, flags, s, router);
  vlb::note_precision(router ? VLB200_PREC_BF16_ROUTER : VLB200_PREC_EXACT);
}

template <typename T>
vl_size encode_host(T *enc, const T *means, vl_size D, vl_size K, const T *covs, const T *priors,
                    const T *data, vl_size N, int flags, int precision) {
  VLB_CHECK(K >= 1 && D >= 1, VL_ERR_BAD_ARG, "numClusters and dimension must be >= 1");
  cudaStream_t s = vlb::thread_stream();
  vlb::Scratch &sc = vlb::thread_scratch();
  T *dX = sc.slot[25].get<T>(std::max<vl_size>(1, N) * D);
  T *dm = sc.slot[26].get<T>(K * D);
  T *dc = sc.slot[27].get<T>(K * D);
  T *dp = sc.slot[28].get<T>(K);
  T *de = sc.slot[29].get<T>(2 * K * D);
  unsigned long long *dnt = sc.slot[30].get<unsigned long long>(1);
  if (N) VLB_CUDA(cudaMemcpyAsync(dX, data, sizeof(T) * N * D, cudaMemcpyHostToDevice, s));
  VLB_CUDA(cudaMemcpyAsync(dm, means, sizeof(T) * K * D, cudaMemcpyHostToDevice, s));
  VLB_CUDA(cudaMemcpyAsync(dc, covs, sizeof(T) * K * D, cudaMemcpyHostToDevice, s));
  VLB_CUDA(cudaMemcpyAsync(dp, priors, sizeof(T) * K, cudaMemcpyHostToDevice, s));
  vlb::DevModel<T> m;
  m.means = dm; m.covs = dc; m.priors = dp;
  m.K = (i64)K; m.D = (i64)D;
  const i64 off[2] = {0, (i64)N};
  encode_batch<T>(de, m, dX, off, 1, flags, precision, dnt, s);
  unsigned long long nt = 0;
  VLB_CUDA(cudaMemcpyAsync(enc, de, sizeof(T) * 2 * K * D, cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaMemcpyAsync(&nt, dnt, sizeof(nt), cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaStreamSynchronize(s));
  return (vl_size)nt;
}

}  // namespace

extern "C" {

vl_size vl_fisher_encode(void *enc, vl_type dataType, void const *means, vl_size dimension,
                         vl_size numClusters, void const *covariances, void const *priors,
                         void const *data, vl_size numData, int flags) {
  return guarded(
      [&]() -> vl_size {
        if (dataType == VL_TYPE_FLOAT)
          return encode_host<float>((float *)enc, (const float *)means, dimension, numClusters,
                                    (const float *)covariances, (const float *)priors,
                                    (const float *)data, numData, flags,
                                    vlb::resolve_precision(VLB200_PREC_DEFAULT, false));
        VLB_CHECK(dataType == VL_TYPE_DOUBLE, VL_ERR_BAD_ARG,
                  "vl_fisher_encode: data type must be VL_TYPE_FLOAT or VL_TYPE_DOUBLE");
        return encode_host<double>((double *)enc, (const double *)means, dimension, numClusters,
                                   (const double *)covariances, (const double *)priors,
                                   (const double *)data, numData, flags, VLB200_PREC_EXACT);
      },
      (vl_size)0);
}

int vlb200_fisher_encode_device(float *enc, float const *means, vl_size dimension,
                                vl_size numClusters, float const *covariances, float const *priors,
                                float const *data, vl_size numData, int flags, int precision,
                                vl_uint64 *numTerms, void *stream) {
  return guarded(
      [&]() -> int {
        VLB_CHECK(numClusters >= 1 && dimension >= 1, VL_ERR_BAD_ARG,
                  "numClusters and dimension must be >= 1");
        cudaStream_t s = vlb::pick_stream(stream);
        vlb::DevModel<float> m;
        m.means = means; m.covs = covariances; m.priors = priors;
        m.K = (i64)numClusters; m.D = (i64)dimension;
        unsigned long long *dnt = vlb::thread_scratch().slot[30].get<unsigned long long>(1);
        const i64 off[2] = {0, (i64)numData};
        encode_batch<float>(enc, m, data, off, 1, flags, vlb::resolve_precision(precision, false),
                            dnt, s);
        if (numTerms) {
          unsigned long long nt = 0;
          VLB_CUDA(cudaMemcpyAsync(&nt, dnt, sizeof(nt), cudaMemcpyDeviceToHost, s));
          VLB_CUDA(cudaStreamSynchronize(s));
          *numTerms = nt;
        }
        return 0;
      },
      (int)VL_ERR_BAD_ARG);
}

int vlb200_fisher_encode_batch_device(float *enc, float const *means, vl_size dimension,
                                      vl_size numClusters, float const *covariances,
                                      float const *priors, float const *data,
                                      vl_int64 const *offsets, vl_size numImages, int flags,
                                      int precision, vl_uint64 *numTerms, void *stream) {
  return guarded(
      [&]() -> int {
        VLB_CHECK(numClusters >= 1 && dimension >= 1, VL_ERR_BAD_ARG,
                  "numClusters and dimension must be >= 1");
        VLB_CHECK(offsets != nullptr && offsets[0] >= 0, VL_ERR_BAD_ARG, "bad offsets");
        for (vl_size j = 0; j < numImages; ++j)
          VLB_CHECK(offsets[j + 1] >= offsets[j], VL_ERR_BAD_ARG,
                    "offsets must be non-decreasing");
        if (numImages == 0) return 0;
        vlb::DevModel<float> m;
        m.means = means; m.covs = covariances; m.priors = priors;
        m.K = (i64)numClusters; m.D = (i64)dimension;
        encode_batch<float>(enc, m, data, (const i64 *)offsets, (i64)numImages, flags,
                            vlb::resolve_precision(precision, false),
                            (unsigned long long *)numTerms, vlb::pick_stream(stream));
        return 0;
      },
      (int)VL_ERR_BAD_ARG);
}

int vlb200_selftest_bounded_wait(double limit_ms) {
  return guarded(
      [&]() -> int {
        vlb::wait_selftest(limit_ms, vlb::thread_stream());
        return 0;
      },
      (int)VL_ERR_BAD_ARG);
}

}  // extern "C"
