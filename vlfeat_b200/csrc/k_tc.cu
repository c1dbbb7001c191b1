// Tensor-core (tcgen05) path: not built yet; every call routes to the exact kernels.
#include "engine.h"
namespace vlb {
bool tc_supported(i64, i64) { return false; }
void tc_estep(const float *, i64, const DevModel<float> &, float *, double *, bool, int, cudaStream_t) {
  throw Error(VL_ERR_BAD_ARG, "tensor-core E-step not available");
}
void tc_fisher_batch(const float *, const i64 *, i64, const DevModel<float> &, float *,
                     unsigned long long *, int, int, cudaStream_t) {
  throw Error(VL_ERR_BAD_ARG, "tensor-core Fisher encoder not available");
}
}  // namespace vlb
