// Fisher encoding of one image without any allocation.
//
// Some callers cannot allocate device memory on the call path: real-time or
// embedded services that forbid allocation after start-up, loops that cannot
// accept the implicit device synchronisation of cudaMalloc / cudaFree, and
// hosts that hand the library a fixed memory budget.  vlb200_fisher_encode_noalloc
// serves them: its scratch (posteriors, per-component constants, partial
// statistics, segment tables) lives in one file-scope device array of fixed
// size, and the call performs no cudaMalloc / cudaFree, no host-to-device
// copy and no allocating library routine.  The arithmetic is the exact
// (CUDA-core, fp32) path, the same kernels as vlb200_fisher_encode_device in
// VLB200_PREC_EXACT mode.
#include <mutex>

#include "engine.h"

extern "C" {
#include "vlb200.h"
}

namespace vlb {
namespace {

// 8 MiB, held by every GPU that loads the library until the process exits.
constexpr size_t kNoAllocBytes = 8u << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr i64 kMaxData = 4096, kMaxClusters = 256, kMaxDim = 128;

// Device address of the array for the current device.  The array's name in
// host code is only a handle; the address comes from cudaGetSymbolAddress,
// asked once per device with that device current.
std::mutex g_mu;
void *g_addr[128] = {};

void *scratch_address() {
  int dev = 0;
  VLB_CUDA(cudaGetDevice(&dev));
  VLB_CHECK(dev >= 0 && dev < 128, VL_ERR_BAD_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) throw_cuda(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
    g_addr[dev] = p;
  }
  return g_addr[dev];
}

size_t up256(size_t b) { return (b + 255) / 256 * 256; }

// Carves the scratch of one call out of the array; returns the bytes used.
size_t carve(char *base, i64 N, i64 K, i64 D, ExactFvScratch &sc) {
  const i64 nseg = exact_fv_segments(N);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char *p = base + off;
    off += up256(bytes);
    return p;
  };
  sc.inv = (float *)take(sizeof(float) * K * D);
  sc.sis = (float *)take(sizeof(float) * K * D);
  sc.cst = (double *)take(sizeof(double) * K);
  sc.q = (float *)take(sizeof(float) * std::max<i64>(1, N) * K);
  sc.llp = (double *)take(sizeof(double) * ((N + 7) / 8 + 1));
  sc.segs = (Segment *)take(sizeof(Segment) * nseg);
  sc.segBegin = (int *)take(sizeof(int) * 2);
  sc.rows = (i64 *)take(sizeof(i64));
  sc.pu = (double *)take(sizeof(double) * nseg * K * D);
  sc.pv = (double *)take(sizeof(double) * nseg * K * D);
  sc.pnt = (unsigned long long *)take(sizeof(unsigned long long) * nseg * K);
  return off;
}

}  // namespace
}  // namespace vlb

extern "C" int vlb200_fisher_encode_noalloc(float *enc, float const *means, vl_size dimension,
                                            vl_size numClusters, float const *covariances,
                                            float const *priors, float const *data,
                                            vl_size numData, int flags, vl_uint64 *numTerms,
                                            void *stream) {
  try {
    using vlb::i64;
    VLB_CHECK(numClusters >= 1 && dimension >= 1, VL_ERR_BAD_ARG,
              "vlb200_fisher_encode_noalloc: numClusters and dimension must be >= 1");
    // Compared as unsigned sizes before any conversion to i64, so that no
    // size of 2^63 or more can wrap to a negative value and pass.
    VLB_CHECK(numData <= (vl_size)vlb::kMaxData && numClusters <= (vl_size)vlb::kMaxClusters &&
                  dimension <= (vl_size)vlb::kMaxDim,
              VL_ERR_BAD_ARG,
              "vlb200_fisher_encode_noalloc: request exceeds the fixed scratch "
              "(numData <= 4096, numClusters <= 256, dimension <= 128)");
    vlb::ExactFvScratch sc;
    char *base = (char *)vlb::scratch_address();
    const size_t used = vlb::carve(base, (i64)numData, (i64)numClusters, (i64)dimension, sc);
    VLB_CHECK(used <= vlb::kNoAllocBytes, VL_ERR_BAD_ARG,
              "vlb200_fisher_encode_noalloc: request exceeds the 8 MiB fixed scratch");
    vlb::DevModel<float> m;
    m.means = means;
    m.covs = covariances;
    m.priors = priors;
    m.K = (i64)numClusters;
    m.D = (i64)dimension;
    vlb::exact_fisher_single_fixed(data, (i64)numData, m, enc, (unsigned long long *)numTerms,
                                   flags, sc, (cudaStream_t)stream);
    return 0;
  } catch (const vlb::Error &e) {
    return vl_set_last_error(e.code, "%s", e.what());
  } catch (const std::exception &e) {
    return vl_set_last_error(VL_ERR_BAD_ARG, "%s", e.what());
  }
}
