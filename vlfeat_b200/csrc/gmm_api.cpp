// VLFeat's GMM object and EM driver (vl/gmm.h) on the GPU.
//
// The object keeps VLFeat's host-memory contract: means / covariances /
// priors / posteriors are host arrays owned by the object, getters return
// borrowed pointers (vl/gmm.c:430-675), setters copy in.  EM runs on the GPU:
// the data is staged to device memory once per call, parameters live on the
// device during the loop and are copied back at the end; posteriors are
// copied back lazily on the first vl_gmm_get_posteriors() call.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "engine.h"

extern "C" {
#include "vl/gmm.h"
#include "vlb200.h"
}

using vlb::i64;

// The k-means object of the KMeans initialisation.  The library creates one
// the first time a GMM needs it, with the reference's settings
// (vl/gmm.c:1336-1356), and owns it; objects from elsewhere are refused.
struct _VlKMeans {
  static constexpr uint32_t kMagic = 0x4b4d6231u;
  uint32_t magic = kMagic;
  vlb::KMeansSettings cfg;
};

struct _VlGMM {
  vl_type dataType = VL_TYPE_FLOAT;
  vl_size dimension = 0, numClusters = 0, numData = 0;
  vl_size maxNumIterations = 50, numRepetitions = 1;  // defaults, vl/gmm.c:365-380
  int verbosity = 0;
  void *means = nullptr, *covariances = nullptr, *priors = nullptr;
  void *posteriors = nullptr;
  vl_size posteriorsCap = 0;  // rows the host posterior buffer can hold
  double *sigmaLowBound = nullptr;
  VlGMMInitialization initialization = VlGMMRand;
  VlKMeans *kmeansInit = nullptr;
  bool kmeansInitIsOwner = false;
  double LL = 0;
  // GPU state.
  bool postOnDevice = false;  // the device buffer holds the current posteriors
  vlb::DevBuf dX, dq, dmeans, dcovs, dpriors, dlb, dtmp, dassign;
  std::vector<double> llTrace;
  vl_size numRestarts = 0;
  // Parameter snapshots of the last EM run (vlb200_gmm_set_param_trace):
  // entry t holds means, covariances and priors after t M-steps, in double.
  bool traceParams = false;
  std::vector<std::vector<double>> paramTrace;
  // Streamed EM (vlb200_gmm_em_stream_device): one report row per E-step, and
  // what the posteriors are recomputed from when they are asked for (they are
  // never resident: N x K can exceed the device's memory).
  std::vector<std::array<double, 6>> streamReport;
  bool postLazy = false;
  const void *lazyX = nullptr;
  int lazyPrec = 0;
  VlB200Router *lazyRouter = nullptr;
  vl_size lazyM = 8;
  float lazyThr = 0.99f;
  vl_size lazyChunk = 0;
  vlb::DevBuf dpart, dpm, dp1, dp2, dqr, dpe;
};

namespace vlb {
double router_estep(VlB200Router *r, const float *X, i64 n, const DevModel<float> &m, float *q,
                    size_t mcand, float thr, unsigned long long *fallback, cudaStream_t s);
double router_missed_sum(const float *qfull, const float *qc, i64 n, i64 K, cudaStream_t s);
void router_fit(VlB200Router *r, const float *X, i64 n, const float *q, int epochs, float lr, cudaStream_t s);
}  // namespace vlb

namespace {

size_t tsize(vl_type t) { return t == VL_TYPE_DOUBLE ? 8 : 4; }

void check_type(vl_type t) {
  VLB_CHECK(t == VL_TYPE_FLOAT || t == VL_TYPE_DOUBLE, VL_ERR_BAD_ARG,
            "data type must be VL_TYPE_FLOAT or VL_TYPE_DOUBLE");
}

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

template <typename T>
double device_estep(const T *dX, i64 N, const vlb::DevModel<T> &m, T *dq, int precision,
                    bool fast, cudaStream_t s, bool em_image = false);

// Posteriors of a streamed EM, recomputed chunk by chunk from the data and
// the final parameters with the final E-step's arithmetic (the loop ends
// after an E-step, so they are that E-step's posteriors, vl/gmm.c:1220-1308).
template <typename T>
void lazy_posteriors(VlGMM *self) {
  cudaStream_t s = vlb::thread_stream();
  const i64 K = (i64)self->numClusters, D = (i64)self->dimension, N = (i64)self->numData;
  const i64 chunk = std::max<i64>(1, (i64)self->lazyChunk);
  vlb::DevModel<T> m;
  m.means = self->dmeans.get<T>(K * D);
  m.covs = self->dcovs.get<T>(K * D);
  m.priors = self->dpriors.get<T>(K);
  m.K = K;
  m.D = D;
  T *dq = self->dq.get<T>((size_t)std::min(chunk, N) * K);
  const T *X = (const T *)self->lazyX;
  for (i64 r0 = 0; r0 < N; r0 += chunk) {
    const i64 n = std::min(chunk, N - r0);
    bool done = false;
    if constexpr (sizeof(T) == 4) {
      if (self->lazyRouter) {
        vlb::router_estep(self->lazyRouter, X + r0 * D, n, m, dq, self->lazyM, self->lazyThr, nullptr, s);
        done = true;
      }
    }
    if (!done) device_estep<T>(X + r0 * D, n, m, dq, self->lazyPrec, false, s, false);
    VLB_CUDA(cudaMemcpyAsync((T *)self->posteriors + r0 * K, dq, sizeof(T) * n * K, cudaMemcpyDeviceToHost, s));
    VLB_CUDA(cudaStreamSynchronize(s));
  }
}

// Host copy of the posteriors, refreshed from the device when stale.
void sync_posteriors(VlGMM *self) {
  if (self->postLazy) {
    const size_t bytes = tsize(self->dataType) * self->numData * self->numClusters;
    if (self->posteriorsCap < self->numData || !self->posteriors) {
      vl_free(self->posteriors);
      self->posteriors = vl_malloc(bytes ? bytes : 1);
      VLB_CHECK(self->posteriors != nullptr, VL_ERR_ALLOC, "vl_gmm_get_posteriors: host allocation failed");
      self->posteriorsCap = self->numData;
    }
    if (self->dataType == VL_TYPE_FLOAT) lazy_posteriors<float>(self);
    else lazy_posteriors<double>(self);
    self->postLazy = false;
    return;
  }
  if (!self->postOnDevice) return;
  const size_t bytes = tsize(self->dataType) * self->numData * self->numClusters;
  if (self->posteriorsCap < self->numData || !self->posteriors) {
    vl_free(self->posteriors);
    self->posteriors = vl_malloc(bytes ? bytes : 1);
    self->posteriorsCap = self->numData;
  }
  cudaStream_t s = vlb::thread_stream();
  if (bytes) VLB_CUDA(cudaMemcpyAsync(self->posteriors, self->dq.p, bytes, cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaStreamSynchronize(s));
  self->postOnDevice = false;
}

// em_image: also write the posteriors as the tensor-core M-step's operand
// image (EM with the tensor-core path; see vlb::tc_estep_em).
template <typename T>
double device_estep(const T *dX, i64 N, const vlb::DevModel<T> &m, T *dq, int precision,
                    bool fast, cudaStream_t s, bool em_image) {
  vlb::Scratch &sc = vlb::thread_scratch();
  double *llp = sc.slot[15].get<double>(vlb::estep_ll_parts(N));
  double *dll = sc.slot[16].get<double>(1);
  bool done = false;
  i64 nparts = 0;
  if constexpr (sizeof(T) == 4) {
    // The EM image format needs a dimension the kernels are built for; the
    // posteriors alone also run zero-padded (vlb::tc_supported_padded).
    if (precision != VLB200_PREC_EXACT &&
        (em_image ? vlb::tc_supported(m.K, m.D) : vlb::tc_supported_padded(m.K, m.D))) {
      nparts = em_image ? vlb::tc_estep_em(dX, N, m, dq, llp, precision, s)
                        : vlb::tc_estep(dX, N, m, dq, llp, fast, precision, s);
      done = true;
      vlb::note_precision(precision);
    }
  }
  if (!done) {
    vlb::DevDerived<T> der;
    der.inv = sc.slot[17].get<T>(m.K * m.D);
    der.sis = sc.slot[18].get<T>(m.K * m.D);
    der.cst = sc.slot[19].get<double>(m.K);
    vlb::exact_prepare(m, der, s);
    nparts = vlb::exact_estep(dX, N, m, der, dq, llp, fast, s);
    vlb::note_precision(VLB200_PREC_EXACT);
  }
  if (N <= 0) return 0.0;
  vlb::sum_doubles(llp, nparts, dll, s);
  double ll = 0;
  VLB_CUDA(cudaMemcpyAsync(&ll, dll, sizeof(double), cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaStreamSynchronize(s));
  return ll;
}

// Empty-mode restarts, vl/gmm.c:814-999, with the posteriors and parameters
// on the device and the (cheap) selection logic on the host.
template <typename T>
vl_size restart_empty_modes(VlGMM *self, const T *dX, i64 N, T *dq, T *dmeans, T *dcovs,
                            T *dpriors, const double *dlb, cudaStream_t s) {
  const i64 K = (i64)self->numClusters, D = (i64)self->dimension;
  if (K <= 1) return 0;
  double *dmass = self->dtmp.get<double>(K);
  vlb::column_mass(dq, N, K, dmass, s);
  std::vector<double> mass(K);
  VLB_CUDA(cudaMemcpyAsync(mass.data(), dmass, sizeof(double) * K, cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaStreamSynchronize(s));
  const double cutoff = 1e-2 * std::max(1.0, (double)N / (double)K);
  vl_size nsplit = 0;
  std::vector<T> pr(K), cv(K * D), mu(K * D);
  bool have = false;
  for (i64 icl = 0; icl < K; ++icl) {
    if (mass[icl] >= cutoff) continue;
    if (self->verbosity) VLB_PRINTF("gmm: mode %d is nearly empty (mass %f)\n", (int)icl, mass[icl]);
    if (!have) {
      VLB_CUDA(cudaMemcpyAsync(pr.data(), dpriors, sizeof(T) * K, cudaMemcpyDeviceToHost, s));
      VLB_CUDA(cudaMemcpyAsync(cv.data(), dcovs, sizeof(T) * K * D, cudaMemcpyDeviceToHost, s));
      VLB_CUDA(cudaMemcpyAsync(mu.data(), dmeans, sizeof(T) * K * D, cudaMemcpyDeviceToHost, s));
      VLB_CUDA(cudaStreamSynchronize(s));
      have = true;
    }
    // Mode with the largest entropy contribution, vl/gmm.c:920-939.
    double bestScore = -INFINITY;
    i64 best = -1;
    for (i64 j = 0; j < K; ++j) {
      if ((double)pr[j] < 1e-6) continue;
      double sc = 0.5 * (double)D * (1.0 + log(2 * 3.141592653589793));
      for (i64 d = 0; d < D; ++d) sc += 0.5 * log((double)cv[j * D + d]);
      sc = (double)pr[j] * (sc - log((double)pr[j]));
      if (sc > bestScore) {
        bestScore = sc;
        best = j;
      }
    }
    if (best == icl || best < 0) {
      if (self->verbosity)
        VLB_PRINTF("gmm: mode %d is empty, but no other mode to split could be found\n", (int)icl);
      continue;
    }
    if (self->verbosity)
      VLB_PRINTF("gmm: reinitializing empty mode %d with mode %d (prior %f, mass %f, score %f)\n",
                 (int)icl, (int)best, (double)pr[best], mass[best], bestScore);
    // Largest-variance dimension, vl/gmm.c:958-966.
    double bv = -INFINITY;
    i64 bd = -1;
    for (i64 d = 0; d < D; ++d)
      if ((double)cv[best * D + d] > bv) {
        bv = (double)cv[best * D + d];
        bd = d;
      }
    if (bd < 0) continue;  // every variance NaN: no dimension to split along
    vlb::restart_split<T>(dq, dX, N, K, D, icl, best, bd, mu[best * D + bd], s);
    vlb::exact_mstep<T>(dX, N, dq, dmeans, dcovs, dpriors, K, D, dlb, s);
    VLB_CUDA(cudaMemcpyAsync(pr.data(), dpriors, sizeof(T) * K, cudaMemcpyDeviceToHost, s));
    VLB_CUDA(cudaMemcpyAsync(cv.data(), dcovs, sizeof(T) * K * D, cudaMemcpyDeviceToHost, s));
    VLB_CUDA(cudaMemcpyAsync(mu.data(), dmeans, sizeof(T) * K * D, cudaMemcpyDeviceToHost, s));
    VLB_CUDA(cudaStreamSynchronize(s));
    ++nsplit;
  }
  return nsplit;
}

struct StreamCfg;
template <typename T>
double em_stream_device(VlGMM *self, const T *dX, i64 N, int precision, const StreamCfg &cfg);
template <typename T>
double em_stream_default(VlGMM *self, const T *dX, i64 N, int precision);

// The EM loop, vl/gmm.c:1220-1308, on device-resident data dX (N x D).  When
// the N x K posteriors (and the tensor-core M-step's operand image) would not
// fit in free device memory, the streamed loop runs instead.
template <typename T>
double em_device(VlGMM *self, const T *dX, i64 N, int precision) {
  cudaStream_t s = vlb::thread_stream();
  const i64 K = (i64)self->numClusters, D = (i64)self->dimension;
  {
    size_t freeB = 0, totalB = 0;
    VLB_CUDA(cudaMemGetInfo(&freeB, &totalB));
    const double need = (double)N * (double)K * (sizeof(T) + 4.0);
    if (need > 0.8 * (double)(freeB + self->dq.cap)) return em_stream_default<T>(self, dX, N, precision);
  }
  T *dmeans = self->dmeans.get<T>(K * D);
  T *dcovs = self->dcovs.get<T>(K * D);
  T *dpriors = self->dpriors.get<T>(K);
  double *dlb = self->dlb.get<double>(D);
  T *dq = self->dq.get<T>(std::max<i64>(1, N) * K);
  VLB_CUDA(cudaMemcpyAsync(dmeans, self->means, sizeof(T) * K * D, cudaMemcpyHostToDevice, s));
  VLB_CUDA(cudaMemcpyAsync(dcovs, self->covariances, sizeof(T) * K * D, cudaMemcpyHostToDevice, s));
  VLB_CUDA(cudaMemcpyAsync(dpriors, self->priors, sizeof(T) * K, cudaMemcpyHostToDevice, s));
  VLB_CUDA(cudaMemcpyAsync(dlb, self->sigmaLowBound, sizeof(double) * D, cudaMemcpyHostToDevice, s));
  self->numData = (vl_size)N;  // _vl_gmm_prepare_for_data, vl/gmm.c:336-344
  self->llTrace.clear();
  self->paramTrace.clear();
  self->numRestarts = 0;

  vlb::DevModel<T> m;
  m.means = dmeans;
  m.covs = dcovs;
  m.priors = dpriors;
  m.K = K;
  m.D = D;

  vlb::apply_bounds<T>(dcovs, K, D, dlb, s);  // vl/gmm.c:1233
  // Tensor-core modes run the M-step's statistics on the tensor cores from
  // the E-step's posterior image; EXACT and double stay on the CUDA cores.
  bool tcm = false;
  if constexpr (sizeof(T) == 4) tcm = precision != VLB200_PREC_EXACT && vlb::tc_supported(K, D);
  double prevLL = -INFINITY, LL = -INFINITY;
  std::vector<T> snap;
  for (vl_size it = 0;; ++it) {
    if (self->traceParams) {
      // The parameters this iteration's E-step uses: after `it` M-steps.
      snap.resize((size_t)(2 * K * D + K));
      VLB_CUDA(cudaMemcpyAsync(snap.data(), dmeans, sizeof(T) * K * D, cudaMemcpyDeviceToHost, s));
      VLB_CUDA(cudaMemcpyAsync(snap.data() + K * D, dcovs, sizeof(T) * K * D, cudaMemcpyDeviceToHost, s));
      VLB_CUDA(cudaMemcpyAsync(snap.data() + 2 * K * D, dpriors, sizeof(T) * K, cudaMemcpyDeviceToHost, s));
      VLB_CUDA(cudaStreamSynchronize(s));
      self->paramTrace.emplace_back(snap.begin(), snap.end());
    }
    LL = device_estep<T>(dX, N, m, dq, precision, false, s, tcm);
    self->llTrace.push_back(LL);
    if (self->verbosity)
      VLB_PRINTF("gmm: em: iteration %d: loglikelihood = %f (variation = %f)\n", (int)it, LL,
                 LL - prevLL);
    if (it >= self->maxNumIterations) {
      if (self->verbosity)
        VLB_PRINTF("gmm: em: terminating because the maximum number of iterations (%d) has been reached.\n",
                   (int)self->maxNumIterations);
      break;
    }
    const double eps = fabs((LL - prevLL) / LL);
    if (it > 0 && eps < 0.00001) {
      if (self->verbosity)
        VLB_PRINTF("gmm: em: terminating because the algorithm fully converged (log-likelihood variation = %f).\n",
                   eps);
      break;
    }
    prevLL = LL;
    vl_size r = 0;
    if (it > 1) {
      r = restart_empty_modes<T>(self, dX, N, dq, dmeans, dcovs, dpriors, dlb, s);
      self->numRestarts += r;
      if (r > 0 && self->verbosity)
        VLB_PRINTF("gmm: em: %d Gaussian modes restarted because they had become empty.\n", (int)r);
    }
    // A restart rewrites posteriors (vl/gmm.c:969-989), so the image is stale:
    // that iteration's M-step reads the rows.
    bool done = false;
    if constexpr (sizeof(T) == 4) {
      if (tcm && r == 0) {
        vlb::tc_mstep(dX, N, dmeans, dcovs, dpriors, K, D, dlb, precision, s);
        done = true;
      }
    }
    if (!done) vlb::exact_mstep<T>(dX, N, dq, dmeans, dcovs, dpriors, K, D, dlb, s);
  }
  VLB_CUDA(cudaMemcpyAsync(self->means, dmeans, sizeof(T) * K * D, cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaMemcpyAsync(self->covariances, dcovs, sizeof(T) * K * D, cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaMemcpyAsync(self->priors, dpriors, sizeof(T) * K, cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaStreamSynchronize(s));
  self->postOnDevice = true;
  self->postLazy = false;
  return LL;
}

// ------------------------------------------------------------ streamed EM
// The EM loop of vl/gmm.c:1220-1308 over data whose N x K posteriors do not
// stay on the device: each pass runs the E-step chunk by chunk (rows
// [r0, r0 + n)), and while a chunk's posteriors exist it adds their column
// masses (for the restart check, vl/gmm.c:814-999), the chunk's log-
// likelihood and its M-step statistics (vl/gmm.c:1036-1213: tensor-core item
// partials, or the exact path's slab partials) to the pass's totals; the
// M-step is finalised from all of them in f64 once the loop's checks allow it.
// With a router, the E-steps of iterations that are not multiples of
// `judgeEvery` evaluate the exact posteriors of each row's router candidates
// only (full E-step on rows whose predicted candidate mass is below thr);
// every judgeEvery-th iteration runs the full E-step, re-fits the router on
// the first rows' posteriors, and measures the router's missed posterior
// mass on the other rows against it.  Restarts re-derive the iteration's
// posteriors chunk by chunk (the same E-step on the same parameters, then
// the splits so far in order) for each M-step they need, as the reference
// re-runs its M-step on the modified posteriors.
struct StreamCfg {
  i64 chunk = 0;
  VlB200Router *router = nullptr;
  vl_size m = 8;
  float thr = 0.99f;
  vl_size judgeEvery = 5;
  i64 fitRows = 1 << 20;
  // Sharded EM: this rank's rows are part of totalN; every sum over rows
  // (log-likelihood, restart masses, M-step sums) is completed across ranks
  // by allreduce before it is used.
  vlb200_allreduce_fn allreduce = nullptr;
  void *arctx = nullptr;
  i64 totalN = 0;
};

template <typename T>
double em_stream_device(VlGMM *self, const T *dX, i64 N, int precision, const StreamCfg &cfg) {
  using clk = std::chrono::steady_clock;
  cudaStream_t s = vlb::thread_stream();
  const i64 K = (i64)self->numClusters, D = (i64)self->dimension;
  VLB_CHECK(N >= 1, VL_ERR_BAD_ARG, "streamed EM: no data");
  T *dmeans = self->dmeans.get<T>(K * D);
  T *dcovs = self->dcovs.get<T>(K * D);
  T *dpriors = self->dpriors.get<T>(K);
  double *dlb = self->dlb.get<double>(D);
  VLB_CUDA(cudaMemcpyAsync(dmeans, self->means, sizeof(T) * K * D, cudaMemcpyHostToDevice, s));
  VLB_CUDA(cudaMemcpyAsync(dcovs, self->covariances, sizeof(T) * K * D, cudaMemcpyHostToDevice, s));
  VLB_CUDA(cudaMemcpyAsync(dpriors, self->priors, sizeof(T) * K, cudaMemcpyHostToDevice, s));
  VLB_CUDA(cudaMemcpyAsync(dlb, self->sigmaLowBound, sizeof(double) * D, cudaMemcpyHostToDevice, s));
  self->numData = (vl_size)N;
  self->llTrace.clear();
  self->paramTrace.clear();
  self->streamReport.clear();
  self->numRestarts = 0;
  self->postOnDevice = false;
  self->postLazy = false;

  vlb::DevModel<T> m;
  m.means = dmeans; m.covs = dcovs; m.priors = dpriors; m.K = K; m.D = D;
  vlb::apply_bounds<T>(dcovs, K, D, dlb, s);  // vl/gmm.c:1233

  bool tcm = false;
  if constexpr (sizeof(T) == 4) tcm = precision != VLB200_PREC_EXACT && vlb::tc_supported(K, D);
  VlB200Router *router = nullptr;
  if constexpr (sizeof(T) == 4) router = cfg.router;
  const vl_size judgeEvery = std::max<vl_size>(1, cfg.judgeEvery);
  const bool sharded = cfg.allreduce != nullptr;
  VLB_CHECK(!sharded || (!router && cfg.totalN >= N), VL_ERR_BAD_ARG,
            "sharded EM: no router, and totalData at least this rank's rows");
  const i64 Ntot = sharded ? cfg.totalN : N;
  std::vector<double> hsum;
  // Completes the exact M-step's slab partials across ranks (summed into slab
  // 0 first) and finalises from them; unsharded, the finalize over all slabs.
  auto exact_finalize = [&](int nsl, double *qm, double *q1, double *q2) {
    if (!sharded) {
      vlb::exact_mstep_finalize_slabs<T>(nsl, qm, q1, q2, dlb, dmeans, dcovs, dpriors, K, D, s);
      return;
    }
    vlb::exact_sum_slabs(nsl, qm, q1, q2, K, D, s);
    hsum.resize((size_t)(2 * D + 1) * K);
    VLB_CUDA(cudaMemcpyAsync(hsum.data(), qm, sizeof(double) * K, cudaMemcpyDeviceToHost, s));
    VLB_CUDA(cudaMemcpyAsync(hsum.data() + K, q1, sizeof(double) * K * D, cudaMemcpyDeviceToHost, s));
    VLB_CUDA(cudaMemcpyAsync(hsum.data() + K + K * D, q2, sizeof(double) * K * D, cudaMemcpyDeviceToHost, s));
    VLB_CUDA(cudaStreamSynchronize(s));
    cfg.allreduce(hsum.data(), (vl_size)hsum.size(), cfg.arctx);
    VLB_CUDA(cudaMemcpyAsync(qm, hsum.data(), sizeof(double) * K, cudaMemcpyHostToDevice, s));
    VLB_CUDA(cudaMemcpyAsync(q1, hsum.data() + K, sizeof(double) * K * D, cudaMemcpyHostToDevice, s));
    VLB_CUDA(cudaMemcpyAsync(q2, hsum.data() + K + K * D, sizeof(double) * K * D, cudaMemcpyHostToDevice, s));
    vlb::exact_mstep_finalize_slabs<T>(1, qm, q1, q2, dlb, dmeans, dcovs, dpriors, K, D, s);
  };
  // Chunks start on the exact M-step's slab boundaries (its partition of all
  // N rows), so restarts can use the exact M-step chunk by chunk.
  const i64 rps = vlb::exact_mstep_slab_rows(N);
  const int nslab = (int)((N + rps - 1) / rps);
  i64 want = cfg.chunk > 0 ? cfg.chunk : std::max<i64>(rps, (i64)((1ll << 33) / (K * (i64)sizeof(T))));
  const i64 chunk = std::min<i64>(N + rps - 1, (want + rps - 1) / rps * rps) / rps * rps;
  T *dq = self->dq.get<T>((size_t)chunk * K);
  T *dqr = router ? self->dqr.get<T>((size_t)chunk * K) : nullptr;
  double *dmass = self->dtmp.get<double>(K);
  i64 nitems = 0;
  for (i64 r0 = 0; r0 < N; r0 += chunk) nitems += vlb::tc_em_items(std::min(chunk, N - r0));
  float *dpart = tcm ? self->dpart.get<float>((size_t)nitems * vlb::tc_em_partial_floats(K, D)) : nullptr;
  double *pm = self->dpm.get<double>((size_t)nslab * K);
  double *p1 = self->dp1.get<double>((size_t)nslab * K * D);
  double *p2 = self->dp2.get<double>((size_t)nslab * K * D);
  // The parameters an iteration's E-step used (restarts re-derive from them).
  T *pe = self->dpe.get<T>((size_t)(2 * K * D + K));

  // E-step of one chunk into q (row-major): full (tensor-core image for the
  // M-step when tcm) or through the router.  Returns the chunk's LL.
  auto chunk_estep = [&](const vlb::DevModel<T> &mm, i64 r0, i64 n, bool viaRouter, T *q,
                         unsigned long long *fb) -> double {
    if constexpr (sizeof(T) == 4) {
      if (viaRouter) {
        const double ll = vlb::router_estep(router, dX + r0 * D, n, mm, q, cfg.m, cfg.thr, fb, s);
        if (tcm) vlb::tc_em_image_from_rows(q, n, mm, s);
        return ll;
      }
    }
    return device_estep<T>(dX + r0 * D, n, mm, q, precision, false, s, tcm);
  };

  double prevLL = -INFINITY, LL = -INFINITY;
  std::vector<T> snap;
  for (vl_size it = 0;; ++it) {
    const auto t0 = clk::now();
    const bool judged = router && it % judgeEvery == 0;
    const bool viaRouter = router && !judged;
    if (self->traceParams) {
      snap.resize((size_t)(2 * K * D + K));
      VLB_CUDA(cudaMemcpyAsync(snap.data(), dmeans, sizeof(T) * K * D, cudaMemcpyDeviceToHost, s));
      VLB_CUDA(cudaMemcpyAsync(snap.data() + K * D, dcovs, sizeof(T) * K * D, cudaMemcpyDeviceToHost, s));
      VLB_CUDA(cudaMemcpyAsync(snap.data() + 2 * K * D, dpriors, sizeof(T) * K, cudaMemcpyDeviceToHost, s));
      VLB_CUDA(cudaStreamSynchronize(s));
      self->paramTrace.emplace_back(snap.begin(), snap.end());
    }
    std::vector<double> mass(K, 0.0), mchunk(K);
    double missed = 0, missedRows = 0;
    unsigned long long fb = 0, fbJudge = 0;
    LL = 0;
    int item0 = 0;
    for (i64 r0 = 0; r0 < N; r0 += chunk) {
      const i64 n = std::min(chunk, N - r0);
      LL += chunk_estep(m, r0, n, viaRouter, dq, &fb);
      if constexpr (sizeof(T) == 4) {
        if (judged) {
          // Re-fit the router on this pass's first rows, then judge it on the rest.
          const i64 skip = r0 == 0 ? std::min<i64>(n, cfg.fitRows) : 0;
          if (r0 == 0) vlb::router_fit(router, dX, skip, dq, it == 0 ? 4 : 1, 2e-3f, s);
          if (n > skip) {
            vlb::router_estep(router, dX + (r0 + skip) * D, n - skip, m, dqr, cfg.m, cfg.thr, &fbJudge, s);
            missed += vlb::router_missed_sum(dq + skip * K, dqr, n - skip, K, s);
            missedRows += (double)(n - skip);
          }
        }
      }
      if (it > 1) {
        vlb::column_mass<T>(dq, n, K, dmass, s);
        VLB_CUDA(cudaMemcpyAsync(mchunk.data(), dmass, sizeof(double) * K, cudaMemcpyDeviceToHost, s));
        VLB_CUDA(cudaStreamSynchronize(s));
        for (i64 k = 0; k < K; ++k) mass[k] += mchunk[k];
      }
      bool tcStats = false;
      if constexpr (sizeof(T) == 4) {
        if (tcm) {
          const int split = (!viaRouter && precision == VLB200_PREC_FP32) ? 2 : 1;
          vlb::tc_em_stats((const float *)dX, r0, n, K, D, split, dpart, item0, s);
          item0 += (int)vlb::tc_em_items(n);
          tcStats = true;
        }
      }
      if (!tcStats) vlb::exact_mstep_stats_rows<T>(dX, r0, n, rps, dq, dmeans, K, D, pm, p1, p2, s);
    }
    if (sharded) {
      // This pass's log-likelihood and (for the restart check) masses, over all ranks.
      hsum.assign(1 + (it > 1 ? K : 0), 0.0);
      hsum[0] = LL;
      for (i64 k = 0; k < (it > 1 ? K : 0); ++k) hsum[1 + k] = mass[k];
      cfg.allreduce(hsum.data(), (vl_size)hsum.size(), cfg.arctx);
      LL = hsum[0];
      for (i64 k = 0; k < (it > 1 ? K : 0); ++k) mass[k] = hsum[1 + k];
    }
    self->llTrace.push_back(LL);
    const double ms = std::chrono::duration<double, std::milli>(clk::now() - t0).count();
    self->streamReport.push_back({LL, judged ? 1.0 : 0.0, viaRouter ? 1.0 : 0.0,
                                  missedRows > 0 ? missed / missedRows : (judged ? 0.0 : NAN),
                                  (double)(viaRouter ? fb : fbJudge), ms});
    if (self->verbosity)
      VLB_PRINTF("gmm: em: iteration %d: loglikelihood = %f (variation = %f)\n", (int)it, LL, LL - prevLL);
    if (it >= self->maxNumIterations) break;
    const double eps = fabs((LL - prevLL) / LL);
    if (it > 0 && eps < 0.00001) break;
    prevLL = LL;

    // Restarts (vl/gmm.c:1292, 814-999) with the masses of this pass.
    vl_size nsplit = 0;
    if (it > 1 && K > 1) {
      const double cutoff = 1e-2 * std::max(1.0, (double)Ntot / (double)K);
      std::vector<std::array<double, 4>> splits;  // (empty mode, split mode, dimension, cut)
      std::vector<T> pr(K), cv(K * D), mu(K * D);
      bool saved = false;
      auto rederive_mstep = [&]() {
        vlb::DevModel<T> me;
        me.means = pe; me.covs = pe + K * D; me.priors = pe + 2 * K * D; me.K = K; me.D = D;
        for (i64 r0 = 0; r0 < N; r0 += chunk) {
          const i64 n = std::min(chunk, N - r0);
          chunk_estep(me, r0, n, viaRouter, dq, nullptr);
          for (auto &sp : splits)
            vlb::restart_split<T>(dq, dX + r0 * D, n, K, D, (i64)sp[0], (i64)sp[1], (i64)sp[2], (T)sp[3], s);
          vlb::exact_mstep_stats_rows<T>(dX, r0, n, rps, dq, dmeans, K, D, pm, p1, p2, s);
        }
        exact_finalize(nslab, pm, p1, p2);
        VLB_CUDA(cudaMemcpyAsync(pr.data(), dpriors, sizeof(T) * K, cudaMemcpyDeviceToHost, s));
        VLB_CUDA(cudaMemcpyAsync(cv.data(), dcovs, sizeof(T) * K * D, cudaMemcpyDeviceToHost, s));
        VLB_CUDA(cudaMemcpyAsync(mu.data(), dmeans, sizeof(T) * K * D, cudaMemcpyDeviceToHost, s));
        VLB_CUDA(cudaStreamSynchronize(s));
      };
      for (i64 icl = 0; icl < K; ++icl) {
        if (mass[icl] >= cutoff) continue;
        if (self->verbosity) VLB_PRINTF("gmm: mode %d is nearly empty (mass %f)\n", (int)icl, mass[icl]);
        if (!saved) {
          VLB_CUDA(cudaMemcpyAsync(pe, dmeans, sizeof(T) * K * D, cudaMemcpyDeviceToDevice, s));
          VLB_CUDA(cudaMemcpyAsync(pe + K * D, dcovs, sizeof(T) * K * D, cudaMemcpyDeviceToDevice, s));
          VLB_CUDA(cudaMemcpyAsync(pe + 2 * K * D, dpriors, sizeof(T) * K, cudaMemcpyDeviceToDevice, s));
          VLB_CUDA(cudaMemcpyAsync(pr.data(), dpriors, sizeof(T) * K, cudaMemcpyDeviceToHost, s));
          VLB_CUDA(cudaMemcpyAsync(cv.data(), dcovs, sizeof(T) * K * D, cudaMemcpyDeviceToHost, s));
          VLB_CUDA(cudaMemcpyAsync(mu.data(), dmeans, sizeof(T) * K * D, cudaMemcpyDeviceToHost, s));
          VLB_CUDA(cudaStreamSynchronize(s));
          saved = true;
        }
        double bestScore = -INFINITY;
        i64 best = -1;
        for (i64 j = 0; j < K; ++j) {
          if ((double)pr[j] < 1e-6) continue;
          double sc = 0.5 * (double)D * (1.0 + log(2 * 3.141592653589793));
          for (i64 d = 0; d < D; ++d) sc += 0.5 * log((double)cv[j * D + d]);
          sc = (double)pr[j] * (sc - log((double)pr[j]));
          if (sc > bestScore) {
            bestScore = sc;
            best = j;
          }
        }
        if (best == icl || best < 0) continue;
        double bv = -INFINITY;
        i64 bd = -1;
        for (i64 d = 0; d < D; ++d)
          if ((double)cv[best * D + d] > bv) {
            bv = (double)cv[best * D + d];
            bd = d;
          }
        if (bd < 0) continue;
        if (self->verbosity)
          VLB_PRINTF("gmm: reinitializing empty mode %d with mode %d (prior %f, mass %f, score %f)\n",
                     (int)icl, (int)best, (double)pr[best], mass[best], bestScore);
        splits.push_back({(double)icl, (double)best, (double)bd, (double)mu[best * D + bd]});
        rederive_mstep();
        ++nsplit;
      }
      if (nsplit > 0) {
        self->numRestarts += nsplit;
        rederive_mstep();  // the iteration's own M-step on the modified posteriors
      }
    }
    if (nsplit == 0) {
      bool done = false;
      if constexpr (sizeof(T) == 4) {
        if (tcm && !sharded) {
          vlb::tc_em_finalize(item0, dpart, dmeans, dcovs, dpriors, K, D, dlb, s);
          done = true;
        } else if (tcm) {
          // The item sums (f64, into slab 0 of the exact partials), completed
          // across ranks, then the update.
          vlb::tc_em_sums(item0, dpart, K, D, pm, p1, p2, s);
          hsum.resize((size_t)(2 * D + 1) * K);
          VLB_CUDA(cudaMemcpyAsync(hsum.data(), pm, sizeof(double) * K, cudaMemcpyDeviceToHost, s));
          VLB_CUDA(cudaMemcpyAsync(hsum.data() + K, p1, sizeof(double) * K * D, cudaMemcpyDeviceToHost, s));
          VLB_CUDA(cudaMemcpyAsync(hsum.data() + K + K * D, p2, sizeof(double) * K * D, cudaMemcpyDeviceToHost, s));
          VLB_CUDA(cudaStreamSynchronize(s));
          cfg.allreduce(hsum.data(), (vl_size)hsum.size(), cfg.arctx);
          VLB_CUDA(cudaMemcpyAsync(pm, hsum.data(), sizeof(double) * K, cudaMemcpyHostToDevice, s));
          VLB_CUDA(cudaMemcpyAsync(p1, hsum.data() + K, sizeof(double) * K * D, cudaMemcpyHostToDevice, s));
          VLB_CUDA(cudaMemcpyAsync(p2, hsum.data() + K + K * D, sizeof(double) * K * D, cudaMemcpyHostToDevice, s));
          vlb::tc_em_apply(pm, p1, p2, dmeans, dcovs, dpriors, K, D, dlb, s);
          done = true;
        }
      }
      if (!done) exact_finalize(nslab, pm, p1, p2);
    }
  }
  VLB_CUDA(cudaMemcpyAsync(self->means, dmeans, sizeof(T) * K * D, cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaMemcpyAsync(self->covariances, dcovs, sizeof(T) * K * D, cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaMemcpyAsync(self->priors, dpriors, sizeof(T) * K, cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaStreamSynchronize(s));
  // The final E-step's posteriors are recomputed on demand from the data.
  const vl_size last = self->llTrace.size() - 1;
  self->postLazy = true;
  self->lazyX = dX;
  self->lazyPrec = precision;
  self->lazyRouter = (router && last % judgeEvery != 0) ? router : nullptr;
  self->lazyM = cfg.m;
  self->lazyThr = cfg.thr;
  self->lazyChunk = (vl_size)chunk;
  return LL;
}

template <typename T>
double em_stream_default(VlGMM *self, const T *dX, i64 N, int precision) {
  return em_stream_device<T>(self, dX, N, precision, StreamCfg());
}

template <typename T>
const T *stage_data(VlGMM *self, const void *data, i64 N) {
  const i64 D = (i64)self->dimension;
  T *dX = self->dX.get<T>(std::max<i64>(1, N) * D);
  if (N > 0) {
    cudaStream_t s = vlb::thread_stream();
    VLB_CUDA(cudaMemcpyAsync(dX, data, sizeof(T) * N * D, cudaMemcpyHostToDevice, s));
  }
  return dX;
}

// Lanes of the reference's distance kernel on this host (vl/mathop.c:489-510):
// AVX, SSE2 or scalar.
int simd_lanes(bool isFloat) {
  if (vl_get_simd_enabled()) {
    if (vl_cpu_has_avx()) return isFloat ? 8 : 4;
    if (vl_cpu_has_sse2()) return isFloat ? 4 : 2;
  }
  return 1;
}

void drop_kmeans(VlGMM *self) {
  if (self->kmeansInit && self->kmeansInitIsOwner) delete self->kmeansInit;
  self->kmeansInit = nullptr;
  self->kmeansInitIsOwner = false;
}

// Rand initialisation, vl/gmm.c:1416-1443, on device data: uniform priors,
// every covariance the global data variance, means by k-means++ seeding.  The
// random draws come from the calling thread's generator in the reference's
// order (one index, then one real per centre, vl/kmeans.c:615-623), and the
// distances use the summation order of the reference's SIMD kernel for this
// host (AVX, SSE2 or scalar, vl/mathop.c:489-510).  Results go to the host
// parameter arrays, like every VlGMM parameter.
template <typename T>
void init_rand(VlGMM *self, const T *dX, i64 N) {
  VLB_CHECK(N >= 1, VL_ERR_BAD_ARG, "Rand initialisation needs at least one data point");
  cudaStream_t s = vlb::thread_stream();
  const i64 K = (i64)self->numClusters, D = (i64)self->dimension;
  self->numData = (vl_size)N;  // _vl_gmm_prepare_for_data, vl/gmm.c:336-344
  T *pr = (T *)self->priors;
  for (i64 k = 0; k < K; ++k) pr[k] = (T)(1.0 / (double)K);
  VlRand *r = vl_get_rand();
  const i64 x0 = (i64)vl_rand_uindex(r, (vl_uindex)N);
  std::vector<T> thresh((size_t)K);
  for (i64 k = 0; k < K; ++k) thresh[k] = (T)vl_rand_real1(r);
  const int lanes = simd_lanes(sizeof(T) == 4);
  T *dsigma = self->dtmp.get<T>(D);
  T *dcenters = self->dmeans.get<T>(K * D);
  vlb::global_variance<T>(dX, N, D, dsigma, s);
  vlb::kmeanspp<T>(dX, N, D, K, dcenters, x0, thresh, lanes, s);
  std::vector<T> sigma((size_t)D);
  VLB_CUDA(cudaMemcpyAsync(sigma.data(), dsigma, sizeof(T) * D, cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaMemcpyAsync(self->means, dcenters, sizeof(T) * K * D, cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaStreamSynchronize(s));
  T *cv = (T *)self->covariances;
  for (i64 k = 0; k < K; ++k) memcpy(cv + k * D, sigma.data(), sizeof(T) * D);
}

// KMeans initialisation, vl/gmm.c:1315-1370, on device data: k-means (the
// GMM's own object, created on first use with numData/4 comparisons, at least
// 10), exact assignment of every row, then one M-step from the one-hot
// posteriors and zero parameters.  Parameters go to the host arrays; the
// one-hot posteriors stay on the device as the current posteriors.
template <typename T>
void init_kmeans(VlGMM *self, const T *dX, i64 N) {
  VLB_CHECK(N >= 1, VL_ERR_BAD_ARG, "KMeans initialisation needs at least one data point");
  if (!self->kmeansInit) {
    VlKMeans *k = new VlKMeans();
    k->cfg.maxNumComparisons = std::max<i64>(N / 4, 10);
    k->cfg.maxNumIterations = 5;
    k->cfg.numRepetitions = 1;
    self->kmeansInit = k;
    self->kmeansInitIsOwner = true;
  }
  VLB_CHECK(self->kmeansInit->magic == VlKMeans::kMagic, VL_ERR_BAD_ARG,
            "KMeans initialisation: only the library's own k-means object is supported");
  cudaStream_t s = vlb::thread_stream();
  const i64 K = (i64)self->numClusters, D = (i64)self->dimension;
  self->numData = (vl_size)N;  // _vl_gmm_prepare_for_data, vl/gmm.c:336-344
  T *dcenters = self->dtmp.get<T>(K * D);
  uint32_t *dassign = self->dassign.get<uint32_t>(N);
  vlb::kmeans_ann<T>(dX, N, D, K, self->kmeansInit->cfg, simd_lanes(sizeof(T) == 4), dcenters, dassign, s);
  T *dmeans = self->dmeans.get<T>(K * D);
  T *dcovs = self->dcovs.get<T>(K * D);
  T *dpriors = self->dpriors.get<T>(K);
  double *dlb = self->dlb.get<double>(D);
  T *dq = self->dq.get<T>(N * K);
  vlb::onehot_posteriors<T>(dassign, N, K, dq, s);
  VLB_CUDA(cudaMemsetAsync(dmeans, 0, sizeof(T) * K * D, s));  // vl/gmm.c:1326-1328
  VLB_CUDA(cudaMemsetAsync(dcovs, 0, sizeof(T) * K * D, s));
  VLB_CUDA(cudaMemsetAsync(dpriors, 0, sizeof(T) * K, s));
  VLB_CUDA(cudaMemcpyAsync(dlb, self->sigmaLowBound, sizeof(double) * D, cudaMemcpyHostToDevice, s));
  vlb::exact_mstep<T>(dX, N, dq, dmeans, dcovs, dpriors, K, D, dlb, s);
  VLB_CUDA(cudaMemcpyAsync(self->means, dmeans, sizeof(T) * K * D, cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaMemcpyAsync(self->covariances, dcovs, sizeof(T) * K * D, cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaMemcpyAsync(self->priors, dpriors, sizeof(T) * K, cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaStreamSynchronize(s));
  self->postOnDevice = true;
  self->postLazy = false;
}

double em_host(VlGMM *self, const void *data, vl_size N) {
  const int prec = vlb::resolve_precision(VLB200_PREC_DEFAULT, self->dataType == VL_TYPE_DOUBLE);
  if (self->dataType == VL_TYPE_FLOAT)
    return em_device<float>(self, stage_data<float>(self, data, (i64)N), (i64)N, prec);
  return em_device<double>(self, stage_data<double>(self, data, (i64)N), (i64)N, prec);
}

}  // namespace

extern "C" {

VlGMM *vl_gmm_new(vl_type dataType, vl_size dimension, vl_size numComponents) {
  return guarded(
      [&]() -> VlGMM * {
        check_type(dataType);
        VlGMM *self = new VlGMM();
        const size_t sz = tsize(dataType);
        self->dataType = dataType;
        self->dimension = dimension;
        self->numClusters = numComponents;
        self->priors = vl_calloc(numComponents ? numComponents : 1, sz);
        self->means = vl_calloc(numComponents * dimension ? numComponents * dimension : 1, sz);
        self->covariances = vl_calloc(numComponents * dimension ? numComponents * dimension : 1, sz);
        self->sigmaLowBound = (double *)vl_calloc(dimension ? dimension : 1, sizeof(double));
        for (vl_size i = 0; i < dimension; ++i) self->sigmaLowBound[i] = 1e-4;
        return self;
      },
      (VlGMM *)nullptr);
}

VlGMM *vl_gmm_new_copy(VlGMM const *self) {
  VlGMM *g = vl_gmm_new(self->dataType, self->dimension, self->numClusters);
  if (!g) return g;
  const size_t sz = tsize(self->dataType);
  g->initialization = self->initialization;
  g->maxNumIterations = self->maxNumIterations;
  g->numRepetitions = self->numRepetitions;
  g->verbosity = self->verbosity;
  g->LL = self->LL;
  memcpy(g->means, self->means, sz * self->numClusters * self->dimension);
  memcpy(g->covariances, self->covariances, sz * self->numClusters * self->dimension);
  memcpy(g->priors, self->priors, sz * self->numClusters);
  return g;
}

void vl_gmm_reset(VlGMM *self) {
  if (self->posteriors) {
    vl_free(self->posteriors);
    self->posteriors = nullptr;
    self->posteriorsCap = 0;
  }
  self->numData = 0;
  self->postOnDevice = false;
  self->postLazy = false;
  drop_kmeans(self);
}

void vl_gmm_delete(VlGMM *self) {
  if (!self) return;
  vl_free(self->means);
  vl_free(self->covariances);
  vl_free(self->priors);
  vl_free(self->posteriors);
  vl_free(self->sigmaLowBound);
  drop_kmeans(self);
  delete self;
}

// -------------------------------------------------------------- getters
vl_type vl_gmm_get_data_type(VlGMM const *self) { return self->dataType; }
vl_size vl_gmm_get_num_clusters(VlGMM const *self) { return self->numClusters; }
vl_size vl_gmm_get_num_data(VlGMM const *self) { return self->numData; }
double vl_gmm_get_loglikelihood(VlGMM const *self) { return self->LL; }
int vl_gmm_get_verbosity(VlGMM const *self) { return self->verbosity; }
void vl_gmm_set_verbosity(VlGMM *self, int v) { self->verbosity = v; }
void const *vl_gmm_get_means(VlGMM const *self) { return self->means; }
void const *vl_gmm_get_covariances(VlGMM const *self) { return self->covariances; }
void const *vl_gmm_get_priors(VlGMM const *self) { return self->priors; }
void const *vl_gmm_get_posteriors(VlGMM const *self) {
  VlGMM *m = const_cast<VlGMM *>(self);
  guarded(
      [&]() -> int {
        sync_posteriors(m);
        return 0;
      },
      0);
  return m->posteriors;
}
vl_size vl_gmm_get_max_num_iterations(VlGMM const *self) { return self->maxNumIterations; }
void vl_gmm_set_max_num_iterations(VlGMM *self, vl_size n) { self->maxNumIterations = n; }
vl_size vl_gmm_get_num_repetitions(VlGMM const *self) { return self->numRepetitions; }
void vl_gmm_set_num_repetitions(VlGMM *self, vl_size n) {
  if (n < 1) {
    vl_set_last_error(VL_ERR_BAD_ARG, "vl_gmm_set_num_repetitions: must be >= 1");
    return;
  }
  self->numRepetitions = n;
}
vl_size vl_gmm_get_dimension(VlGMM const *self) { return self->dimension; }
VlGMMInitialization vl_gmm_get_initialization(VlGMM const *self) { return self->initialization; }
void vl_gmm_set_initialization(VlGMM *self, VlGMMInitialization init) { self->initialization = init; }
VlKMeans *vl_gmm_get_kmeans_init_object(VlGMM const *self) { return self->kmeansInit; }
void vl_gmm_set_kmeans_init_object(VlGMM *self, VlKMeans *k) {  // vl/gmm.c:628-638
  drop_kmeans(self);
  self->kmeansInit = k;
  self->kmeansInitIsOwner = false;
}
double const *vl_gmm_get_covariance_lower_bounds(VlGMM const *self) { return self->sigmaLowBound; }
void vl_gmm_set_covariance_lower_bounds(VlGMM *self, double const *b) {
  memcpy(self->sigmaLowBound, b, sizeof(double) * self->dimension);
}
void vl_gmm_set_covariance_lower_bound(VlGMM *self, double b) {
  for (vl_size i = 0; i < self->dimension; ++i) self->sigmaLowBound[i] = b;
}

// -------------------------------------------------------------- setters
void vl_gmm_set_means(VlGMM *self, void const *means) {
  memcpy(self->means, means, self->dimension * self->numClusters * tsize(self->dataType));
}
void vl_gmm_set_covariances(VlGMM *self, void const *covs) {
  memcpy(self->covariances, covs, self->dimension * self->numClusters * tsize(self->dataType));
}
void vl_gmm_set_priors(VlGMM *self, void const *priors) {
  memcpy(self->priors, priors, self->numClusters * tsize(self->dataType));
}

// -------------------------------------------------------- processing
void vl_gmm_init_with_rand_data(VlGMM *self, void const *data, vl_size numData) {
  guarded(
      [&]() -> int {
        if (self->dataType == VL_TYPE_FLOAT)
          init_rand<float>(self, stage_data<float>(self, data, (i64)numData), (i64)numData);
        else
          init_rand<double>(self, stage_data<double>(self, data, (i64)numData), (i64)numData);
        return 0;
      },
      0);
}

void vl_gmm_init_with_kmeans(VlGMM *self, void const *data, vl_size numData, VlKMeans *kmeansInit) {
  guarded(
      [&]() -> int {
        if (kmeansInit) vl_gmm_set_kmeans_init_object(self, kmeansInit);  // vl/gmm.c:1333
        if (self->dataType == VL_TYPE_FLOAT)
          init_kmeans<float>(self, stage_data<float>(self, data, (i64)numData), (i64)numData);
        else
          init_kmeans<double>(self, stage_data<double>(self, data, (i64)numData), (i64)numData);
        return 0;
      },
      0);
}

double vl_gmm_em(VlGMM *self, void const *data, vl_size numData) {
  return guarded([&]() -> double { return em_host(self, data, numData); }, (double)NAN);
}

// vl_gmm_cluster, vl/gmm.c:1557-1648.  With VlGMMCustom every repetition
// starts from the parameters present at entry (the reference reuses buffers
// whose contents are undefined after the first repetition).
double vl_gmm_cluster(VlGMM *self, void const *data, vl_size numData) {
  return guarded(
      [&]() -> double {
        const size_t sz = tsize(self->dataType);
        const size_t nKD = self->numClusters * self->dimension;
        std::vector<char> m0((char *)self->means, (char *)self->means + sz * nKD);
        std::vector<char> c0((char *)self->covariances, (char *)self->covariances + sz * nKD);
        std::vector<char> p0((char *)self->priors, (char *)self->priors + sz * self->numClusters);
        std::vector<char> bm, bc, bp;
        double bestLL = -INFINITY;
        bool bestOnDevice = false;
        const int prec = vlb::resolve_precision(VLB200_PREC_DEFAULT, self->dataType == VL_TYPE_DOUBLE);
        const void *dX = self->dataType == VL_TYPE_FLOAT
                             ? (const void *)stage_data<float>(self, data, (i64)numData)
                             : (const void *)stage_data<double>(self, data, (i64)numData);
        for (vl_size rep = 0; rep < self->numRepetitions; ++rep) {
          if (self->verbosity)
            VLB_PRINTF("gmm: clustering: starting repetition %d of %d\n", (int)rep + 1,
                       (int)self->numRepetitions);
          if (self->initialization == VlGMMRand) {  // vl/gmm.c:1588-1593
            if (self->dataType == VL_TYPE_FLOAT)
              init_rand<float>(self, (const float *)dX, (i64)numData);
            else
              init_rand<double>(self, (const double *)dX, (i64)numData);
          } else if (self->initialization == VlGMMKMeans) {
            if (self->dataType == VL_TYPE_FLOAT)
              init_kmeans<float>(self, (const float *)dX, (i64)numData);
            else
              init_kmeans<double>(self, (const double *)dX, (i64)numData);
          } else if (rep > 0) {
            memcpy(self->means, m0.data(), m0.size());
            memcpy(self->covariances, c0.data(), c0.size());
            memcpy(self->priors, p0.data(), p0.size());
          }
          double LL = self->dataType == VL_TYPE_FLOAT
                          ? em_device<float>(self, (const float *)dX, (i64)numData, prec)
                          : em_device<double>(self, (const double *)dX, (i64)numData, prec);
          if (LL > bestLL || rep == 0) {
            bestLL = LL;
            bm.assign((char *)self->means, (char *)self->means + m0.size());
            bc.assign((char *)self->covariances, (char *)self->covariances + c0.size());
            bp.assign((char *)self->priors, (char *)self->priors + p0.size());
            // Posteriors of the best repetition: only the last repetition's are
            // on the device; materialise earlier winners on the host now.
            if (self->numRepetitions > 1) {
              sync_posteriors(self);
              bestOnDevice = false;
            } else {
              bestOnDevice = true;
            }
          }
        }
        if (self->numRepetitions > 1) {
          memcpy(self->means, bm.data(), bm.size());
          memcpy(self->covariances, bc.data(), bc.size());
          memcpy(self->priors, bp.data(), bp.size());
        }
        // The host copy holds an earlier winner's posteriors; a streamed run
        // (posteriors never resident) recomputes them when they are asked for.
        self->postOnDevice = bestOnDevice && !self->postLazy;
        self->LL = bestLL;
        if (self->verbosity)
          VLB_PRINTF("gmm: all repetitions terminated with final loglikelihood %f\n", self->LL);
        return bestLL;
      },
      (double)NAN);
}

// Stand-alone E-step with host pointers, vl/gmm.c:711-798.
static double posteriors_host(vl_type t, void *post, vl_size K, vl_size N, const void *priors,
                              const void *means, vl_size D, const void *covs, const void *data) {
  return guarded(
      [&]() -> double {
        VLB_CHECK(K >= 1 && D >= 1, VL_ERR_BAD_ARG, "numClusters and dimension must be >= 1");
        cudaStream_t s = vlb::thread_stream();
        vlb::Scratch &sc = vlb::thread_scratch();
        const size_t sz = tsize(t);
        char *dX = sc.slot[20].get<char>(sz * std::max<vl_size>(1, N) * D);
        char *dm = sc.slot[21].get<char>(sz * K * D);
        char *dc = sc.slot[22].get<char>(sz * K * D);
        char *dp = sc.slot[23].get<char>(sz * K);
        char *dq = sc.slot[24].get<char>(sz * std::max<vl_size>(1, N) * K);
        if (N) VLB_CUDA(cudaMemcpyAsync(dX, data, sz * N * D, cudaMemcpyHostToDevice, s));
        VLB_CUDA(cudaMemcpyAsync(dm, means, sz * K * D, cudaMemcpyHostToDevice, s));
        VLB_CUDA(cudaMemcpyAsync(dc, covs, sz * K * D, cudaMemcpyHostToDevice, s));
        VLB_CUDA(cudaMemcpyAsync(dp, priors, sz * K, cudaMemcpyHostToDevice, s));
        double ll;
        if (t == VL_TYPE_FLOAT) {
          vlb::DevModel<float> m;
          m.means = (float *)dm; m.covs = (float *)dc; m.priors = (float *)dp;
          m.K = (i64)K; m.D = (i64)D;
          ll = device_estep<float>((float *)dX, (i64)N, m, (float *)dq,
                                   vlb::resolve_precision(VLB200_PREC_DEFAULT, false), false, s);
        } else {
          vlb::DevModel<double> m;
          m.means = (double *)dm; m.covs = (double *)dc; m.priors = (double *)dp;
          m.K = (i64)K; m.D = (i64)D;
          ll = device_estep<double>((double *)dX, (i64)N, m, (double *)dq, VLB200_PREC_EXACT,
                                    false, s);
        }
        if (N) VLB_CUDA(cudaMemcpyAsync(post, dq, sz * N * K, cudaMemcpyDeviceToHost, s));
        VLB_CUDA(cudaStreamSynchronize(s));
        return ll;
      },
      (double)NAN);
}

double vl_get_gmm_data_posteriors_f(float *posteriors, vl_size numClusters, vl_size numData,
                                    float const *priors, float const *means, vl_size dimension,
                                    float const *covariances, float const *data) {
  return posteriors_host(VL_TYPE_FLOAT, posteriors, numClusters, numData, priors, means,
                         dimension, covariances, data);
}

double vl_get_gmm_data_posteriors_d(double *posteriors, vl_size numClusters, vl_size numData,
                                    double const *priors, double const *means, vl_size dimension,
                                    double const *covariances, double const *data) {
  return posteriors_host(VL_TYPE_DOUBLE, posteriors, numClusters, numData, priors, means,
                         dimension, covariances, data);
}

// ---------------------------------------------------------- extensions
int vlb200_gmm_posteriors_device(float *posteriors, vl_size K, vl_size N, float const *priors,
                                 float const *means, vl_size D, float const *covariances,
                                 float const *data, int precision, double *ll, void *stream) {
  return guarded(
      [&]() -> int {
        VLB_CHECK(K >= 1 && D >= 1, VL_ERR_BAD_ARG, "numClusters and dimension must be >= 1");
        vlb::DevModel<float> m;
        m.means = means; m.covs = covariances; m.priors = priors;
        m.K = (i64)K; m.D = (i64)D;
        double v = device_estep<float>(data, (i64)N, m, posteriors,
                                       vlb::resolve_precision(precision, false), false,
                                       vlb::pick_stream(stream));
        if (ll) *ll = v;
        return 0;
      },
      (int)VL_ERR_BAD_ARG);
}

double vlb200_gmm_em_device(VlGMM *self, float const *data, vl_size numData, int precision) {
  return guarded(
      [&]() -> double {
        VLB_CHECK(self->dataType == VL_TYPE_FLOAT, VL_ERR_BAD_ARG,
                  "vlb200_gmm_em_device: the model must be VL_TYPE_FLOAT");
        return em_device<float>(self, data, (i64)numData, vlb::resolve_precision(precision, false));
      },
      (double)NAN);
}

vl_size vlb200_gmm_get_ll_trace(VlGMM const *self, double *trace, vl_size maxEntries) {
  vl_size n = std::min<vl_size>(maxEntries, self->llTrace.size());
  for (vl_size i = 0; i < n; ++i) trace[i] = self->llTrace[i];
  return n;
}

vl_size vlb200_gmm_get_num_restarts(VlGMM const *self) { return self->numRestarts; }

double vlb200_gmm_em_stream_device(VlGMM *self, float const *data, vl_size numData, int precision,
                                   vl_size chunkRows, VlB200Router *router, vl_size m, float threshold,
                                   vl_size judgeEvery) {
  return guarded(
      [&]() -> double {
        VLB_CHECK(self->dataType == VL_TYPE_FLOAT, VL_ERR_BAD_ARG,
                  "vlb200_gmm_em_stream_device: the model must be VL_TYPE_FLOAT");
        StreamCfg cfg;
        cfg.chunk = (i64)chunkRows;
        cfg.router = router;
        cfg.m = m;
        cfg.thr = threshold;
        cfg.judgeEvery = judgeEvery;
        const double ll = em_stream_device<float>(self, data, (i64)numData,
                                                  vlb::resolve_precision(precision, false), cfg);
        self->LL = ll;
        return ll;
      },
      (double)NAN);
}

double vlb200_gmm_em_sharded_device(VlGMM *self, void const *data, vl_size numData, vl_size totalData,
                                    int precision, vl_size chunkRows, vlb200_allreduce_fn allreduce,
                                    void *context) {
  return guarded(
      [&]() -> double {
        VLB_CHECK(allreduce != nullptr && data != nullptr && numData >= 1 && totalData >= numData &&
                      totalData <= (vl_size)INT64_MAX,
                  VL_ERR_BAD_ARG, "vlb200_gmm_em_sharded_device: bad arguments");
        StreamCfg cfg;
        cfg.chunk = (i64)chunkRows;
        cfg.allreduce = allreduce;
        cfg.arctx = context;
        cfg.totalN = (i64)totalData;
        const bool isFloat = self->dataType == VL_TYPE_FLOAT;
        const int prec = vlb::resolve_precision(precision, !isFloat);
        const double ll = isFloat ? em_stream_device<float>(self, (const float *)data, (i64)numData, prec, cfg)
                                  : em_stream_device<double>(self, (const double *)data, (i64)numData, prec, cfg);
        self->LL = ll;
        return ll;
      },
      (double)NAN);
}

vl_size vlb200_gmm_get_stream_report(VlGMM const *self, double *rows, vl_size maxIterations) {
  const vl_size n = std::min<vl_size>(maxIterations, self->streamReport.size());
  for (vl_size i = 0; i < n; ++i)
    for (int j = 0; j < 6; ++j) rows[6 * i + j] = self->streamReport[i][j];
  return n;
}

void vlb200_gmm_set_param_trace(VlGMM *self, int on) {
  self->traceParams = on != 0;
  if (!on) self->paramTrace.clear();
}

vl_size vlb200_gmm_get_param_trace(VlGMM const *self, vl_size iteration, double *means,
                                   double *covariances, double *priors) {
  const vl_size n = self->paramTrace.size();
  if (iteration >= n) return n;
  const std::vector<double> &v = self->paramTrace[iteration];
  const size_t KD = (size_t)self->numClusters * self->dimension;
  if (means) std::copy(v.begin(), v.begin() + KD, means);
  if (covariances) std::copy(v.begin() + KD, v.begin() + 2 * KD, covariances);
  if (priors) std::copy(v.begin() + 2 * KD, v.begin() + 2 * KD + self->numClusters, priors);
  return n;
}

}  // extern "C"
