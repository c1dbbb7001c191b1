// Device-side engine of the GMM / Fisher-vector path.  Everything here takes
// device pointers and a stream; the C API files (gmm_api.cpp, fisher_api.cpp)
// stage host data and call these.
//
// Layouts (VLFeat's, vl/gmm.c:711-798): data[i*D + d], means/covs[k*D + d],
// priors[k], posteriors q[i*K + k]; Fisher vector [u_1..u_K | v_1..v_K].
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_bf16.h>

#include "common.h"

namespace vlb {

using i64 = long long;

// Model parameters on the device, data type T.
template <typename T>
struct DevModel {
  const T *means = nullptr, *covs = nullptr, *priors = nullptr;
  i64 K = 0, D = 0;
};

// Derived per-component constants for the exact E-step (vl/gmm.c:741-756):
// inv = 1/sigma^2, cst = log w - (D/2) log 2pi - (1/2) sum log sigma^2
// (-inf when the prior is below 1e-6), sis = sqrt(1/sigma^2) (vl/fisher.c:388).
template <typename T>
struct DevDerived {
  T *inv = nullptr;
  double *cst = nullptr;
  T *sis = nullptr;
};

// ---------------------------------------------------------------- exact path
template <typename T>
void exact_prepare(const DevModel<T> &m, DevDerived<T> &der, cudaStream_t s);

// E-step over rows [0, N): q (N x K) receives posteriors; per-block LL partials
// go to ll_part (capacity estep_ll_parts(N)); returns the number of partials
// written.  If fast, q is replaced by the one-hot arg-max (vl/fisher.c:398-417).
i64 estep_ll_parts(i64 N);
template <typename T>
i64 exact_estep(const T *X, i64 N, const DevModel<T> &m, const DevDerived<T> &der, T *q,
                 double *ll_part, bool fast, cudaStream_t s);

// Deterministic sum of n doubles into *out (device).
void sum_doubles(const double *part, i64 n, double *out, cudaStream_t s);

// M-step (vl/gmm.c:1036-1213) in place on means/covs/priors (device, type T):
// thresholded sufficient statistics, old-mean correction, bounds, prior
// normalisation.  lb: D doubles (device).
template <typename T>
void exact_mstep(const T *X, i64 N, const T *q, T *means, T *covs, T *priors, i64 K, i64 D,
                 const double *lb, cudaStream_t s);
// The same M-step over rows streamed in chunks: the rows are cut into slabs
// of `rps` rows (exact_mstep_slab_rows(N) is exact_mstep's own choice), each
// chunk starting on a slab boundary; exact_mstep_stats_rows writes the slab
// partials of rows [row0, row0 + n) (posteriors q: n x K) centred on
// oldMeans; exact_mstep_finalize_slabs reduces nslab slabs in order and
// updates the parameters.  pmass: nslab x K, ps1/ps2: nslab x K x D doubles.
i64 exact_mstep_slab_rows(i64 N);
template <typename T>
void exact_mstep_stats_rows(const T *X, i64 row0, i64 n, i64 rps, const T *q, const T *oldMeans, i64 K,
                            i64 D, double *pmass, double *ps1, double *ps2, cudaStream_t s);
template <typename T>
void exact_mstep_finalize_slabs(int nslab, const double *pmass, const double *ps1, const double *ps2,
                                const double *lb, T *means, T *covs, T *priors, i64 K, i64 D,
                                cudaStream_t s);
// Sums the nslab slabs' partials into slab 0 (in slab order): the
// finalize over that one slab then gives the same parameters, and the sums
// ((2D + 1) K doubles: pmass[0..K), ps1[0..KD), ps2[0..KD)) can be added
// across ranks first.
void exact_sum_slabs(int nslab, double *pmass, double *ps1, double *ps2, i64 K, i64 D, cudaStream_t s);

// Rand initialisation pieces (vl/gmm.c:1376-1443), bit-exact with the
// reference.  global_variance: sigma (D) from X (N x D).  kmeanspp: K centres
// from X by k-means++ (vl/kmeans.c:588-649); x0 and thresh (K values, already
// cast to T) are the reference's draws from the calling thread's generator;
// lanes (8, 4, 2 or 1) selects the summation order of the reference's
// distance kernel that the host's SIMD support selects.
template <typename T>
void global_variance(const T *X, i64 N, i64 D, T *sigma, cudaStream_t s);
template <typename T>
void kmeanspp(const T *X, i64 N, i64 D, i64 K, T *centers, i64 x0, const std::vector<T> &thresh, int lanes,
              cudaStream_t s);

// KMeans initialisation (vl/gmm.c:1315-1370).  The settings of the k-means
// object that the GMM creates for it (vl/gmm.c:1336-1356); the object itself
// is struct _VlKMeans (k_kmeans.cu).
struct KMeansSettings {
  i64 maxNumIterations = 5;
  i64 maxNumComparisons = 10;
  i64 numRepetitions = 1;
  double minEnergyVariation = 1e-4;  // vl/kmeans.c:416
};
// vl_kmeans_cluster with random-selection seeding and ANN refinement over a
// one-tree kd-forest (vl/kmeans.c:2024-2093, 528-582, 1003-1150), then
// vl_kmeans_quantize (vl/kmeans.c:656-702).  centers (K x D) and assign (N)
// are device outputs; random draws come from the calling thread's generator in
// the reference's order; lanes as for kmeanspp.  Returns the best energy.
template <typename T>
double kmeans_ann(const T *X, i64 N, i64 D, i64 K, const KMeansSettings &cfg, int lanes, T *centers,
                  uint32_t *assign, cudaStream_t s);
// q (N x K) = the one-hot rows of assign (vl/gmm.c:1361-1364).
template <typename T>
void onehot_posteriors(const uint32_t *assign, i64 N, i64 K, T *q, cudaStream_t s);

// priors /= max(sum priors, 1e-12) on the device (vl/gmm.c:1196-1211).
template <typename T>
void normalize_priors(T *priors, i64 K, cudaStream_t s);

// Un-thresholded posterior mass per component (vl/gmm.c:835-844), K doubles.
template <typename T>
void column_mass(const T *q, i64 N, i64 K, double *mass, cudaStream_t s);

// Hard split of mode `best` into empty mode `icl` along dimension `dim`
// (vl/gmm.c:969-989).
template <typename T>
void restart_split(T *q, const T *X, i64 N, i64 K, i64 D, i64 icl, i64 best, i64 dim, T cut,
                   cudaStream_t s);

// Variance floor applied on device (vl/gmm.c:1005-1030).
template <typename T>
void apply_bounds(T *covs, i64 K, i64 D, const double *lb, cudaStream_t s);

// --------------------------------------------------------------- Fisher
// One image segment: rows [row0, row1) of image `image`; q rows are indexed
// relative to the chunk's first row.
struct Segment {
  i64 image, row0, row1;
};

// Batched Fisher encoding with the exact path.  h_offsets: numImages+1 host
// array.  enc: numImages x 2KD (device).  nterms: numImages (device) or null.
template <typename T>
void exact_fisher_batch(const T *X, const i64 *h_offsets, i64 numImages, const DevModel<T> &m,
                        T *enc, unsigned long long *nterms, int flags, cudaStream_t s,
                        bool use_router = false);

// Single-image exact Fisher encoding on caller-provided scratch (no
// allocation, no host-to-device copies, no event timing).  Every scratch
// element the kernels read is written earlier in the same call.
struct ExactFvScratch {
  float *inv, *sis, *q;
  double *cst, *llp, *pu, *pv;
  Segment *segs;
  int *segBegin;
  i64 *rows;
  unsigned long long *pnt;
};
i64 exact_fv_segments(i64 N);  // segments one image of N rows is cut into
void exact_fisher_single_fixed(const float *X, i64 N, const DevModel<float> &m, float *enc,
                               unsigned long long *nterms, int flags, const ExactFvScratch &sc,
                               cudaStream_t s);

// Posteriors (N x K, row-major) from the process-wide default router
// (vlb200_router_set_default); implemented in k_router.cu.
void router_default_posteriors(const float *X, i64 N, const DevModel<float> &m, float *q,
                               cudaStream_t s);

// ------------------------------------------------------- tensor-core path
// Implemented in k_tc.cu.  Available for float data only.
bool tc_supported(i64 K, i64 D);
// Dense layer on the tensor cores (k_mlp.cu): C (M x N) = act(A (M x Ka) .
// W (N x Ka)^T + bias), A and W bf16 row-major, fp32 accumulation, ReLU when
// relu, C fp32 when outF32 else bf16; N and Ka multiples of 8.  An expired
// wait writes its code to *err (device).
bool tc_dense_supported(int N, int Ka);
// With selM in 1..16 (N >= 32) the last layer's epilogue does not write C:
// it keeps each row's selM largest outputs (ties: lowest index) in cand
// (rows x selM) and their softmax mass over all N in cmass (rows).
void tc_dense(const __nv_bfloat16 *A, long long M, int Ka, const __nv_bfloat16 *W, int N, const float *bias,
              bool relu, bool outF32, void *C, int *err, cudaStream_t s, int selM = 0, int *cand = nullptr,
              float *cmass = nullptr);
void features_bf16(const float *X, long long n, int D, int Ka, const float *ctr, const float *scl,
                   __nv_bfloat16 *Z, cudaStream_t s);
void weights_bf16(const float *W, int out, int in, int inPad, __nv_bfloat16 *Wb, cudaStream_t s);
// Runs the bounded-wait self-test kernel with a wait limit of limit_ms and
// raises the error a kernel's expired wait raises.
void wait_selftest(double limit_ms, cudaStream_t s);
// The tensor-core Fisher encoder (E-step, statistics and the cluster finalize).
bool tc_fv_supported(i64 K, i64 D);
// Shapes the tensor-core E-step (posteriors) and Fisher encoding take with
// the dimension zero-padded to the next one the kernels are built for (64,
// 80 or 128; any D <= 128).
int tc_pad_dim(i64 D);
bool tc_supported_padded(i64 K, i64 D);
bool tc_fv_supported_padded(i64 K, i64 D);
i64 tc_estep(const float *X, i64 N, const DevModel<float> &m, float *q, double *ll_part,
             bool fast, int precision, cudaStream_t s, Scratch *arena = nullptr);
// EM with the tensor-core M-step.  tc_estep_em is the E-step of tc_estep that
// also writes the posteriors as the statistics operand image, thresholded at
// the M-step's skip (vl/gmm.c:1099); tc_mstep then runs the M-step
// (vl/gmm.c:1036-1213) from that image and the centre of that E-step's model,
// on the same thread, in place on means/covs/priors (device, fp32).
i64 tc_estep_em(const float *X, i64 N, const DevModel<float> &m, float *q, double *ll_part,
                int precision, cudaStream_t s);
void tc_mstep(const float *X, i64 N, float *means, float *covs, float *priors, i64 K, i64 D,
              const double *lb, int precision, cudaStream_t s);
// Streaming EM, one chunk of rows at a time (N x K never resident).  After
// tc_estep_em on a chunk (or tc_em_image_from_rows, which makes the chunk's
// thresholded fp16 image from row-major posteriors), tc_em_stats adds the
// chunk's statistics (rows [row0, row0 + n) of X; split 2: fp16x3 from the
// FP32 mode's image, 1: one fp16 q part) as tc_em_items(n) item partials
// starting at item0 of `partial` (tc_em_partial_floats(K, D) floats each);
// tc_em_finalize then applies the M-step from all nitems partials, in f64.
// Every call of a pass uses the same model, on the same thread.
void tc_em_image_from_rows(const float *qrows, i64 n, const DevModel<float> &m, cudaStream_t s);
i64 tc_em_items(i64 n);
size_t tc_em_partial_floats(i64 K, i64 D);
void tc_em_stats(const float *X, i64 row0, i64 n, i64 K, i64 D, int split, float *partial, int item0,
                 cudaStream_t s);
void tc_em_finalize(int nitems, const float *partial, float *means, float *covs, float *priors, i64 K,
                    i64 D, const double *lb, cudaStream_t s);
// The same M-step in two parts: tc_em_sums writes the f64 sums of the
// partials (S0: K, S1 and S2: K x D, scale factors taken out), which can be
// added across ranks, and tc_em_apply updates the parameters from them
// (using the centre of the last tc_prepare on this thread).
void tc_em_sums(int nitems, const float *partial, i64 K, i64 D, double *S0, double *S1, double *S2,
                cudaStream_t s);
void tc_em_apply(const double *S0, const double *S1, const double *S2, float *means, float *covs, float *priors,
                 i64 K, i64 D, const double *lb, cudaStream_t s);
void tc_fisher_batch(const float *X, const i64 *h_offsets, i64 numImages,
                     const DevModel<float> &m, float *enc, unsigned long long *nterms, int flags,
                     int precision, cudaStream_t s);

// Tunable shapes of the batched Fisher encoder (0: the built-in choice).
struct TcFvConfig {
  i64 itemRows = 8192;  // rows per statistics work item (multiple of 128)
  int statsMT = 0;      // 128-component M tiles per statistics CTA: 0 (two when they fit), 1, 2
  int statsStages = 0;  // operand stages of the statistics kernel (0: as many as fit)
  int estepStages = 0;  // operand stages of the E-step (0: as many as fit, at most 8)
  i64 rowBudget = 0;    // rows per E-step launch (0: a 4 GB q image)
};

// A batched encoder bound to one batch layout (image offsets), flags and
// precision.  It owns its tables and scratch, so that tc_fv_plan_run only
// launches kernels: no allocation after the first run, no host copies and no
// synchronisation, which makes it capturable in a CUDA graph.
struct TcFvPlan;
TcFvPlan *tc_fv_plan_new(i64 D, i64 K, const i64 *offsets, i64 numImages, int flags, int precision,
                         cudaStream_t s);
void tc_fv_plan_delete(TcFvPlan *p);
TcFvConfig tc_fv_plan_config(const TcFvPlan *p);
void tc_fv_plan_set_config(TcFvPlan *p, const TcFvConfig &c, cudaStream_t s);
void tc_fv_plan_run(TcFvPlan *p, const DevModel<float> &m, const float *X, float *enc,
                    unsigned long long *nterms, cudaStream_t s);
int tc_fv_plan_error(TcFvPlan *p, cudaStream_t s);  // the kernels' error word (synchronises)
// Host buffers in and out, copies overlapped with the encode chunk by chunk;
// returns when the encodings are on the host.
void tc_fv_plan_run_host(TcFvPlan *p, const DevModel<float> &m, const float *Xh, float *ench,
                         unsigned long long *nth, cudaStream_t s);
TcFvConfig tc_fv_plan_autotune(TcFvPlan *p, const DevModel<float> &m, const float *X, float *enc,
                               unsigned long long *nterms, cudaStream_t s, double *best_ms);

}  // namespace vlb
