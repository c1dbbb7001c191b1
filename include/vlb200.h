/* vlb200.h -- extension entry points of the B200 GMM / Fisher-vector library.
 *
 * These are NOT VLFeat names.  The reference's API (vl/gmm.h, vl/fisher.h)
 * takes host pointers, which bounds throughput by host<->device copies
 * (320 B per D=80 float descriptor).  The entry points below take device
 * pointers, encode many images in one call, and select the arithmetic used
 * on the GPU.  All pointers marked "device" must be CUDA device (or managed)
 * memory of the current device; "stream" is a cudaStream_t (NULL = the
 * calling thread's library stream).  Every function returns 0 on success and
 * a VL_ERR_* code on failure, with the message in vl_get_last_error_message().
 */
#ifndef VLB200_H
#define VLB200_H

#include "vl/generic.h"
#include "vl/gmm.h"

struct _VlB200Router; /* the learned router, declared below */

/* Arithmetic used on the GPU.
 *  EXACT      direct (x-mu)^2/sigma^2 evaluation in the data type on CUDA cores
 *             (float or double), the reference's own formulation
 *             (vl/gmm.c:762-775, vl/fisher.c:442-447).
 *  FP32       tensor cores: E-step and statistics contractions in fp16x3
 *             split precision (two fp16 parts per operand, power-of-two
 *             scaled) with fp32 accumulation (FP32-grade results).
 *  BF16       tensor cores: fp16x3 E-step, statistics with a single fp16 part
 *             of the posteriors (rel err ~1e-4; the name is the mode's).
 *  BF16_ROUTER  learned router picks candidate components; exact posteriors
 *             on the candidates only; fp16 statistics; full E-step fallback
 *             for descriptors whose predicted candidate mass is < 0.99.
 * DEFAULT resolves to the process-wide mode (vlb200_set_precision), which
 * starts as EXACT -- VLFeat's own float arithmetic, so that a relinked
 * program gets the reference's float results -- unless the environment
 * variable VLB200_PRECISION names fp32 or bf16 at load time.  (FP32 is the
 * faster and, against FP64, the more accurate of the two float modes; EXACT
 * is the one that reproduces VLFeat's float roundings.)  VL_TYPE_DOUBLE calls
 * always run EXACT in double. */
#define VLB200_PREC_DEFAULT 0
#define VLB200_PREC_EXACT 1
#define VLB200_PREC_FP32 2
#define VLB200_PREC_BF16 3
#define VLB200_PREC_BF16_ROUTER 4

VL_EXPORT int vlb200_set_precision(int precision);
VL_EXPORT int vlb200_get_precision(void);
/* The arithmetic (VLB200_PREC_EXACT .. BF16_ROUTER) that the calling
 * thread's most recent Fisher encode, E-step or EM iteration actually ran; 0
 * before any such call.  A tensor-core mode requested for a shape the
 * tensor-core kernels do not take (tensor-core E-step: 8 <= numClusters <=
 * 2048, numClusters % 8 == 0, dimension <= 128; Fisher encoding also needs
 * numClusters % 4 == 0 and the finalisation's shared memory) runs EXACT,
 * and this reports it.  No reference counterpart. */
VL_EXPORT int vlb200_last_precision(void);

/* Library / device information. */
VL_EXPORT char const *vlb200_version(void);
VL_EXPORT int vlb200_device_ok(void); /* 1 if a usable CUDA device is present */

/* Count of kernels this library has launched in this process (all threads). */
VL_EXPORT vl_uint64 vlb200_launch_count(void);

/* Kernel timing.  When enabled, every launch is bracketed by CUDA events on
 * its own stream; vlb200_profile_read() synchronises and reports, per kernel
 * name, the number of launches and the summed device time in ms. */
VL_EXPORT void vlb200_profile_enable(int on);
VL_EXPORT int vlb200_profile_read(char *names, vl_size nameStride, double *ms,
                                  vl_uint64 *launches, vl_size maxEntries);
VL_EXPORT void vlb200_profile_reset(void);

/* E-step on device data (vl_get_gmm_data_posteriors_f, vl/gmm.h:94-103, with
 * device pointers).  posteriors: numData x numClusters, device.  *ll receives
 * the log-likelihood (host pointer).  The tensor-core modes read the data with
 * TMA and store the posteriors 16 bytes at a time: both device arrays must
 * start 16-byte aligned there (else VL_ERR_BAD_ARG, nothing launched); the
 * exact mode takes any float alignment. */
VL_EXPORT int vlb200_gmm_posteriors_device(float *posteriors, vl_size numClusters,
                                           vl_size numData, float const *priors,
                                           float const *means, vl_size dimension,
                                           float const *covariances, float const *data,
                                           int precision, double *ll, void *stream);

/* EM on device-resident data: the vl_gmm_em loop (vl/gmm.c:1220-1308) with
 * the data already in device memory.  The model's parameters stay the host
 * copies visible through vl_gmm_get_*; posteriors are fetched lazily. */
VL_EXPORT double vlb200_gmm_em_device(VlGMM *self, float const *data, vl_size numData,
                                      int precision);

/* EM on device-resident data whose N x numClusters posteriors are never
 * resident (no reference counterpart; the loop is vl_gmm_em's, vl/gmm.c:
 * 1220-1308, with the reference's stopping rules and empty-mode restarts).
 * Each E-step pass runs in chunks of about chunkRows rows (0: about 8 GB of
 * posteriors per chunk), and the chunk's M-step statistics, column masses and
 * log-likelihood are accumulated while its posteriors exist; the M-step is
 * reduced in f64.  With a router (not NULL, trained or not; numClusters and
 * dimension as the model's, set_input_transform applied), iterations that
 * are not multiples of judgeEvery take the exact posteriors of each row's m
 * router candidates only (full E-step for rows whose predicted candidate
 * mass is below threshold; their log-likelihood is the log-sum-exp over the
 * components evaluated), and every judgeEvery-th iteration runs the full
 * E-step, re-fits the router on the first 2^20 rows' posteriors (4 epochs at
 * iteration 0, then 1) and measures its missed posterior mass on the other
 * rows.  vl_gmm_get_posteriors afterwards recomputes the final E-step chunk
 * by chunk from `data`, which must then still be valid.  vl_gmm_em and
 * vl_gmm_cluster take this path by themselves when the posteriors would not
 * fit in free device memory.  Returns the final log-likelihood (NaN on
 * error). */
VL_EXPORT double vlb200_gmm_em_stream_device(VlGMM *self, float const *data, vl_size numData,
                                             int precision, vl_size chunkRows,
                                             struct _VlB200Router *router, vl_size m,
                                             float threshold, vl_size judgeEvery);
/* Sums `count` doubles in place over all ranks of a sharded EM.  Every rank
 * calls it with the same counts in the same order (the rank's C-ABI call
 * below makes the calls); it returns when the sums are complete. */
typedef void (*vlb200_allreduce_fn)(double *values, vl_size count, void *context);

/* EM with the rows sharded over ranks (one process and device each): this
 * rank holds numData rows of data (device, VL_TYPE_FLOAT or VL_TYPE_DOUBLE as
 * the model, at least one row) of totalData in all.  Every rank sets the same
 * initial parameters and options.  The loop is the streamed EM's
 * (vlb200_gmm_em_stream_device, no router) on the rank's rows; each sum over
 * rows is completed by `allreduce` before it is used: per iteration the
 * log-likelihood and (from iteration 2) the component masses of the restart
 * check (vl/gmm.c:814-999, with totalData in its cut-off), and the M-step
 * sums ((2 D + 1) numClusters doubles, vl/gmm.c:1036-1213), once more per
 * restart.  All ranks end with the same parameters and log-likelihood
 * (returned; NaN on error).  vl_gmm_get_posteriors gives this rank's rows. */
VL_EXPORT double vlb200_gmm_em_sharded_device(VlGMM *self, void const *data, vl_size numData,
                                              vl_size totalData, int precision, vl_size chunkRows,
                                              vlb200_allreduce_fn allreduce, void *context);

/* One row of 6 doubles per E-step of the last streamed EM: log-likelihood,
 * judged (1: full E-step with the router judged), routed (1: router E-step),
 * mean missed posterior mass of the router on the judged rows (NaN when not
 * judged), rows that fell back to the full E-step, milliseconds (wall clock,
 * the E-step pass with its statistics).  Returns the rows written. */
VL_EXPORT vl_size vlb200_gmm_get_stream_report(VlGMM const *self, double *rows, vl_size maxIterations);

/* Per-iteration log-likelihood trace of the last EM run (up to maxEntries
 * values; returns the number written). */
VL_EXPORT vl_size vlb200_gmm_get_ll_trace(VlGMM const *self, double *trace, vl_size maxEntries);
/* Number of empty modes re-seeded in the last EM run. */
VL_EXPORT vl_size vlb200_gmm_get_num_restarts(VlGMM const *self);
/* Parameter trace of EM runs (off by default; no reference counterpart: the
 * reference returns only the final parameters, vl/gmm.c:1220-1308).  When on,
 * each EM iteration first copies the parameters its E-step uses back to the
 * host, so entry t holds them after t M-steps (t = 0 .. the number of
 * iterations).  get copies entry `iteration` as double (means and covariances
 * numClusters x dimension, priors numClusters; each pointer may be NULL) and
 * returns the number of entries, writing nothing when iteration is past
 * them. */
VL_EXPORT void vlb200_gmm_set_param_trace(VlGMM *self, int on);
VL_EXPORT vl_size vlb200_gmm_get_param_trace(VlGMM const *self, vl_size iteration, double *means,
                                             double *covariances, double *priors);

/* Fisher encoding of one image with device pointers (vl_fisher_encode,
 * vl/fisher.h:48-54).  enc: 2*D*K floats, device.  numTerms: host pointer or
 * NULL. */
VL_EXPORT int vlb200_fisher_encode_device(float *enc, float const *means, vl_size dimension,
                                          vl_size numClusters, float const *covariances,
                                          float const *priors, float const *data,
                                          vl_size numData, int flags, int precision,
                                          vl_uint64 *numTerms, void *stream);

/* Batched Fisher encoding of many images of uneven size in one call.
 * data: total x D floats (device), image j owns rows offsets[j] ..
 * offsets[j+1]-1; offsets: numImages+1 int64 (host).  enc: numImages x 2DK
 * floats (device), image-major.  numTerms: numImages uint64 (device) or NULL.
 * Equivalent to numImages calls of vl_fisher_encode. */
VL_EXPORT int vlb200_fisher_encode_batch_device(float *enc, float const *means, vl_size dimension,
                                                vl_size numClusters, float const *covariances,
                                                float const *priors, float const *data,
                                                vl_int64 const *offsets, vl_size numImages,
                                                int flags, int precision, vl_uint64 *numTerms,
                                                void *stream);

/* Batched VLAD encoding (vl_vlad_encode, vl/vlad.h:45-50) of many images
 * of uneven size in one call, with device pointers.  dataType: VL_TYPE_FLOAT
 * or VL_TYPE_DOUBLE, for every array.  data: total x dimension rows; image j
 * owns rows offsets[j] .. offsets[j+1]-1 of data and of assignments (total x
 * numClusters weights); offsets: numImages+1 int64 (host).  enc: numImages x
 * numClusters x dimension (device), image-major.  Each image's encoding is
 * bit-equal to vl_vlad_encode on its rows.  dimension <= 1024.  Returns 0, or
 * a VL_ERR_* code (recorded as the last error).  Returns once the encodings
 * are written. */
VL_EXPORT int vlb200_vlad_encode_batch_device(void *enc, vl_type dataType, void const *means,
                                              vl_size dimension, vl_size numClusters,
                                              void const *data, void const *assignments,
                                              vl_int64 const *offsets, vl_size numImages,
                                              int flags, void *stream);

/* ---------------------------------------------------- descriptor prologue
 * The recognition app's step before encoding (apps/recognition/encodeImage.m:
 * 91-103): out = P (data - center), each row optionally L2-renormalised
 * (times 1 / max(1e-12, norm)), then, when frames is not NULL, the frame
 * position normalised by the image size appended ('xy' geometric extension,
 * apps/recognition/extendDescriptorsWithGeometry.m:19-21): row i of out is
 * [y_i, (fx - w/2)/w, (fy - h/2)/h].  All arrays are device pointers except
 * offsets (numImages+1 int64, host).  projection: dimOut x dimIn, center:
 * dimIn, data: numData x dimIn, out: numData x (dimOut + 2 if frames);
 * frames: numData x 2 (pixel x, y); imageSizes: numImages x 2 (w, h), image j
 * owning rows offsets[j] .. offsets[j+1]-1.  dimIn, dimOut <= 128.  FP32
 * arithmetic.  Returns 0 or a VL_ERR_* code. */
VL_EXPORT int vlb200_pca_project_device(float *out, vl_size dimOut, float const *data, vl_size dimIn,
                                        vl_size numData, float const *projection, float const *center,
                                        int renormalize, float const *frames, vl_int64 const *offsets,
                                        float const *imageSizes, vl_size numImages, void *stream);

/* PCA of a descriptor sample as the app learns it (apps/recognition/
 * trainEncoder.m:150-171): center = mean, C = (data - center)^T (data -
 * center) / numData (fp64 on the GPU), eigenvectors by decreasing eigenvalue
 * d (cyclic Jacobi, fp64, host), d += whiteningRegul * max(d); projection
 * (numPcaDimensions x dimIn, device) = the first eigenvectors as rows,
 * scaled by 1/sqrt(d) when whitening, each with its largest-magnitude entry
 * positive; center: dimIn (device); eigenvalues: numPcaDimensions regularised
 * eigenvalues (host) or NULL.  dimIn <= 128. */
VL_EXPORT int vlb200_pca_learn_device(float *projection, float *center, vl_size numPcaDimensions,
                                      float const *data, vl_size dimIn, vl_size numData, int whitening,
                                      double whiteningRegul, double *eigenvalues, void *stream);

/* ------------------------------------------------------ batched encode plan
 * A plan binds the tensor-core batched encoder to one batch layout (offsets,
 * numImages), dimension, numClusters, flags and precision (FP32, BF16 or
 * BF16_ROUTER; DEFAULT resolves as elsewhere).  It owns every table and
 * scratch buffer of the encode, so that execute only launches kernels: after
 * its first call it allocates nothing, copies nothing from the host and does
 * not synchronise, and a whole encode can be captured in a CUDA graph and
 * replayed.  Results equal numImages calls of vl_fisher_encode
 * (vl/fisher.c:548-579) computed in the chosen precision; no reference
 * counterpart.  Functions returning int return 0 or a VL_ERR_* code (also
 * recorded as the last error); vlb200_fisher_plan_new returns NULL on error.
 *
 * Tile configuration (vlb200_fisher_plan_get/set_config), five int64:
 *   [0] rows per statistics work item (multiple of 128, default 8192)
 *   [1] 128-component M tiles per statistics CTA (0: two when they fit; 1; 2)
 *   [2] operand stages of the statistics kernel (0: as many as fit)
 *   [3] operand stages of the E-step (0: as many as fit)
 *   [4] rows per E-step launch (0: a 4 GB posterior image)
 * vlb200_fisher_plan_autotune times a set of candidates on the given data
 * (CUDA events, median of three runs each) and keeps the fastest; bestMs
 * (may be NULL) receives its time per encode. */
typedef struct _VlB200FisherPlan VlB200FisherPlan;
VL_EXPORT VlB200FisherPlan *vlb200_fisher_plan_new(vl_size dimension, vl_size numClusters,
                                                   vl_int64 const *offsets, vl_size numImages,
                                                   int flags, int precision);
VL_EXPORT void vlb200_fisher_plan_delete(VlB200FisherPlan *plan);
/* Binds the GMM by device pointers (means, covariances: K x D; priors: K).
 * Every execute reads their current contents. */
VL_EXPORT int vlb200_fisher_plan_set_gmm(VlB200FisherPlan *plan, float const *means,
                                         float const *covariances, float const *priors);
VL_EXPORT int vlb200_fisher_plan_execute(VlB200FisherPlan *plan, float *enc, float const *data,
                                         vl_uint64 *numTerms, void *stream);
/* The same encode from HOST buffers (data: the batch's rows, enc: numImages x
 * 2DK, numTerms: numImages or NULL), like vl_fisher_encode: the batch is cut
 * into about 16 chunks of whole images whose host -> device copies, encodes
 * and device -> host copies overlap on three streams.  Returns when the
 * results are on the host.  Page-locked buffers (cudaHostAlloc,
 * cudaHostRegister) are needed for the copies to overlap. */
VL_EXPORT int vlb200_fisher_plan_execute_host(VlB200FisherPlan *plan, float *enc,
                                              float const *data, vl_uint64 *numTerms,
                                              void *stream);
VL_EXPORT int vlb200_fisher_plan_autotune(VlB200FisherPlan *plan, float *enc, float const *data,
                                          vl_uint64 *numTerms, void *stream, double *bestMs);
VL_EXPORT int vlb200_fisher_plan_get_config(VlB200FisherPlan const *plan, vl_int64 config[5]);
VL_EXPORT int vlb200_fisher_plan_set_config(VlB200FisherPlan *plan, vl_int64 const config[5],
                                            void *stream);
/* Runs one encode outside capture, then captures one into a CUDA graph bound
 * to these buffers and this stream (a created stream, not the default one).
 * vlb200_fisher_plan_launch replays it.  set_gmm, set_config and autotune
 * drop the graph. */
VL_EXPORT int vlb200_fisher_plan_capture(VlB200FisherPlan *plan, float *enc, float const *data,
                                         vl_uint64 *numTerms, void *stream);
VL_EXPORT int vlb200_fisher_plan_launch(VlB200FisherPlan *plan, void *stream);
/* Synchronises the stream and returns the kernels' error word: 0, or the
 * code of a bounded wait that gave up. */
VL_EXPORT int vlb200_fisher_plan_status(VlB200FisherPlan *plan, void *stream);

/* ----------------------------------------------------------------- router
 * Learned candidate router for the E-step (no reference counterpart; the
 * reference always evaluates every component, vl/gmm.c:758-791).  An MLP
 * D -> hidden... -> K (ReLU, bf16 weights, fp32 accumulation) predicts each
 * descriptor's top-m components; the exact posterior is computed on those
 * only, and the full E-step is used for descriptors whose predicted candidate
 * mass is below a threshold.  Trained on the GPU by the library's own
 * forward / backward / Adam kernels against the top-8 posteriors of the full
 * E-step.  All pointers to data are device pointers unless stated. */
typedef struct _VlB200Router VlB200Router;
VL_EXPORT VlB200Router *vlb200_router_new(vl_size dimension, vl_size numClusters,
                                          vl_size const *hidden, vl_size numHidden,
                                          vl_uint32 seed);
VL_EXPORT void vlb200_router_delete(VlB200Router *router);
VL_EXPORT vl_size vlb200_router_num_params(VlB200Router const *router);
/* Host vector: per layer W (out x in, row-major) then b. */
VL_EXPORT int vlb200_router_get_params(VlB200Router const *router, float *params);
VL_EXPORT int vlb200_router_set_params(VlB200Router *router, float const *params);
/* Input features z = (x - centre) * scale; host arrays of D. */
VL_EXPORT int vlb200_router_set_input_transform(VlB200Router *router, float const *centre,
                                                float const *scale);
/* Top-8 targets (N x 8 indices and renormalised weights) of posteriors. */
VL_EXPORT int vlb200_router_targets(float const *posteriors, vl_size numData,
                                    vl_size numClusters, int *targetIdx, float *targetWeight);
/* Mean top-8 cross-entropy of a batch and, if grads (host) is non-NULL, its
 * gradient in the get_params layout. */
VL_EXPORT int vlb200_router_loss_grad(VlB200Router *router, float const *data, vl_size batch,
                                      int const *targetIdx, float const *targetWeight,
                                      double *loss, float *grads);
VL_EXPORT int vlb200_router_train(VlB200Router *router, float const *data, vl_size numData,
                                  int const *targetIdx, float const *targetWeight, vl_size epochs,
                                  vl_size batch, float learningRate, double *lastEpochLoss);
/* Posteriors (N x K, zero off the candidates) from the top-m candidates;
 * fallbackRows (host, may be NULL) counts rows that used the full E-step. */
VL_EXPORT int vlb200_router_posteriors(VlB200Router *router, float *posteriors,
                                       float const *priors, float const *means,
                                       float const *covariances, float const *data,
                                       vl_size numData, vl_size m, float threshold,
                                       vl_uint64 *fallbackRows, void *stream);
VL_EXPORT int vlb200_router_missed_mass(float const *fullPosteriors,
                                        float const *candidatePosteriors, vl_size numData,
                                        vl_size numClusters, double *meanMissedMass);
/* Inference engine: 1 (default) runs the network's layers as tcgen05 dense
 * layers (bf16 features, activations and weights, fp32 accumulation, TMA-
 * staged tiles) when every layer width is a multiple of 8; 0 runs the
 * training forward (fp32 activations, bf16-rounded weights) on the CUDA
 * cores.  vlb200_router_logits returns the inference logits (N x K fp32,
 * device) of rows X (N x D, device). */
VL_EXPORT int vlb200_router_set_tensor_core_inference(VlB200Router *router, int on);
VL_EXPORT int vlb200_router_logits(VlB200Router *router, float const *data, vl_size numData,
                                   float *logits, void *stream);
/* Top-m candidates (numData x m int, descending logits, ties: lowest index)
 * and their predicted softmax mass (numData floats) of rows `data`, device
 * arrays.  fused = 1: selected in the last dense layer's epilogue (tensor-core
 * inference, m <= 16, numClusters >= 32), else by the selection kernel on
 * the logits; both are what vlb200_router_posteriors uses. */
VL_EXPORT int vlb200_router_candidates(VlB200Router *router, float const *data, vl_size numData, vl_size m,
                                       int *candidates, float *mass, int fused, void *stream);
/* Router used by VLB200_PREC_BF16_ROUTER calls (not owned; NULL clears). */
VL_EXPORT int vlb200_router_set_default(VlB200Router *router, vl_size m, float threshold);

/* Fisher encoding of one image that allocates nothing.  No counterpart in
 * the reference: it exists for callers that cannot allocate device memory on
 * the call path (services that forbid allocation after start-up, loops that
 * cannot accept cudaMalloc's implicit device synchronisation, hosts with a
 * fixed memory budget).  The caller passes inputs and outputs as device pointers, as for
 * vlb200_fisher_encode_device; the scratch is a fixed 8 MiB device array
 * inside the library, held by every GPU that loads it until the process
 * exits.  Limits: numData <= 4096, numClusters <= 256, dimension <= 128;
 * larger requests fail with VL_ERR_BAD_ARG.  Arithmetic: the exact fp32
 * path (VLB200_PREC_EXACT).  numTerms: one uint64 in device memory, or NULL.
 * stream: a cudaStream_t; NULL is the legacy default stream.  The first call
 * on a device looks up the array's device address (cudaGetSymbolAddress), so
 * make that first call before any stream capture.  All calls share the one
 * array: calls that overlap on the GPU (on different streams, or from
 * different threads) race and must be serialised by the caller. */
VL_EXPORT int vlb200_fisher_encode_noalloc(float *enc, float const *means, vl_size dimension,
                                           vl_size numClusters, float const *covariances,
                                           float const *priors, float const *data,
                                           vl_size numData, int flags, vl_uint64 *numTerms,
                                           void *stream);

/* ------------------------------------------------------ failure checks
 * No reference counterpart.  Every wait of the library's tcgen05 kernels on
 * an mbarrier is bounded (2 s): a wait that expires records a code in the
 * launch's error word, raises the block's abort flag so that every role
 * leaves its loop and TMEM is freed, and the host raises VL_ERR_BAD_ARG with
 * "gave up waiting (code N)".  vlb200_selftest_bounded_wait runs that
 * mechanism on a barrier that nothing arrives on, with a wait limit of
 * limit_ms (0 < limit_ms <= 1000): it returns VL_ERR_BAD_ARG with the
 * message of an expired wait (code 99), and the CUDA context stays usable.
 * vlb200_debug_fail_allocations(n) makes the library's next n device
 * allocations fail as a failed cudaMalloc does (VL_ERR_ALLOC, the call
 * returns its error sentinel); 0 clears it. */
VL_EXPORT int vlb200_selftest_bounded_wait(double limit_ms);
VL_EXPORT void vlb200_debug_fail_allocations(vl_size n);

#endif /* VLB200_H */
