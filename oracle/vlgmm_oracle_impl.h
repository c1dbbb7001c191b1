/* CPU restatement of VLFeat's diagonal-GMM EM and Fisher-vector encoding.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle the GPU library is
 * checked against; it is never linked into, loaded by or called from the
 * product library.  It is included twice by vlgmm_oracle.c, once with
 * REAL=float (suffix _f) and once with REAL=double (suffix _d), mirroring how
 * the reference instantiates vl/gmm.c and vl/fisher.c for both types
 * (vl/gmm.c:1446-1464, vl/fisher.c:490-508).
 *
 * Every function cites the reference lines whose algorithm it restates.  The
 * arithmetic types follow the reference: values stored in REAL, log/exp taken
 * in double, log-likelihood accumulated in double.  Summation orders are
 * plain sequential loops (the reference's AVX kernels use 8-lane partial sums,
 * vl/mathop_avx.c:113-169), so float results agree with the reference to
 * rounding, not bit for bit.  Parallel loops only split independent outputs,
 * so every result is deterministic.
 */

#define ORC_CAT2(a, b) a##b
#define ORC_CAT(a, b) ORC_CAT2(a, b)
#define ORC(name) ORC_CAT(name, SFX)

/* E-step: posteriors and log-likelihood.
 * Restates vl_get_gmm_data_posteriors (vl/gmm.c:711-798):
 *   log w_k = log pi_k, or -inf when pi_k < 1e-6           (gmm.c:746-750)
 *   logdet_k = sum_d log sigma2_kd, inv_kd = 1/sigma2_kd    (gmm.c:751-755)
 *   p_ik = log w_k - (D/2) log 2pi - logdet_k/2 - maha/2   (gmm.c:767-773)
 *   q_ik = exp(p_ik - max_k p) / sum                        (gmm.c:778-790)
 *   LL  = sum_i (log sum + max)                            (gmm.c:786)  */
double ORC(orc_posteriors_)(REAL *post, size_t K, size_t N,
                            const REAL *priors, const REAL *means, size_t D,
                            const REAL *covs, const REAL *data)
{
  REAL *logw = (REAL *)malloc(sizeof(REAL) * (K ? K : 1));
  REAL *logdet = (REAL *)malloc(sizeof(REAL) * (K ? K : 1));
  REAL *inv = (REAL *)malloc(sizeof(REAL) * (K * D > 0 ? K * D : 1));
  double *rowll = (double *)malloc(sizeof(double) * (N ? N : 1));
  REAL halfDimLog2Pi = (REAL)((D / 2.0) * log(2.0 * ORC_PI));
  double LL = 0;
  long long i, k;

  for (k = 0; k < (long long)K; ++k) {
    REAL acc = 0;
    size_t d;
    logw[k] = (double)priors[k] < 1e-6 ? (REAL)(-INFINITY) : (REAL)log(priors[k]);
    for (d = 0; d < D; ++d) {
      acc += (REAL)log(covs[k * D + d]);
      inv[k * D + d] = (REAL)1.0 / covs[k * D + d];
    }
    logdet[k] = acc;
  }

#pragma omp parallel for schedule(static) private(k)
  for (i = 0; i < (long long)N; ++i) {
    const REAL *x = data + (size_t)i * D;
    REAL *q = post + (size_t)i * K;
    REAL mx = (REAL)(-INFINITY), sum = 0;
    for (k = 0; k < (long long)K; ++k) {
      const REAL *mu = means + (size_t)k * D;
      const REAL *iv = inv + (size_t)k * D;
      REAL maha = 0;
      size_t d;
      for (d = 0; d < D; ++d) {
        REAL diff = x[d] - mu[d];
        maha += diff * diff * iv[d];
      }
      q[k] = (REAL)(logw[k] - halfDimLog2Pi - 0.5 * logdet[k] - 0.5 * maha);
      if (q[k] > mx) mx = q[k];
    }
    for (k = 0; k < (long long)K; ++k) {
      q[k] = (REAL)exp((double)(q[k] - mx));
      sum += q[k];
    }
    rowll[i] = log((double)sum) + (double)mx;
    for (k = 0; k < (long long)K; ++k) q[k] /= sum;
  }
  for (i = 0; i < (long long)N; ++i) LL += rowll[i];

  free(logw); free(logdet); free(inv); free(rowll);
  return LL;
}

/* Lower bounds on the variances.  Restates _vl_gmm_apply_bounds_
 * (vl/gmm.c:1005-1030): sigma2_kd = lb_d wherever sigma2_kd < lb_d. */
void ORC(orc_apply_bounds_)(REAL *covs, size_t K, size_t D, const double *lb)
{
  size_t k, d;
  for (k = 0; k < K; ++k)
    for (d = 0; d < D; ++d)
      if (covs[k * D + d] < lb[d]) covs[k * D + d] = (REAL)lb[d];
}

/* M-step.  Restates _vl_gmm_maximization_ (vl/gmm.c:1036-1213):
 *   skip q_ik < 1e-2/K                                  (gmm.c:1099)
 *   mass_k = sum q, S1 = sum q x, S2 = sum q (x - mu_old)^2   (1101-1148)
 *   if mass_k >= 1e-6/K: mu = S1/mass, sigma2 = S2/mass - (mu - mu_old)^2
 *                                                      (1169-1192)
 *   bounds (1194); pi = mass / max(sum mass, 1e-12)     (1196-1205)
 * The loop over components is parallel; each component's sums run over the
 * data in index order, so the result does not depend on the thread count. */
void ORC(orc_maximization_)(REAL *priors, REAL *means, REAL *covs,
                            const REAL *post, const REAL *data,
                            size_t N, size_t D, size_t K, const double *lb)
{
  REAL *oldMeans = (REAL *)malloc(sizeof(REAL) * (K * D > 0 ? K * D : 1));
  long long k;
  memcpy(oldMeans, means, sizeof(REAL) * K * D);

#pragma omp parallel for schedule(dynamic)
  for (k = 0; k < (long long)K; ++k) {
    REAL mass = 0;
    REAL *mu = means + (size_t)k * D, *s2 = covs + (size_t)k * D;
    const REAL *mo = oldMeans + (size_t)k * D;
    size_t i, d;
    const double thr = 1e-2 / (double)K;
    for (d = 0; d < D; ++d) { mu[d] = 0; s2[d] = 0; }
    for (i = 0; i < N; ++i) {
      REAL p = post[i * K + (size_t)k];
      const REAL *x = data + i * D;
      if ((double)p < thr) continue;
      mass += p;
      for (d = 0; d < D; ++d) {
        REAL diff = x[d] - mo[d];
        mu[d] += p * x[d];
        s2[d] += p * (diff * diff);
      }
    }
    priors[k] = mass;
    if ((double)mass >= 1e-6 / (double)K) {
      for (d = 0; d < D; ++d) {
        REAL diff;
        mu[d] /= mass;
        s2[d] /= mass;
        diff = mu[d] - mo[d];
        s2[d] -= diff * diff;
      }
    }
  }

  ORC(orc_apply_bounds_)(covs, K, D, lb);
  {
    REAL sum = 0;
    size_t kk;
    for (kk = 0; kk < K; ++kk) sum += priors[kk];
    if ((double)sum < 1e-12) sum = (REAL)1e-12;
    for (kk = 0; kk < K; ++kk) priors[kk] /= sum;
  }
  free(oldMeans);
}

/* Empty-mode restart.  Restates _vl_gmm_restart_empty_modes_
 * (vl/gmm.c:814-999): masses from all posteriors (835-844); a mode with
 * mass < 1e-2 * max(1, N/K) (888-889) is re-seeded by splitting the mode with
 * the largest entropy contribution pi_j (D/2 (1 + log 2pi) + sum log sigma/2
 * - log pi_j) (920-939) along its largest-variance dimension (958-966), moving
 * posteriors on either side of the mean (969-989) and re-running the M-step
 * (994-995).  Returns the number of split modes (the reference returns 0). */
size_t ORC(orc_restart_empty_modes_)(REAL *priors, REAL *means, REAL *covs,
                                     REAL *post, const REAL *data,
                                     size_t N, size_t D, size_t K, const double *lb)
{
  REAL *mass;
  size_t i, k, nsplit = 0;
  long long icl;
  if (K <= 1) return 0;
  mass = (REAL *)calloc(K, sizeof(REAL));
  for (i = 0; i < N; ++i)
    for (k = 0; k < K; ++k) mass[k] += post[i * K + k];

  for (icl = 0; icl < (long long)K; ++icl) {
    double best_score = -INFINITY, cutoff = 1e-2 * ((double)N / (double)K > 1.0 ? (double)N / (double)K : 1.0);
    long long j, best = -1, bestDim = -1;
    double bestVar = -INFINITY;
    size_t d;
    REAL cut;
    if ((double)mass[icl] >= cutoff) continue;
    for (j = 0; j < (long long)K; ++j) {
      double score;
      if ((double)priors[j] < 1e-6) continue;
      score = 0.5 * (double)D * (1.0 + log(2 * ORC_PI));
      for (d = 0; d < D; ++d) score += 0.5 * log((double)covs[(size_t)j * D + d]);
      score = (double)priors[j] * (score - log((double)priors[j]));
      if (score > best_score) { best_score = score; best = j; }
    }
    if (best == icl || best < 0) continue;
    for (d = 0; d < D; ++d) {
      double v = (double)covs[(size_t)best * D + d];
      if (v > bestVar) { bestVar = v; bestDim = (long long)d; }
    }
    cut = means[(size_t)best * D + (size_t)bestDim];
    for (i = 0; i < N; ++i) {
      REAL p = post[i * K + (size_t)best];
      REAL q = post[i * K + (size_t)icl];
      if (data[i * D + (size_t)bestDim] < cut) {
        post[i * K + (size_t)icl] = p + q;
        post[i * K + (size_t)best] = 0;
      } else {
        post[i * K + (size_t)icl] = 0;
        post[i * K + (size_t)best] = p + q;
      }
    }
    ORC(orc_maximization_)(priors, means, covs, post, data, N, D, K, lb);
    nsplit++;
  }
  free(mass);
  return nsplit;
}

/* EM loop.  Restates _vl_gmm_em_ (vl/gmm.c:1220-1308): bounds on the initial
 * variances (1233); then E-step, stop when iteration >= maxIter (1270) or when
 * iteration > 0 and |(LL - LLprev)/LL| < 1e-5 (1279-1286), restart empty modes
 * from iteration 2 on (1292-1299), M-step (1304).  So maxIter iterations run
 * maxIter M-steps and maxIter+1 E-steps.  Outputs: final LL; *iters = number
 * of M-steps run; *restarts = total modes split. */
double ORC(orc_em_)(REAL *priors, REAL *means, REAL *covs, REAL *post,
                    const REAL *data, size_t N, size_t D, size_t K,
                    const double *lb, size_t maxIter,
                    size_t *iters, size_t *restarts, double *llTrace)
{
  double prevLL = -INFINITY, LL = -INFINITY;
  size_t it, nrest = 0;
  ORC(orc_apply_bounds_)(covs, K, D, lb);
  for (it = 0;; ++it) {
    double eps;
    LL = ORC(orc_posteriors_)(post, K, N, priors, means, D, covs, data);
    if (llTrace) llTrace[it] = LL;
    if (it >= maxIter) break;
    eps = fabs((LL - prevLL) / LL);
    if (it > 0 && eps < 1e-5) break;
    prevLL = LL;
    if (it > 1) nrest += ORC(orc_restart_empty_modes_)(priors, means, covs, post, data, N, D, K, lb);
    ORC(orc_maximization_)(priors, means, covs, post, data, N, D, K, lb);
  }
  if (iters) *iters = it;
  if (restarts) *restarts = nrest;
  return LL;
}

/* Global per-dimension variance with the N-1 denominator.  Restates
 * _vl_gmm_compute_init_sigma_ (vl/gmm.c:1376-1413). */
void ORC(orc_global_variance_)(REAL *var, const REAL *data, size_t N, size_t D)
{
  size_t i, d;
  for (d = 0; d < D; ++d) var[d] = 0;
  if (N <= 1) return;
  for (d = 0; d < D; ++d) {
    REAL m = 0, v = 0;
    for (i = 0; i < N; ++i) m += data[i * D + d];
    m /= (REAL)N;
    for (i = 0; i < N; ++i) { REAL t = data[i * D + d] - m; v += t * t; }
    var[d] = v / (REAL)(N - 1);
  }
}

/* Fisher vector.  Restates _vl_fisher_encode_ (vl/fisher.c:363-488):
 *   s_kd = sqrt(1/sigma2_kd)                               (386-390)
 *   q = E-step posteriors                                  (392-396)
 *   FAST: one-hot at the first arg-max of each row         (398-417)
 *   for pi_k >= 1e-6 and q_ik >= 1e-6:                      (436-441)
 *     u_kd += q (x-mu) s,  v_kd += q ((x-mu)^2 s^2 - 1)       (442-447)
 *   u *= 1/(N sqrt pi), v *= 1/(N sqrt(2 pi))               (450-457)
 *   SQUARE_ROOT: sign(z) sqrt|z|; NORMALIZED: z / max(||z||, 1e-12)
 * Layout: enc = [u_1 .. u_K | v_1 .. v_K], each u_k, v_k of length D.
 * Returns the number of (i,k) terms accumulated. */
size_t ORC(orc_fisher_)(REAL *enc, const REAL *means, size_t D, size_t K,
                        const REAL *covs, const REAL *priors,
                        const REAL *data, size_t N, int flags)
{
  REAL *post = (REAL *)malloc(sizeof(REAL) * (N * K > 0 ? N * K : 1));
  REAL *sis = (REAL *)malloc(sizeof(REAL) * (K * D > 0 ? K * D : 1));
  size_t numTerms = 0, i, k, d;
  long long kk;

  memset(enc, 0, sizeof(REAL) * 2 * D * K);
  for (k = 0; k < K * D; ++k) sis[k] = (REAL)sqrt(1.0 / (double)covs[k]);
  ORC(orc_posteriors_)(post, K, N, priors, means, D, covs, data);

  if (flags & ORC_FLAG_FAST) {
    for (i = 0; i < N; ++i) {
      size_t best = 0;
      REAL bv = post[i * K];
      for (k = 1; k < K; ++k)
        if (post[i * K + k] > bv) { bv = post[i * K + k]; best = k; }
      for (k = 0; k < K; ++k) post[i * K + k] = (REAL)(k == best);
    }
  }

#pragma omp parallel for schedule(dynamic) reduction(+ : numTerms)
  for (kk = 0; kk < (long long)K; ++kk) {
    REAL *u = enc + (size_t)kk * D, *v = enc + (size_t)kk * D + K * D;
    const REAL *mu = means + (size_t)kk * D, *s = sis + (size_t)kk * D;
    size_t ii, dd;
    if ((double)priors[kk] < 1e-6) continue;
    for (ii = 0; ii < N; ++ii) {
      REAL p = post[ii * K + (size_t)kk];
      const REAL *x = data + ii * D;
      if ((double)p < 1e-6) continue;
      numTerms += 1;
      for (dd = 0; dd < D; ++dd) {
        REAL diff = (x[dd] - mu[dd]) * s[dd];
        u[dd] += p * diff;
        v[dd] += p * (diff * diff - 1);
      }
    }
    if (N > 0) {
      REAL up = (REAL)(1.0 / ((double)N * sqrt((double)priors[kk])));
      REAL vp = (REAL)(1.0 / ((double)N * sqrt(2.0 * (double)priors[kk])));
      for (dd = 0; dd < D; ++dd) { u[dd] *= up; v[dd] *= vp; }
    }
  }

  if (flags & ORC_FLAG_SQUARE_ROOT) {
    for (d = 0; d < 2 * D * K; ++d) {
      REAL z = enc[d];
      enc[d] = z >= 0 ? (REAL)sqrt((double)z) : -(REAL)sqrt((double)-z);
    }
  }
  if (flags & ORC_FLAG_NORMALIZED) {
    REAL n = 0;
    for (d = 0; d < 2 * D * K; ++d) n += enc[d] * enc[d];
    n = (REAL)sqrt((double)n);
    if ((double)n < 1e-12) n = (REAL)1e-12;
    for (d = 0; d < 2 * D * K; ++d) enc[d] /= n;
  }
  free(post); free(sis);
  return numTerms;
}

#undef ORC
#undef ORC_CAT
#undef ORC_CAT2
