/* gmm_fisher_drop_in.c -- a VLFeat client program for the drop-in check.
 *
 * Written against VLFeat's public C API only (vl/gmm.h, vl/fisher.h,
 * vl/vlad.h, vl/random.h, vl/generic.h), in the manner of the reference's
 * own smoke driver src/test_gmm.c:23-191: data drawn with vl_rand_real3 from
 * a generator seeded with 49000, a VlGMM fitted with the Custom and the Rand
 * initialisations, vl_gmm_cluster, the getters, then vl_fisher_encode
 * (VL_FISHER_FLAG_IMPROVED) and vl_vlad_encode of 2,000 fresh points.  The
 * KMeans initialisation of src/test_gmm.c is left out: it goes through the
 * vl_kmeans_* API, which the drop-in does not export.
 *
 * The same source is compiled against this library's include/ twice: once
 * linked with the GPU library and once with VLFeat's own CPU library built
 * from the reference's sources; the two runs' outputs are then compared.
 *
 * Usage: gmm_fisher_drop_in OUT.bin
 * OUT.bin: for each case (float custom, float rand, double custom, double
 * rand) in that order, as doubles: the log-likelihood, means (K x D),
 * covariances (K x D), priors (K), posteriors (N x K), the Fisher vector
 * (2 K D), its numTerms, the VLAD vector (K D). */
#include <stdio.h>
#include <stdlib.h>

#include <vl/fisher.h>
#include <vl/generic.h>
#include <vl/gmm.h>
#include <vl/random.h>
#include <vl/vlad.h>

enum { kN = 1000, kD = 3, kK = 20, kIters = 5, kNf = 2000 };

static FILE *out;

static void put(double v) { fwrite(&v, sizeof v, 1, out); }

static void put_array(void const *p, vl_type t, vl_size n) {
  vl_size i;
  for (i = 0; i < n; ++i) put(t == VL_TYPE_FLOAT ? (double)((float const *)p)[i] : ((double const *)p)[i]);
}

static double get(void const *p, vl_type t, vl_size i) {
  return t == VL_TYPE_FLOAT ? (double)((float const *)p)[i] : ((double const *)p)[i];
}

static void set(void *p, vl_type t, vl_size i, double v) {
  if (t == VL_TYPE_FLOAT) ((float *)p)[i] = (float)v;
  else ((double *)p)[i] = v;
}

static void run(vl_type t, VlGMMInitialization init) {
  vl_size const ts = t == VL_TYPE_FLOAT ? sizeof(float) : sizeof(double);
  VlRand rand;
  VlGMM *gmm;
  void *data = vl_malloc(ts * kN * kD), *fvdata = vl_malloc(ts * kNf * kD);
  void *enc = vl_malloc(ts * 2 * kD * kK), *venc = vl_malloc(ts * kD * kK);
  void *assign = vl_malloc(ts * kNf * kK);
  vl_size i, nterms;
  double ll;

  vl_rand_init(&rand);
  vl_rand_seed(&rand, 49000);
  for (i = 0; i < kN * kD; ++i) set(data, t, i, vl_rand_real3(&rand));
  gmm = vl_gmm_new(t, kD, kK);
  if (init == VlGMMCustom) {
    void *m = vl_malloc(ts * kK * kD), *s = vl_malloc(ts * kK * kD), *w = vl_malloc(ts * kK);
    vl_size c, d;
    for (c = 0; c < kK; ++c) {
      for (d = 0; d < kD; ++d) {
        set(m, t, c * kD + d, vl_rand_real3(&rand));
        set(s, t, c * kD + d, vl_rand_real3(&rand));
      }
      set(w, t, c, vl_rand_real3(&rand));
    }
    vl_gmm_set_initialization(gmm, VlGMMCustom);
    vl_gmm_set_priors(gmm, w);
    vl_gmm_set_covariances(gmm, s);
    vl_gmm_set_means(gmm, m);
    vl_free(m);
    vl_free(s);
    vl_free(w);
  } else {
    /* The Rand initialisation draws from the calling thread's generator. */
    vl_rand_seed(vl_get_rand(), 1234);
    vl_gmm_set_initialization(gmm, VlGMMRand);
  }
  vl_gmm_set_max_num_iterations(gmm, kIters);
  vl_gmm_set_num_repetitions(gmm, 1);
  vl_gmm_set_verbosity(gmm, 0);
  vl_gmm_set_covariance_lower_bound(gmm, 0.000001);
  ll = vl_gmm_cluster(gmm, data, kN);

  put(ll);
  put_array(vl_gmm_get_means(gmm), t, kK * kD);
  put_array(vl_gmm_get_covariances(gmm), t, kK * kD);
  put_array(vl_gmm_get_priors(gmm), t, kK);
  put_array(vl_gmm_get_posteriors(gmm), t, kN * kK);

  for (i = 0; i < kNf * kD; ++i) set(fvdata, t, i, vl_rand_real3(&rand));
  nterms = vl_fisher_encode(enc, t, vl_gmm_get_means(gmm), kD, kK, vl_gmm_get_covariances(gmm),
                            vl_gmm_get_priors(gmm), fvdata, kNf, VL_FISHER_FLAG_IMPROVED);
  put_array(enc, t, 2 * kK * kD);
  put((double)nterms);

  /* Hard assignments to the nearest mean, then VLAD (src/test_gmm.c:192-214
   * fills the assignments with random draws instead). */
  for (i = 0; i < kNf; ++i) {
    vl_size c, d, best = 0;
    double bestd = 1e300;
    for (c = 0; c < kK; ++c) {
      double s = 0;
      for (d = 0; d < kD; ++d) {
        double x = get(fvdata, t, i * kD + d), mu = get(vl_gmm_get_means(gmm), t, c * kD + d);
        s += (x - mu) * (x - mu);
      }
      if (s < bestd) {
        bestd = s;
        best = c;
      }
    }
    for (c = 0; c < kK; ++c) set(assign, t, i * kK + c, (double)(c == best));
  }
  vl_vlad_encode(venc, t, vl_gmm_get_means(gmm), kD, kK, fvdata, kNf, assign, 0);
  put_array(venc, t, kK * kD);

  vl_gmm_delete(gmm);
  vl_free(data);
  vl_free(fvdata);
  vl_free(enc);
  vl_free(venc);
  vl_free(assign);
}

int main(int argc, char **argv) {
  if (argc != 2) {
    fprintf(stderr, "usage: %s OUT.bin\n", argv[0]);
    return 2;
  }
  out = fopen(argv[1], "wb");
  if (!out) return 1;
  vl_set_num_threads(0); /* the default number of threads, as src/test_gmm.c:57 */
  run(VL_TYPE_FLOAT, VlGMMCustom);
  run(VL_TYPE_FLOAT, VlGMMRand);
  run(VL_TYPE_DOUBLE, VlGMMCustom);
  run(VL_TYPE_DOUBLE, VlGMMRand);
  fclose(out);
  if (vl_get_last_error()) {
    fprintf(stderr, "last error: %s\n", vl_get_last_error_message());
    return 1;
  }
  return 0;
}
