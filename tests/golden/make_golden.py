"""Generate the golden fixtures in this directory from VLFeat's own CPU code.

Run where the reference sources exist:

    make -C oracle ref && python tests/golden/make_golden.py

Every output comes from ``oracle/_ref/libvl_ref.so`` (the reference compiled
from its own sources by ``oracle/Makefile``) through VLFeat's C API, run with
one thread so the M-step merge order (vl/gmm.c:1152-1166) is fixed.  Inputs are
seeded and stored beside the outputs, so the tests need neither the reference
nor the generators.  The reference ships no golden vectors of its own; the
Fisher known-answer case restates the setup of toolbox/xtest/vl_test_fisher.m:9-20
(D=5, N=21, K=3, unit variances, uniform priors) with seeded NumPy data.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import (FLAG_FAST, FLAG_IMPROVED, FLAG_NORMALIZED,  # noqa: E402
                           FLAG_SQUARE_ROOT, Reference, VL_GMM_KMEANS)
from vlfeat_b200 import workloads as W  # noqa: E402

FLAG_SETS = [0, FLAG_SQUARE_ROOT, FLAG_NORMALIZED, FLAG_IMPROVED, FLAG_IMPROVED | FLAG_FAST, FLAG_FAST]


def rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def fisher_kat(ref, out):
    r = rng(1)
    D, N, K = 5, 21, 3
    x = r.standard_normal((N, D))
    mu = r.standard_normal((K, D))
    cv = np.ones((K, D))
    pr = np.full(K, 1.0 / K)
    out.update(kat_data=x, kat_means=mu, kat_covs=cv, kat_priors=pr)
    for dt, tag in ((np.float32, "f"), (np.float64, "d")):
        for fl in FLAG_SETS:
            enc, nt = ref.fisher(x.astype(dt), mu.astype(dt), cv.astype(dt), pr.astype(dt), fl)
            out[f"kat_enc_{tag}_{fl}"] = enc
            out[f"kat_nterms_{tag}_{fl}"] = np.int64(nt)


def posteriors_case(ref, out):
    D, N, K = 16, 500, 8
    x = W.mixture_data(N, D, K, seed=11)
    pr, mu, cv = W.custom_init(x, K, seed=12)
    pr = rng(13).dirichlet(np.ones(K))
    pr[3] = 5e-7  # below the 1e-6 prior floor: log-weight -inf (vl/gmm.c:746-747)
    pr /= pr.sum()
    out.update(post_data=x, post_priors=pr, post_means=mu.astype(np.float64), post_covs=cv.astype(np.float64))
    for dt, tag in ((np.float32, "f"), (np.float64, "d")):
        q, ll = ref.posteriors(x.astype(dt), pr.astype(dt), mu.astype(dt), cv.astype(dt))
        out[f"post_q_{tag}"] = q
        out[f"post_ll_{tag}"] = np.float64(ll)


def em_case(ref, out):
    """EM with an initial mean far from the data, so that mode empties and the
    restart path (vl/gmm.c:814-999) fires.  Snapshots after t = 0..T
    iterations come from separate vl_gmm_cluster calls with maxNumIterations = t
    from the same custom initialisation (exact, restarts included)."""
    D, N, K, T = 24, 3000, 12, 8
    x = W.mixture_data(N, D, 10, seed=21)
    pr, mu, cv = W.custom_init(x, K, seed=22)
    mu = mu.astype(np.float64)
    mu[5] = mu[5] + 60.0  # far outlier mean -> empty mode -> restart at iteration 2
    cv = cv.astype(np.float64)
    pr = pr.astype(np.float64)
    lb = np.full(D, 1e-3)
    out.update(em_data=x, em_priors0=pr, em_means0=mu, em_covs0=cv, em_lb=lb)
    out["em_T"] = np.int64(T)
    for dt, tag in ((np.float32, "f"), (np.float64, "d")):
        lls, P, M, S = [], [], [], []
        for t in range(T + 1):
            r = ref.em(x.astype(dt), pr.astype(dt), mu.astype(dt), cv.astype(dt), lb, t,
                       want_posteriors=(t == T))
            lls.append(r["ll"])
            P.append(r["priors"])
            M.append(r["means"])
            S.append(r["covs"])
            if t == T:
                out[f"em_post_{tag}"] = r["posteriors"]
        out[f"em_ll_{tag}"] = np.array(lls)
        out[f"em_priors_{tag}"] = np.stack(P)
        out[f"em_means_{tag}"] = np.stack(M)
        out[f"em_covs_{tag}"] = np.stack(S)


def fv_case(ref, out):
    D, K, N = 32, 16, 400
    pr, mu, cv = W.fv_gmm(K, D, seed=31, dtype=np.float64)
    pr[2] = 3e-7  # component skipped by the encoder (vl/fisher.c:436)
    pr /= pr.sum()
    x = W.pca_like(N, D, seed=32)
    out.update(fv_data=x, fv_priors=pr, fv_means=mu, fv_covs=cv)
    for dt, tag in ((np.float32, "f"), (np.float64, "d")):
        for fl in FLAG_SETS:
            enc, nt = ref.fisher(x.astype(dt), mu.astype(dt), cv.astype(dt), pr.astype(dt), fl)
            out[f"fv_enc_{tag}_{fl}"] = enc
            out[f"fv_nterms_{tag}_{fl}"] = np.int64(nt)


def edge_cases(ref, out):
    D, K = 7, 5
    pr, mu, cv = W.fv_gmm(K, D, seed=41, dtype=np.float64)
    x = W.pca_like(3, D, seed=42)
    out.update(edge_priors=pr, edge_means=mu, edge_covs=cv, edge_data=x)
    for dt, tag in ((np.float32, "f"), (np.float64, "d")):
        for n in (0, 1, 3):
            enc, nt = ref.fisher(x[:n].astype(dt), mu.astype(dt), cv.astype(dt), pr.astype(dt), FLAG_IMPROVED)
            out[f"edge_enc_{tag}_n{n}"] = enc
            out[f"edge_nterms_{tag}_n{n}"] = np.int64(nt)
        # K = 1 and D = 1
        enc, nt = ref.fisher(x.astype(dt), mu[:1].astype(dt), cv[:1].astype(dt), np.ones(1, dt), FLAG_IMPROVED)
        out[f"edge_enc_{tag}_k1"] = enc
        enc, nt = ref.fisher(x[:, :1].copy().astype(dt), mu[:, :1].copy().astype(dt), cv[:, :1].copy().astype(dt),
                             pr.astype(dt), FLAG_IMPROVED)
        out[f"edge_enc_{tag}_d1"] = enc


def rand_case(ref, out):
    """VlGMMRand initialisation (vl/gmm.c:1416-1443) from a seeded thread
    generator: the first MT19937 draws, then vl_gmm_cluster with Rand
    initialisation, without EM (max iterations 0) and with 5 EM iterations.
    The distances of k-means++ follow the reference's SIMD kernel for this host
    (recorded as rand_lanes)."""
    ref.seed(2024)
    r = ref.lib.vl_get_rand()
    out["rng_seed"] = np.int64(2024)
    out["rng_seq"] = np.array([ref.lib.vl_rand_uint32(r) for _ in range(1500)], np.uint32)
    out["rand_lanes"] = np.int64(ref.distance_lanes())
    cases = {"small": (rng(41).standard_normal((300, 13)) * 3.0, 7, 301),
             "mix": (W.mixture_data(5000, 64, 32, seed=42), 32, 302)}
    for name, (x, K, seed) in cases.items():
        out[f"rand_{name}_data"] = x
        out[f"rand_{name}_K"] = np.int64(K)
        out[f"rand_{name}_seed"] = np.int64(seed)
        for dt, tag in ((np.float32, "f"), (np.float64, "d")):
            for T in (0, 5):
                res = ref.rand_init(x.astype(dt), K, seed, max_iter=T, lb=1e-4)
                for k in ("means", "covs", "priors"):
                    out[f"rand_{name}_{tag}_t{T}_{k}"] = res[k]
                out[f"rand_{name}_{tag}_t{T}_ll"] = np.float64(res["ll"])


def vlad_case(ref, out):
    """VLAD encodings (vl/vlad.c:163-242) for every combination of the four
    flags: hard assignments to the nearest mean with one component left empty
    (mass 0), soft assignments with zeroed and negative weights (only positive
    weights count, vl/vlad.c:182), and an image without descriptors."""
    r = rng(51)
    x = W.mixture_data(400, 24, 10, seed=52)
    mu = x[r.choice(400, 10, replace=False)] + 0.1 * r.standard_normal((10, 24))
    d2 = ((x[:, None, :] - mu[None]) ** 2).sum(2)
    d2[:, 4] = np.inf
    hard = np.zeros((400, 10))
    hard[np.arange(400), d2.argmin(1)] = 1.0
    xs = r.standard_normal((300, 40)) * 2.0
    mus = r.standard_normal((12, 40))
    soft = r.dirichlet(np.ones(12) * 0.5, 300)
    soft[soft < 0.02] = 0.0
    soft[::11, 3] = -0.25
    cases = {"hard": (x, mu, hard), "soft": (xs, mus, soft),
             "empty": (np.zeros((0, 6)), r.standard_normal((3, 6)), np.zeros((0, 3)))}
    for name, (cx, cm, ca) in cases.items():
        out.update({f"vlad_{name}_data": cx, f"vlad_{name}_means": cm, f"vlad_{name}_assign": ca})
        for dt, tag in ((np.float32, "f"), (np.float64, "d")):
            for fl in range(16):
                out[f"vlad_{name}_enc_{tag}_{fl}"] = ref.vlad(cx.astype(dt), cm.astype(dt), ca.astype(dt), fl)


def kmeans_data(name):
    """Inputs of the KMeans-initialisation cases (regenerated by the tests from
    the same seeds): uniform rows, an integer grid (many equal distances and
    split values), 25 distinct rows repeated (duplicate seeds, constant
    leaves), too few rows for a full search (N/4 < K: the comparison budget
    cuts the search), a mixture, more than 1024 centres (the kd-tree samples
    variances with random draws), SIFT-sized rows, and the edge shapes K = 1,
    N = K and D = 1."""
    if name == "small":
        return rng(61).random((400, 5)), 8, 611
    if name == "grid":
        return rng(62).integers(0, 4, (500, 3)).astype(np.float64), 16, 621
    if name == "dup":
        base = rng(63).random((25, 5))
        return base[rng(631).integers(0, 25, 200)], 30, 632
    if name == "trunc":
        return rng(64).random((60, 4)), 20, 641
    if name == "mix":
        return W.mixture_data(20000, 16, 64, seed=65, dtype=np.float64), 64, 651
    if name == "wide":
        return W.mixture_data(6000, 6, 300, seed=66, dtype=np.float64), 1100, 661
    if name == "sift":
        return W.mixture_data(50000, 80, 256, seed=67, dtype=np.float64), 256, 671
    if name == "k1":  # one centre: a one-leaf tree
        return rng(68).random((40, 3)), 1, 681
    if name == "nk":  # as many rows as centres: every row becomes a centre
        return rng(69).random((12, 2)), 12, 691
    if name == "d1":  # one dimension
        return rng(70).random((300, 1)), 5, 701
    raise KeyError(name)


KMEANS_CASES = {"small": ("f", "d"), "grid": ("f",), "dup": ("f",), "trunc": ("f",), "mix": ("f", "d"),
                "wide": ("f",), "sift": ("f",), "k1": ("f",), "nk": ("f", "d"), "d1": ("f",)}


def kmeans_case(ref, out):
    """VlGMMKMeans initialisation (vl/gmm.c:1315-1370) from a seeded thread
    generator through vl_gmm_init_with_kmeans: the k-means assignment of every
    row, the generator's next draw, the one-hot M-step's parameters; and
    vl_gmm_cluster with KMeans initialisation and 5 EM iterations for two cases."""
    for name, tags in KMEANS_CASES.items():
        x, K, seed = kmeans_data(name)
        for tag in tags:
            dt = np.float32 if tag == "f" else np.float64
            res = ref.kmeans_init(x.astype(dt), K, seed)
            out[f"km_{name}_{tag}_assign"] = res["assign"].astype(np.int32)
            out[f"km_{name}_{tag}_next"] = np.uint32(res["next_draw"])
            for k in ("means", "covs", "priors"):
                out[f"km_{name}_{tag}_{k}"] = res[k]
            if name in ("small", "mix"):
                em = ref.rand_init(x.astype(dt), K, seed, max_iter=5, lb=1e-4, init=VL_GMM_KMEANS)
                out[f"km_{name}_{tag}_t5_ll"] = np.float64(em["ll"])
                for k in ("means", "covs", "priors"):
                    out[f"km_{name}_{tag}_t5_{k}"] = em[k]


def main():
    ref = Reference(threads=1)
    out: dict = {}
    fisher_kat(ref, out)
    posteriors_case(ref, out)
    em_case(ref, out)
    fv_case(ref, out)
    edge_cases(ref, out)
    rand_case(ref, out)
    vlad_case(ref, out)
    kmeans_case(ref, out)
    path = os.path.join(HERE, "golden.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
