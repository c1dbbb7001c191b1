"""CPU tests: the C restatement (oracle/) is pinned against the golden vectors
produced by VLFeat's own code (tests/golden/make_golden.py), and the FP64
NumPy statement of the Fisher vector pins the known-answer case the way
toolbox/xtest/vl_test_fisher.m does (absTol 1e-10 in double)."""
import os

import numpy as np
import pytest

from conftest import rel_err
from oracle.oracle import FLAG_FAST, FLAG_IMPROVED, FLAG_NORMALIZED, FLAG_SQUARE_ROOT, simple_fisher

FLAG_SETS = [0, FLAG_SQUARE_ROOT, FLAG_NORMALIZED, FLAG_IMPROVED, FLAG_IMPROVED | FLAG_FAST, FLAG_FAST]
TOL = {"f": 2e-5, "d": 1e-12}
DT = {"f": np.float32, "d": np.float64}


@pytest.mark.parametrize("tag", ["f", "d"])
@pytest.mark.parametrize("flags", FLAG_SETS)
def test_fisher_known_answer(golden, restatement, tag, flags):
    g = golden
    args = [g["kat_data"].astype(DT[tag]), g["kat_means"], g["kat_covs"], g["kat_priors"]]
    enc, nt = restatement.fisher(args[0], *[a.astype(DT[tag]) for a in args[1:]], flags)
    ref = g[f"kat_enc_{tag}_{flags}"]
    assert rel_err(enc, ref) < TOL[tag]
    assert nt == int(g[f"kat_nterms_{tag}_{flags}"])
    if tag == "d":
        s = simple_fisher(g["kat_data"], g["kat_means"], g["kat_covs"], g["kat_priors"], flags)
        assert np.max(np.abs(s - ref)) < 1e-10


@pytest.mark.parametrize("tag", ["f", "d"])
def test_posteriors(golden, restatement, tag):
    g = golden
    dt = DT[tag]
    q, ll = restatement.posteriors(g["post_data"].astype(dt), g["post_priors"].astype(dt),
                                   g["post_means"].astype(dt), g["post_covs"].astype(dt))
    assert rel_err(q, g[f"post_q_{tag}"]) < TOL[tag]
    assert abs(ll - float(g[f"post_ll_{tag}"])) <= TOL[tag] * abs(float(g[f"post_ll_{tag}"]))
    assert np.all(q[:, 3] == 0)  # prior below 1e-6 -> log-weight -inf


@pytest.mark.parametrize("tag", ["f", "d"])
def test_em_iterations(golden, restatement, tag):
    """Per-iteration parameters after t = 0..T EM iterations, restart included."""
    g = golden
    dt = DT[tag]
    T = int(g["em_T"])
    tol = {"f": 2e-4, "d": 1e-10}[tag]
    for t in range(T + 1):
        r = restatement.em(g["em_data"].astype(dt), g["em_priors0"], g["em_means0"], g["em_covs0"],
                           g["em_lb"], t)
        assert abs(r["ll"] - g[f"em_ll_{tag}"][t]) <= tol * abs(g[f"em_ll_{tag}"][t])
        for name in ("priors", "means", "covs"):
            assert rel_err(r[name], g[f"em_{name}_{tag}"][t]) < tol, (t, name)
        if t == T:
            assert r["restarts"] >= 1  # the seeded outlier mode is re-seeded
            assert rel_err(r["posteriors"], g[f"em_post_{tag}"]) < tol


@pytest.mark.parametrize("tag", ["f", "d"])
@pytest.mark.parametrize("flags", FLAG_SETS)
def test_fisher_case(golden, restatement, tag, flags):
    g = golden
    dt = DT[tag]
    enc, nt = restatement.fisher(g["fv_data"].astype(dt), g["fv_means"].astype(dt),
                                 g["fv_covs"].astype(dt), g["fv_priors"].astype(dt), flags)
    assert rel_err(enc, g[f"fv_enc_{tag}_{flags}"]) < TOL[tag]
    assert nt == int(g[f"fv_nterms_{tag}_{flags}"])
    K, D = g["fv_means"].shape
    assert np.all(enc[2 * D:3 * D] == 0) and np.all(enc[K * D + 2 * D:K * D + 3 * D] == 0)


@pytest.mark.parametrize("tag", ["f", "d"])
def test_fisher_edges(golden, restatement, tag):
    g = golden
    dt = DT[tag]
    x, mu, cv, pr = (g["edge_data"], g["edge_means"], g["edge_covs"], g["edge_priors"])
    for n in (0, 1, 3):
        enc, _ = restatement.fisher(x[:n].astype(dt), mu.astype(dt), cv.astype(dt), pr.astype(dt),
                                    FLAG_IMPROVED)
        assert rel_err(enc, g[f"edge_enc_{tag}_n{n}"]) < TOL[tag]
        if n == 0:
            assert np.all(enc == 0)
    enc, _ = restatement.fisher(x.astype(dt), mu[:1].astype(dt), cv[:1].astype(dt), np.ones(1, dt),
                                FLAG_IMPROVED)
    assert rel_err(enc, g[f"edge_enc_{tag}_k1"]) < TOL[tag]
    enc, _ = restatement.fisher(x[:, :1].copy().astype(dt), mu[:, :1].copy().astype(dt),
                                cv[:, :1].copy().astype(dt), pr.astype(dt), FLAG_IMPROVED)
    assert rel_err(enc, g[f"edge_enc_{tag}_d1"]) < TOL[tag]


def test_oracle_is_deterministic(golden, restatement):
    g = golden
    a = restatement.em(g["em_data"], g["em_priors0"], g["em_means0"], g["em_covs0"], g["em_lb"], 4)
    b = restatement.em(g["em_data"], g["em_priors0"], g["em_means0"], g["em_covs0"], g["em_lb"], 4)
    for n in ("priors", "means", "covs", "posteriors"):
        assert np.array_equal(a[n], b[n])


def test_rng_restatement(golden):
    """MT19937 restatement (oracle.MT19937) against the reference's draws
    after vl_rand_seed (vl/random.c)."""
    from oracle.oracle import MT19937
    g = MT19937(int(golden["rng_seed"]))
    assert [g.uint32() for _ in range(len(golden["rng_seq"]))] == [int(v) for v in golden["rng_seq"]]


@pytest.mark.parametrize("tag", ["f", "d"])
def test_rand_init_restatement(golden, tag):
    """VlGMMRand initialisation restated (oracle.rand_init) against the
    reference's, bit for bit: k-means++ centres, global variance, priors."""
    from oracle.oracle import MT19937, rand_init
    dt = np.float32 if tag == "f" else np.float64
    x = golden["rand_small_data"].astype(dt)
    K, seed = int(golden["rand_small_K"]), int(golden["rand_small_seed"])
    lanes = int(golden["rand_lanes"])
    if dt == np.float64:
        lanes = {8: 4, 4: 2, 1: 1}[lanes]
    o = rand_init(x, K, MT19937(seed), lanes)
    for k in ("means", "covs", "priors"):
        assert np.array_equal(o[k], golden[f"rand_small_{tag}_t0_{k}"]), k


@pytest.mark.parametrize("name,tag", [("small", "f"), ("small", "d"), ("grid", "f"), ("dup", "f"),
                                      ("trunc", "f"), ("k1", "f"), ("nk", "f"), ("nk", "d"), ("d1", "f")])
def test_kmeans_init_restatement(golden, name, tag):
    """The k-means of the KMeans initialisation restated (oracle.kmeans_init:
    seeding shuffle and duplicate test, one-tree kd-forest with its random
    draws, best-bin-first search, ordered centre sums, exact quantisation)
    against the reference's: every assignment and the generator's next draw
    equal."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from make_golden import kmeans_data
    from oracle.oracle import MT19937, kmeans_init
    x, K, seed = kmeans_data(name)
    dt = np.float32 if tag == "f" else np.float64
    lanes = int(golden["rand_lanes"])
    if dt == np.float64:
        lanes = {8: 4, 4: 2, 1: 1}[lanes]
    rng = MT19937(seed)
    o = kmeans_init(x.astype(dt), K, rng, lanes)
    assert np.array_equal(o["assign"], golden[f"km_{name}_{tag}_assign"])
    assert rng.uint32() == int(golden[f"km_{name}_{tag}_next"])


@pytest.mark.parametrize("flags", range(16))
@pytest.mark.parametrize("tag", ["f", "d"])
@pytest.mark.parametrize("name", ["hard", "soft", "empty"])
def test_vlad_restatement(golden, name, tag, flags):
    """The NumPy VLAD restatement reproduces the reference's encodings bit for
    bit: hard assignments with an empty component, soft assignments with
    zero and negative weights, and an image without descriptors."""
    from oracle.oracle import vlad
    dt = np.float32 if tag == "f" else np.float64
    x = golden[f"vlad_{name}_data"].astype(dt)
    mu = golden[f"vlad_{name}_means"].astype(dt)
    a = golden[f"vlad_{name}_assign"].astype(dt)
    want = golden[f"vlad_{name}_enc_{tag}_{flags}"]
    got = vlad(x, mu, a, flags)
    assert got.dtype == want.dtype
    np.testing.assert_array_equal(got.view(np.uint8), want.view(np.uint8))
