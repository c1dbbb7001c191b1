"""GPU parity of the exact (CUDA-core) path through the C-ABI against VLFeat's
own results (golden vectors) and the C restatement.

Tolerances: double results within 1e-10 relative of the reference's double
code; float results within 2e-5 relative of the reference's float code (the
reference's float results are themselves ~1e-6 from FP64)."""
import numpy as np
import pytest

from conftest import rel_err
from oracle.oracle import FLAG_FAST, FLAG_IMPROVED, FLAG_NORMALIZED, FLAG_SQUARE_ROOT

pytestmark = pytest.mark.gpu

FLAG_SETS = [0, FLAG_SQUARE_ROOT, FLAG_NORMALIZED, FLAG_IMPROVED, FLAG_IMPROVED | FLAG_FAST, FLAG_FAST]
DT = {"f": np.float32, "d": np.float64}
TOL = {"f": 2e-5, "d": 1e-10}


@pytest.fixture(autouse=True)
def exact_mode(vl):
    vl.set_precision("exact")
    yield


@pytest.mark.parametrize("tag", ["f", "d"])
@pytest.mark.parametrize("flags", FLAG_SETS)
def test_fisher_known_answer(vl, golden, tag, flags):
    g = golden
    dt = DT[tag]
    enc, nt = vl.fisher_encode(g["kat_data"].astype(dt), g["kat_means"].astype(dt),
                               g["kat_covs"].astype(dt), g["kat_priors"].astype(dt), flags)
    assert rel_err(enc, g[f"kat_enc_{tag}_{flags}"]) < TOL[tag]
    assert nt == int(g[f"kat_nterms_{tag}_{flags}"])


@pytest.mark.parametrize("tag", ["f", "d"])
@pytest.mark.parametrize("flags", FLAG_SETS)
def test_fisher_case(vl, golden, tag, flags):
    g = golden
    dt = DT[tag]
    enc, nt = vl.fisher_encode(g["fv_data"].astype(dt), g["fv_means"].astype(dt),
                               g["fv_covs"].astype(dt), g["fv_priors"].astype(dt), flags)
    assert rel_err(enc, g[f"fv_enc_{tag}_{flags}"]) < TOL[tag]
    assert nt == int(g[f"fv_nterms_{tag}_{flags}"])


@pytest.mark.parametrize("tag", ["f", "d"])
def test_fisher_edges(vl, golden, tag):
    g = golden
    dt = DT[tag]
    x, mu, cv, pr = g["edge_data"], g["edge_means"], g["edge_covs"], g["edge_priors"]
    for n in (0, 1, 3):
        enc, _ = vl.fisher_encode(x[:n].astype(dt), mu.astype(dt), cv.astype(dt), pr.astype(dt),
                                  FLAG_IMPROVED)
        assert rel_err(enc, g[f"edge_enc_{tag}_n{n}"]) < TOL[tag]
    enc, _ = vl.fisher_encode(x.astype(dt), mu[:1].astype(dt), cv[:1].astype(dt), np.ones(1, dt),
                              FLAG_IMPROVED)
    assert rel_err(enc, g[f"edge_enc_{tag}_k1"]) < TOL[tag]
    enc, _ = vl.fisher_encode(x[:, :1].copy().astype(dt), mu[:, :1].copy().astype(dt),
                              cv[:, :1].copy().astype(dt), pr.astype(dt), FLAG_IMPROVED)
    assert rel_err(enc, g[f"edge_enc_{tag}_d1"]) < TOL[tag]


@pytest.mark.parametrize("tag", ["f", "d"])
def test_posteriors(vl, golden, tag):
    g = golden
    dt = DT[tag]
    q, ll = vl.get_gmm_data_posteriors(g["post_data"].astype(dt), g["post_priors"].astype(dt),
                                       g["post_means"].astype(dt), g["post_covs"].astype(dt))
    assert rel_err(q, g[f"post_q_{tag}"]) < TOL[tag]
    ref = float(g[f"post_ll_{tag}"])
    assert abs(ll - ref) <= TOL[tag] * abs(ref)


def _em(vl, g, dt, t):
    K, D = g["em_means0"].shape
    m = vl.GMM(D, K, dt)
    m.set_initialization("custom")
    m.set_max_num_iterations(t)
    m.set_covariance_lower_bound(g["em_lb"])
    m.set_means(g["em_means0"])
    m.set_covariances(g["em_covs0"])
    m.set_priors(g["em_priors0"])
    ll = m.cluster(g["em_data"].astype(dt))
    return m, ll


@pytest.mark.parametrize("tag", ["f", "d"])
def test_em_per_iteration(vl, golden, tag):
    """Parameters after t = 0..T iterations from the same custom init match
    VLFeat's, including the empty-mode restart at iteration 2."""
    g = golden
    dt = DT[tag]
    T = int(g["em_T"])
    # Float: measured maxima over t = 0..T against VLFeat's float run: LL
    # 3.6e-8, priors 9.3e-7, means 7.9e-7, covariances 1.8e-6, posteriors 3.6e-6.
    tol = {"f": 1e-5, "d": 1e-9}[tag]
    for t in range(T + 1):
        m, ll = _em(vl, g, dt, t)
        ref_ll = g[f"em_ll_{tag}"][t]
        assert abs(ll - ref_ll) <= tol * abs(ref_ll), t
        assert rel_err(m.priors, g[f"em_priors_{tag}"][t]) < tol, t
        assert rel_err(m.means, g[f"em_means_{tag}"][t]) < tol, t
        assert rel_err(m.covariances, g[f"em_covs_{tag}"][t]) < tol, t
        if t == T:
            assert m.num_restarts >= 1
            assert rel_err(m.posteriors, g[f"em_post_{tag}"]) < tol


def test_config0_em_and_fv(vl, restatement):
    """Config 0 at full size: 10 EM iterations (restarts fire) and the improved
    FV of 2,000 separate descriptors, double and float, against the
    restatement."""
    from vlfeat_b200 import workloads as W
    c = W.config0()
    # Float against the C restatement in float (its own float rounding):
    # measured LL 1.9e-9, priors 2.4e-6, means 6.2e-6, covariances 1.0e-5.
    for dt, tol in ((np.float64, 1e-9), (np.float32, 5e-5)):
        d = c["data"].astype(dt)
        ref = restatement.em(d, c["priors"], c["means"], c["covs"], c["lower_bound"], c["iters"])
        m = vl.GMM(c["D"], c["K"], dt)
        m.set_initialization("custom")
        m.set_max_num_iterations(c["iters"])
        m.set_covariance_lower_bound(c["lower_bound"])
        m.set_means(c["means"])
        m.set_covariances(c["covs"])
        m.set_priors(c["priors"])
        ll = m.cluster(d)
        assert abs(ll - ref["ll"]) <= tol * abs(ref["ll"])
        assert m.num_restarts == ref["restarts"]
        for name, got in (("priors", m.priors), ("means", m.means), ("covs", m.covariances)):
            assert rel_err(got, ref[name]) < tol, name
        f = c["fv_data"].astype(dt)
        enc, nt = vl.fisher_encode(f, ref["means"], ref["covs"], ref["priors"], FLAG_IMPROVED)
        enc_ref, nt_ref = restatement.fisher(f, ref["means"], ref["covs"], ref["priors"], FLAG_IMPROVED)
        assert rel_err(enc, enc_ref) < (1e-10 if dt == np.float64 else 2e-5)
        assert nt == nt_ref


def test_batched_matches_single(vl, restatement):
    """Batched uneven encoding (empty images included) equals per-image calls."""
    import torch
    from vlfeat_b200 import workloads as W
    pr, mu, cv = W.fv_gmm(32, 24, seed=5)
    counts = np.array([0, 1, 7, 300, 2500, 0, 4100, 33])
    offs = np.concatenate([[0], np.cumsum(counts)])
    x = W.pca_like(int(offs[-1]), 24, seed=6)
    dev = torch.device("cuda")
    enc = torch.zeros((len(counts), 2 * 32 * 24), device=dev)
    nt = torch.zeros(len(counts), dtype=torch.int64, device=dev)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    vl.fisher_encode_batch_device(enc, t(mu), t(cv), t(pr), t(x), offs, FLAG_IMPROVED, "exact", nt)
    enc = enc.cpu().numpy()
    nt = nt.cpu().numpy()
    for j in range(len(counts)):
        e, n = restatement.fisher(x[offs[j]:offs[j + 1]], mu, cv, pr, FLAG_IMPROVED)
        assert rel_err(enc[j], e) < 2e-5, j
        assert nt[j] == n


@pytest.mark.parametrize("K,D", [(200, 128), (130, 80), (7, 3), (257, 33)])
def test_batched_statistics_layouts(vl, restatement, K, D):
    """Batched exact encoding at shapes that reach every layout of the sparse
    statistics kernel: 64-component blocks (D = 128) and 128-component ones, a
    partial last block, 16-byte and 4-byte copies (K or D not a multiple of
    4), one to four dimensions per lane, an empty image and images cut into
    several 2,048-row segments; per image against the C restatement."""
    import torch
    from vlfeat_b200 import workloads as W
    pr, mu, cv = W.fv_gmm(K, D, seed=K + D)
    counts = np.array([0, 5, 1500, 4100, 37])
    offs = np.concatenate([[0], np.cumsum(counts)])
    x = W.pca_like(int(offs[-1]), D, seed=K * D)
    dev = torch.device("cuda")
    enc = torch.zeros((len(counts), 2 * K * D), device=dev)
    nt = torch.zeros(len(counts), dtype=torch.int64, device=dev)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    vl.fisher_encode_batch_device(enc, t(mu), t(cv), t(pr), t(x), offs, FLAG_IMPROVED, "exact", nt)
    enc = enc.cpu().numpy()
    nt = nt.cpu().numpy()
    for j in range(len(counts)):
        e, n = restatement.fisher(x[offs[j]:offs[j + 1]], mu, cv, pr, FLAG_IMPROVED)
        assert rel_err(enc[j], e) < 2e-5, j
        assert nt[j] == n


@pytest.mark.parametrize("K,D", [(96, 128), (70, 33)])
def test_em_statistics_layouts(vl, restatement, K, D):
    """Exact float EM at shapes that reach the sparse M-step statistics'
    64-component blocks (D = 128) and its 4-byte copies with a partial block
    (K = 70, D = 33): 4 iterations from the same custom initialisation against
    the C restatement in float."""
    from vlfeat_b200 import workloads as W
    pr, mu, cv = W.fv_gmm(K, D, seed=3 * K + D)
    x = W.pca_like(12000, D, seed=K + 7 * D)
    ref = restatement.em(x, pr, mu, cv, 1e-4, 4)
    m = vl.GMM(D, K, np.float32)
    m.set_initialization("custom")
    m.set_max_num_iterations(4)
    m.set_covariance_lower_bound(1e-4)
    m.set_means(mu)
    m.set_covariances(cv)
    m.set_priors(pr)
    ll = m.cluster(x)
    tol = 5e-5
    assert abs(ll - ref["ll"]) <= tol * abs(ref["ll"])
    assert m.num_restarts == ref["restarts"]
    for name, got in (("priors", m.priors), ("means", m.means), ("covs", m.covariances)):
        assert rel_err(got, ref[name]) < tol, name


def test_deterministic(vl, golden):
    g = golden
    a = _em(vl, g, np.float32, 5)[0]
    b = _em(vl, g, np.float32, 5)[0]
    assert np.array_equal(a.means, b.means) and np.array_equal(a.covariances, b.covariances)
    e1, _ = vl.fisher_encode(g["fv_data"], g["fv_means"].astype(np.float32),
                             g["fv_covs"].astype(np.float32), g["fv_priors"].astype(np.float32))
    e2, _ = vl.fisher_encode(g["fv_data"], g["fv_means"].astype(np.float32),
                             g["fv_covs"].astype(np.float32), g["fv_priors"].astype(np.float32))
    assert np.array_equal(e1, e2)


def _lanes_match(vl, golden):
    """The fixtures' k-means++ distances follow the SIMD kernel the reference
    picked on the fixture host; the library picks by the same rule here."""
    L = vl.lib()
    ours = 8 if L.vl_cpu_has_avx() else (4 if L.vl_cpu_has_sse2() else 1)
    return ours == int(golden["rand_lanes"])


def _rand_em(vl, golden, name, tag, T):
    dt = DT[tag]
    x = golden[f"rand_{name}_data"].astype(dt)
    K = int(golden[f"rand_{name}_K"])
    m = vl.GMM(x.shape[1], K, dt)
    m.set_initialization("rand")
    m.set_max_num_iterations(T)
    m.set_covariance_lower_bound(1e-4)
    vl.rand_seed(int(golden[f"rand_{name}_seed"]))
    ll = m.cluster(x)
    return m, ll


@pytest.mark.parametrize("name", ["small", "mix"])
@pytest.mark.parametrize("tag", ["f", "d"])
def test_rand_init_bit_exact(vl, golden, name, tag):
    """VlGMMRand initialisation (the default of vl_gmm_new) reproduces the
    reference bit for bit from the same seed: k-means++ centres drawn with
    the thread's MT19937, global data variance, uniform priors."""
    if not _lanes_match(vl, golden):
        pytest.skip("this host's SIMD support differs from the fixture host's")
    m, _ = _rand_em(vl, golden, name, tag, 0)
    for k, got in (("means", m.means), ("covs", m.covariances), ("priors", m.priors)):
        assert np.array_equal(got, golden[f"rand_{name}_{tag}_t0_{k}"]), k


@pytest.mark.parametrize("name", ["small", "mix"])
@pytest.mark.parametrize("tag", ["f", "d"])
def test_rand_init_then_em(vl, golden, name, tag):
    """Five EM iterations from the Rand initialisation match the reference's
    run (exact path; the same bounds as the custom-init EM test)."""
    if not _lanes_match(vl, golden):
        pytest.skip("this host's SIMD support differs from the fixture host's")
    m, ll = _rand_em(vl, golden, name, tag, 5)
    # Float: measured at most 1.1e-6 (means) against VLFeat's float run.
    tol = {"f": 1e-5, "d": 1e-9}[tag]
    ref_ll = float(golden[f"rand_{name}_{tag}_t5_ll"])
    assert abs(ll - ref_ll) <= tol * abs(ref_ll)
    assert rel_err(m.means, golden[f"rand_{name}_{tag}_t5_means"]) < tol
    assert rel_err(m.covariances, golden[f"rand_{name}_{tag}_t5_covs"]) < tol
    assert rel_err(m.priors, golden[f"rand_{name}_{tag}_t5_priors"]) < tol


def test_rand_init_api_and_repetitions(vl, golden):
    """vl_gmm_init_with_rand_data alone gives the same parameters as the
    cluster call's initialisation; with two repetitions the second draws
    fresh centres from the same generator (vl/gmm.c:1588-1593)."""
    import ctypes as C
    x = golden["rand_small_data"].astype(np.float32)
    K, seed = int(golden["rand_small_K"]), int(golden["rand_small_seed"])
    m = vl.GMM(x.shape[1], K, np.float32)
    vl.rand_seed(seed)
    vl.lib().vl_gmm_init_with_rand_data(m._h, x.ctypes.data_as(C.c_void_p), x.shape[0])
    if _lanes_match(vl, golden):
        assert np.array_equal(m.means, golden["rand_small_f_t0_means"])
    a = m.means.copy()
    m2 = vl.GMM(x.shape[1], K, np.float32)
    m2.set_initialization("rand")
    m2.set_max_num_iterations(0)
    m2.set_num_repetitions(2)
    vl.rand_seed(seed)
    m2.cluster(x)
    assert vl.lib().vl_get_last_error() == 0
    assert m2.means.shape == a.shape
