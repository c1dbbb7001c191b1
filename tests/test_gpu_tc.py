"""GPU parity of the tensor-core (tcgen05) paths through the C-ABI.

Reference: the FP64 C restatement (oracle/), itself pinned to VLFeat's own
double results.  Bounds on the relative L2 error of each Fisher vector:

* FP32 mode (fp16x3 on both contractions, fp32 accumulation): 1e-5, or --
  where VLFeat's own float path (oracle/_ref, the same image) is further
  than that from FP64 -- VLFeat's float error.  The improved Fisher vector's
  signed square root magnifies the absolute error of near-zero statistics, so
  fp32 arithmetic of either kind exceeds 1e-5 on a few images: on 256 images
  of the benchmark's shape VLFeat's float path measured max 1.5e-5 (median
  4.3e-6, 2 images above 1e-5), this path max 1.2e-5 (median 3.4e-6, 2
  images above 1e-5), the exact CUDA-core path max 1.7e-5.
* BF16 mode: 1e-3 (the metric's bound; measured ~1-2e-4, set by the single
  fp16 part of q)."""
import os

import numpy as np
import pytest

from conftest import rel_err
from oracle.oracle import FLAG_FAST, FLAG_IMPROVED, FLAG_NORMALIZED, FLAG_SQUARE_ROOT

pytestmark = pytest.mark.gpu

TOL = {"fp32": 1e-5, "bf16": 1e-3}


@pytest.fixture(scope="module")
def vlfeat_float():
    """VLFeat's own CPU library (float path), or None where it is not built."""
    from oracle.oracle import Reference
    try:
        return Reference(threads=os.cpu_count() or 1)
    except (FileNotFoundError, OSError):
        return None


def fv_bound(mode, ref64, vf, x, mu, cv, pr, flags):
    """The bound for one Fisher vector: TOL[mode], raised for FP32 mode to
    VLFeat's own float error on the same input when that is larger."""
    if mode != "fp32" or vf is None:
        return TOL[mode]
    e, _ = vf.fisher(x.astype(np.float32), mu.astype(np.float32), cv.astype(np.float32),
                     pr.astype(np.float32), flags)
    return max(TOL[mode], rel_err(e, ref64))


@pytest.fixture(autouse=True)
def reset_mode(vl):
    yield
    vl.set_precision("exact")


def _t(a, dev="cuda"):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


@pytest.mark.parametrize("mode", ["fp32", "bf16"])
# (256, 128): W does not fit in shared memory and streams through the stages.
@pytest.mark.parametrize("KD", [(256, 80), (64, 64), (128, 80), (64, 128), (256, 128)])
def test_fv_single(vl, restatement, vlfeat_float, mode, KD):
    from vlfeat_b200 import workloads as W
    K, D = KD
    pr, mu, cv = W.fv_gmm(K, D, seed=3)
    x = W.pca_like(3000, D, seed=4)
    ref, nref = restatement.fisher(x.astype(np.float64), mu.astype(np.float64), cv.astype(np.float64),
                                   pr.astype(np.float64), FLAG_IMPROVED)
    vl.set_precision(mode)
    enc, nt = vl.fisher_encode(x, mu, cv, pr, FLAG_IMPROVED)
    assert vl.last_precision() == mode
    assert rel_err(enc, ref) < fv_bound(mode, ref, vlfeat_float, x, mu, cv, pr, FLAG_IMPROVED)
    assert abs(nt - nref) <= max(2, 1e-3 * nref)


@pytest.mark.parametrize("mode", ["fp32", "bf16"])
@pytest.mark.parametrize("flags", [0, FLAG_SQUARE_ROOT, FLAG_NORMALIZED, FLAG_IMPROVED | FLAG_FAST])
def test_fv_flags(vl, restatement, vlfeat_float, mode, flags):
    from vlfeat_b200 import workloads as W
    pr, mu, cv = W.fv_gmm(256, 80, seed=7)
    x = W.pca_like(1000, 80, seed=8)
    ref, nref = restatement.fisher(x.astype(np.float64), mu.astype(np.float64), cv.astype(np.float64),
                                   pr.astype(np.float64), flags)
    vl.set_precision(mode)
    enc, nt = vl.fisher_encode(x, mu, cv, pr, flags)
    tol = fv_bound(mode, ref, vlfeat_float, x, mu, cv, pr, flags) * (3 if flags & FLAG_FAST else 1)
    assert rel_err(enc, ref) < tol


@pytest.mark.parametrize("mode", ["fp32", "bf16"])
def test_batched_uneven(vl, restatement, vlfeat_float, mode):
    import torch
    from vlfeat_b200 import workloads as W
    K, D = 256, 80
    pr, mu, cv = W.fv_gmm(K, D, seed=9)
    counts = np.array([0, 1, 5, 127, 128, 129, 3000, 0, 9000, 17, 20000, 250])
    offs = np.concatenate([[0], np.cumsum(counts)])
    x = W.pca_like(int(offs[-1]), D, seed=10)
    enc = torch.zeros((len(counts), 2 * K * D), device="cuda")
    nt = torch.zeros(len(counts), dtype=torch.int64, device="cuda")
    vl.fisher_encode_batch_device(enc, _t(mu), _t(cv), _t(pr), _t(x), offs, FLAG_IMPROVED, mode, nt)
    enc = enc.cpu().numpy()
    nt = nt.cpu().numpy()
    for j in range(len(counts)):
        e, n = restatement.fisher(x[offs[j]:offs[j + 1]].astype(np.float64), mu.astype(np.float64),
                                  cv.astype(np.float64), pr.astype(np.float64), FLAG_IMPROVED)
        if counts[j] == 0:
            assert np.all(enc[j] == 0) and nt[j] == 0
        else:
            xj = x[offs[j]:offs[j + 1]]
            assert rel_err(enc[j], e) < fv_bound(mode, e, vlfeat_float, xj, mu, cv, pr, FLAG_IMPROVED), j
            assert abs(int(nt[j]) - n) <= max(2, 1e-3 * n), j


@pytest.mark.parametrize("D", [80, 128])
def test_posteriors_fp32(vl, restatement, D):
    from vlfeat_b200 import workloads as W
    pr, mu, cv = W.fv_gmm(256, D, seed=12)
    x = W.pca_like(5000, D, seed=13)
    q64, ll64 = restatement.posteriors(x.astype(np.float64), pr.astype(np.float64),
                                       mu.astype(np.float64), cv.astype(np.float64))
    vl.set_precision("fp32")
    q, ll = vl.get_gmm_data_posteriors(x, pr, mu, cv)
    # Each score sums 2D fp16x3 products, so the error grows with D.  Measured
    # max |q - q64| 1.3e-5 (D=80), 2.0e-5 (D=128) -- the exact CUDA-core path,
    # VLFeat's formulation in fp32: 2.1e-5, 4.6e-5; LL relative 8.7e-7, 1.7e-6.
    q_tol, ll_tol = {80: (2.5e-5, 2e-6), 128: (4e-5, 4e-6)}[D]
    assert np.max(np.abs(q - q64)) < q_tol
    assert abs(ll - ll64) < ll_tol * abs(ll64)


@pytest.mark.parametrize("mode", ["fp32", "bf16"])
def test_batched_many_tiles_per_block(vl, mode):
    """64 images of the benchmark's count distribution (about 300,000 rows, a
    dozen row tiles per block in one launch): every block refills its ring
    of descriptor-row boxes and its q-image staging many times, and the
    statistics read q^T boxes across tile and image boundaries.  Each image
    against the exact CUDA-core path (the FP32 path within 1e-4, the BF16 path
    within 2e-3 of it, term counts within 1e-3 of its) and two runs
    bit-identical."""
    import torch
    from vlfeat_b200 import workloads as W
    K, D = 256, 80
    pr, mu, cv = W.fv_gmm(K, D, seed=11)
    counts = W.config2_counts(4096)[:64]
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    x = _t(W.pca_like(int(offs[-1]), D, seed=16))
    out = {}
    for name, m in (("exact", "exact"), ("a", mode), ("b", mode)):
        enc = torch.zeros((len(counts), 2 * K * D), device="cuda")
        nt = torch.zeros(len(counts), dtype=torch.int64, device="cuda")
        vl.fisher_encode_batch_device(enc, _t(mu), _t(cv), _t(pr), x, offs, FLAG_IMPROVED, m, nt)
        torch.cuda.synchronize()
        out[name] = (enc.cpu().numpy(), nt.cpu().numpy())
    assert np.array_equal(out["a"][0], out["b"][0]) and np.array_equal(out["a"][1], out["b"][1])
    tol = 1e-4 if mode == "fp32" else 2e-3
    for j in range(len(counts)):
        assert rel_err(out["a"][0][j], out["exact"][0][j]) < tol, j
        n = int(out["exact"][1][j])
        assert abs(int(out["a"][1][j]) - n) <= max(2, 1e-3 * n), j


@pytest.mark.parametrize("KD", [(256, 64), (256, 80), (256, 128), (200, 80), (64, 128)])
def test_posteriors_many_tiles_per_block(vl, KD):
    """120,000 rows (938 row tiles, six or seven per block): every block
    reuses its ring of descriptor-row boxes and its operand stages many
    times.  Tensor-core posteriors against the exact CUDA-core path on every
    row, and two runs bit-identical (a box refilled before all its readers
    were done showed up as wrong, run-dependent rows from each block's second
    tile on)."""
    import torch
    from vlfeat_b200 import workloads as W
    K, D = KD
    N = 120_000
    x = W.sift_like(N, D, seed=200) if D == 128 else W.pca_like(N, D, seed=15)
    pr, mu, cv = W.custom_init(x, K, seed=201)
    X, P, M, C = _t(x), _t(pr), _t(mu), _t(cv)
    q = {}
    for name, mode in (("exact", "exact"), ("a", "fp32"), ("b", "fp32")):
        out = torch.zeros((N, K), device="cuda")
        vl.gmm_posteriors_device(out, P, M, C, X, mode)
        torch.cuda.synchronize()
        q[name] = out.cpu().numpy()
    assert np.array_equal(q["a"], q["b"])
    assert np.max(np.abs(q["a"] - q["exact"])) < 1e-4


# EM in the tensor-core modes: E-step and M-step statistics on tcgen05
# (the M-step from the E-step's posterior image, thresholded at 1e-2/K).
# Bounds on the relative L2 error of every parameter against the FP64
# restatement after the run; measured values in the comments.
EM_TOL = {"fp32": 5e-5,   # config 0: means 1.5e-5, covs 3.1e-5, priors 2.0e-5; config 1 and
                          # K=1024: up to 5.8e-6 (the exact CUDA-core path: up to 1.8e-5)
          "bf16": 2e-4}   # config 0: 2.2e-5, 4.4e-5, 2.4e-5; config 1 and K=1024: up to 9.0e-5


def _em(vl, c, T, mode):
    vl.set_precision(mode)
    m = vl.GMM(c["D"], c["K"], np.float32)
    m.set_initialization("custom")
    m.set_max_num_iterations(T)
    m.set_covariance_lower_bound(c["lower_bound"])
    m.set_means(c["means"])
    m.set_covariances(c["covs"])
    m.set_priors(c["priors"])
    return m, m.cluster(c["data"])


@pytest.mark.parametrize("mode", ["fp32", "bf16"])
def test_em_tensor_core(vl, restatement, mode):
    """Config-0 generator (D=64, K=64) for 5 iterations; its empty-mode
    restarts run, and their iterations take the M-step from the rows."""
    from vlfeat_b200 import workloads as W
    c = W.config0(scale=0.3)
    r = restatement.em(c["data"].astype(np.float64), c["priors"], c["means"], c["covs"],
                       c["lower_bound"], 5)
    m, ll = _em(vl, c, 5, mode)
    assert m.num_restarts > 0
    assert abs(ll - r["ll"]) <= 2e-5 * abs(r["ll"])
    assert rel_err(m.means, r["means"]) < EM_TOL[mode]
    assert rel_err(m.covariances, r["covs"]) < EM_TOL[mode]
    assert rel_err(m.priors, r["priors"]) < EM_TOL[mode]


@pytest.mark.parametrize("mode", ["fp32", "bf16"])
def test_em_tensor_core_sift_d128(vl, restatement, mode):
    """EM at D=128, K=256 (W streamed through the E-step's stages) on the
    SIFT-shaped config-1 generator at reduced N."""
    from vlfeat_b200 import workloads as W
    c = W.config1(N=20000, K=256, iters=3)
    r = restatement.em(c["data"].astype(np.float64), c["priors"], c["means"], c["covs"],
                       c["lower_bound"], 3)
    m, ll = _em(vl, c, 3, mode)
    assert abs(ll - r["ll"]) <= 2e-5 * abs(r["ll"])
    assert rel_err(m.means, r["means"]) < EM_TOL[mode]
    assert rel_err(m.covariances, r["covs"]) < EM_TOL[mode]
    assert rel_err(m.priors, r["priors"]) < EM_TOL[mode]


def test_tc_deterministic(vl):
    from vlfeat_b200 import workloads as W
    pr, mu, cv = W.fv_gmm(256, 80, seed=14)
    x = W.pca_like(7000, 80, seed=15)
    vl.set_precision("bf16")
    a, _ = vl.fisher_encode(x, mu, cv, pr)
    b, _ = vl.fisher_encode(x, mu, cv, pr)
    assert np.array_equal(a, b)


# ---------------------------------------------------------------- K > 256
# Above 256 components the E-step runs as thread-block clusters: CTA r of a
# cluster takes components [r Kb, (r+1) Kb) and the CTAs exchange each row's
# (max, sum, argmax) through distributed shared memory before normalising.
# K=300: 2 CTAs x 160; K=520: 3 x 192 (image padded from 576 to 640);
# K=512 and 1024: 2 and 4 x 256 (D=128 streams W through the stages).
CLUSTER_KD = [(1024, 80), (520, 80), (300, 64), (512, 128)]


@pytest.mark.parametrize("mode", ["fp32", "bf16"])
@pytest.mark.parametrize("KD", CLUSTER_KD)
def test_fv_cluster(vl, restatement, vlfeat_float, mode, KD):
    from vlfeat_b200 import workloads as W
    K, D = KD
    pr, mu, cv = W.fv_gmm(K, D, seed=31)
    x = W.pca_like(3000, D, seed=32)
    ref, nref = restatement.fisher(x.astype(np.float64), mu.astype(np.float64), cv.astype(np.float64),
                                   pr.astype(np.float64), FLAG_IMPROVED)
    vl.set_precision(mode)
    enc, nt = vl.fisher_encode(x, mu, cv, pr, FLAG_IMPROVED)
    assert rel_err(enc, ref) < fv_bound(mode, ref, vlfeat_float, x, mu, cv, pr, FLAG_IMPROVED)
    assert abs(nt - nref) <= max(2, 1e-3 * nref)


@pytest.mark.parametrize("mode", ["fp32", "bf16"])
def test_fv_cluster_fast(vl, restatement, mode):
    """FAST (hard assignment to the row's argmax) across the CTAs of a
    cluster: the first maximum over all K wins."""
    from vlfeat_b200 import workloads as W
    pr, mu, cv = W.fv_gmm(1024, 80, seed=33)
    x = W.pca_like(2000, 80, seed=34)
    flags = FLAG_IMPROVED | FLAG_FAST
    ref, nref = restatement.fisher(x.astype(np.float64), mu.astype(np.float64), cv.astype(np.float64),
                                   pr.astype(np.float64), flags)
    vl.set_precision(mode)
    enc, nt = vl.fisher_encode(x, mu, cv, pr, flags)
    assert rel_err(enc, ref) < 3 * TOL[mode]
    assert nt == nref == 2000


@pytest.mark.parametrize("mode", ["fp32", "bf16"])
def test_batched_uneven_cluster(vl, restatement, vlfeat_float, mode):
    import torch
    from vlfeat_b200 import workloads as W
    K, D = 520, 80
    pr, mu, cv = W.fv_gmm(K, D, seed=35)
    counts = np.array([0, 1, 129, 3000, 0, 4100, 17])
    offs = np.concatenate([[0], np.cumsum(counts)])
    x = W.pca_like(int(offs[-1]), D, seed=36)
    enc = torch.zeros((len(counts), 2 * K * D), device="cuda")
    nt = torch.zeros(len(counts), dtype=torch.int64, device="cuda")
    vl.fisher_encode_batch_device(enc, _t(mu), _t(cv), _t(pr), _t(x), offs, FLAG_IMPROVED, mode, nt)
    enc = enc.cpu().numpy()
    nt = nt.cpu().numpy()
    for j in range(len(counts)):
        e, n = restatement.fisher(x[offs[j]:offs[j + 1]].astype(np.float64), mu.astype(np.float64),
                                  cv.astype(np.float64), pr.astype(np.float64), FLAG_IMPROVED)
        if counts[j] == 0:
            assert np.all(enc[j] == 0) and nt[j] == 0
        else:
            xj = x[offs[j]:offs[j + 1]]
            assert rel_err(enc[j], e) < fv_bound(mode, e, vlfeat_float, xj, mu, cv, pr, FLAG_IMPROVED), j
            assert abs(int(nt[j]) - n) <= max(2, 1e-3 * n), j


@pytest.mark.parametrize("KD", [(1024, 80), (1024, 128), (520, 64)])
def test_posteriors_cluster_fp32(vl, restatement, KD):
    from vlfeat_b200 import workloads as W
    K, D = KD
    pr, mu, cv = W.fv_gmm(K, D, seed=37)
    x = W.pca_like(4000, D, seed=38)
    q64, ll64 = restatement.posteriors(x.astype(np.float64), pr.astype(np.float64),
                                       mu.astype(np.float64), cv.astype(np.float64))
    vl.set_precision("fp32")
    q, ll = vl.get_gmm_data_posteriors(x, pr, mu, cv)
    q_tol, ll_tol = {64: (2.5e-5, 2e-6), 80: (2.5e-5, 2e-6), 128: (4e-5, 4e-6)}[D]
    assert np.max(np.abs(q - q64)) < q_tol
    assert abs(ll - ll64) < ll_tol * abs(ll64)


@pytest.mark.parametrize("mode", ["fp32", "bf16"])
def test_em_cluster_k1024(vl, restatement, mode):
    """EM at K=1024, D=128 (the large-EM shape) on the SIFT-like generator at
    reduced N: cluster E-step, statistics over 1,024 components."""
    from vlfeat_b200 import workloads as W
    c = W.config1(N=30000, K=1024, iters=2)
    r = restatement.em(c["data"].astype(np.float64), c["priors"], c["means"], c["covs"],
                       c["lower_bound"], 2)
    m, ll = _em(vl, c, 2, mode)
    assert abs(ll - r["ll"]) <= 2e-5 * abs(r["ll"])
    assert rel_err(m.means, r["means"]) < EM_TOL[mode]
    assert rel_err(m.covariances, r["covs"]) < EM_TOL[mode]
    assert rel_err(m.priors, r["priors"]) < EM_TOL[mode]


def test_config1_full_size_em_per_iteration(vl):
    """Config 1 at its stated size: N = 1,000,000 SIFT-like descriptors, D =
    128, K = 256, custom initialisation from 256 seeded rows, variance floor
    1e-4 x the largest global variance, 20 iterations.  Every iteration's
    parameters (after t M-steps, t = 0..20) and log-likelihood are compared
    with an FP64 run on the GPU from the same initialisation (the library's
    exact double kernels, which match VLFeat's double path to 1e-10).
    Measured maxima over the 21 snapshots (relative L2): FP32 mode means
    7.8e-6, covariances 1.2e-5, priors 6.3e-6, LL 1.3e-7; EXACT (VLFeat's
    float formulation) 8.3e-6, 1.3e-5, 3.8e-5, 2.3e-7; BF16 5.6e-5, 8.6e-5,
    4.3e-5, 1.4e-7.  The errors grow about linearly with the iterations."""
    import torch
    from vlfeat_b200 import workloads as W
    c = W.config1(N=1_000_000, K=256, iters=20)

    def model(dt):
        m = vl.GMM(128, 256, dt)
        m.set_initialization("custom")
        m.set_max_num_iterations(20)
        m.set_covariance_lower_bound(c["lower_bound"])
        m.set_means(c["means"])
        m.set_covariances(c["covs"])
        m.set_priors(c["priors"])
        m.set_param_trace(True)
        return m
    m64 = model(np.float64)
    m64.cluster(c["data"].astype(np.float64))
    tr64, ll64 = m64.param_trace(), m64.ll_trace
    assert len(tr64) == 21
    x = torch.from_numpy(c["data"]).cuda()
    bounds = {"fp32": (2e-5, 2e-5, 2e-5, 5e-7), "exact": (2e-5, 3e-5, 8e-5, 5e-7),
              "bf16": (1.5e-4, 2e-4, 1e-4, 5e-7)}
    for mode, (bm, bc, bp, bl) in bounds.items():
        m = model(np.float32)
        m.em_device(x, mode)
        tr, ll = m.param_trace(), m.ll_trace
        assert len(tr) == 21 and len(ll) == 21, mode
        for t in range(21):
            assert rel_err(tr[t][0], tr64[t][0]) < bm, (mode, t)
            assert rel_err(tr[t][1], tr64[t][1]) < bc, (mode, t)
            assert rel_err(tr[t][2], tr64[t][2]) < bp, (mode, t)
            assert abs(ll[t] - ll64[t]) < bl * abs(ll64[t]), (mode, t)


# ------------------------------------------------- zero-padded dimensions
# Dimensions other than 64, 80 and 128 (up to 128) run on the tensor cores
# zero-padded to the next of them: D = 82 is the recognition app's encoder
# input (PCA-80 plus the 'xy' frame extension, apps/recognition/
# encodeImage.m:91-103).
@pytest.mark.parametrize("mode", ["fp32", "bf16"])
@pytest.mark.parametrize("D", [82, 32, 100])
def test_fv_padded_dimension(vl, restatement, vlfeat_float, mode, D):
    import torch
    from vlfeat_b200 import workloads as W
    K = 256
    pr, mu, cv = W.fv_gmm(K, D, seed=41)
    counts = np.array([3000, 0, 200, 1377])
    offs = np.concatenate([[0], np.cumsum(counts)])
    x = W.pca_like(int(offs[-1]), D, seed=42)
    enc = torch.zeros((len(counts), 2 * K * D), device="cuda")
    vl.fisher_encode_batch_device(enc, _t(mu), _t(cv), _t(pr), _t(x), offs, FLAG_IMPROVED, mode)
    assert vl.last_precision() == mode
    enc = enc.cpu().numpy()
    for j in range(len(counts)):
        xj = x[offs[j]:offs[j + 1]]
        e, _ = restatement.fisher(xj.astype(np.float64), mu.astype(np.float64), cv.astype(np.float64),
                                  pr.astype(np.float64), FLAG_IMPROVED)
        if counts[j] == 0:
            assert np.all(enc[j] == 0)
        else:
            assert rel_err(enc[j], e) < fv_bound(mode, e, vlfeat_float, xj, mu, cv, pr, FLAG_IMPROVED), j


def test_posteriors_padded_dimension(vl, restatement):
    from vlfeat_b200 import workloads as W
    D = 82
    pr, mu, cv = W.fv_gmm(256, D, seed=43)
    x = W.pca_like(5000, D, seed=44)
    q64, ll64 = restatement.posteriors(x.astype(np.float64), pr.astype(np.float64),
                                       mu.astype(np.float64), cv.astype(np.float64))
    vl.set_precision("fp32")
    q, ll = vl.get_gmm_data_posteriors(x, pr, mu, cv)
    assert vl.last_precision() == "fp32"
    assert np.max(np.abs(q - q64)) < 4e-5
    assert abs(ll - ll64) < 4e-6 * abs(ll64)


def test_em_on_padded_dimension(vl, restatement):
    """EM at a dimension the tensor-core M-step is not built for (D = 50): the
    E-steps run zero-padded on the tensor cores (the record says FP32), the
    M-steps on the CUDA cores; the result stays within the FP32 mode's EM
    bound of the FP64 restatement."""
    from vlfeat_b200 import workloads as W
    c = W.config0(scale=0.1)
    c = dict(c, data=c["data"][:, :50].copy(), means=c["means"][:, :50].copy(), covs=c["covs"][:, :50].copy(), D=50)
    r = restatement.em(c["data"].astype(np.float64), c["priors"], c["means"], c["covs"], c["lower_bound"], 3)
    m, ll = _em(vl, c, 3, "fp32")
    assert vl.last_precision() == "fp32"
    assert abs(ll - r["ll"]) <= 2e-5 * abs(r["ll"])
    assert rel_err(m.means, r["means"]) < EM_TOL["fp32"]
    assert rel_err(m.covariances, r["covs"]) < EM_TOL["fp32"]
    assert rel_err(m.priors, r["priors"]) < EM_TOL["fp32"]
