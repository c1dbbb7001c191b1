"""Streamed EM (vlb200_gmm_em_stream_device): the vl_gmm_em loop with the
N x K posteriors never resident -- chunked E-step passes accumulating the
M-step statistics, column masses and log-likelihood, the M-step reduced in
f64, restarts re-deriving the iteration's posteriors chunk by chunk -- and its
router-pruned variant, in which every judge_every-th iteration runs the full
E-step and measures the router's missed posterior mass.

* Without a router it reproduces the resident loop: bit for bit in EXACT mode
  (the same E-step rows and the same M-step slabs), within 1e-6 in FP32 mode
  (statistics items cut at chunk starts), including the empty-mode restarts
  of the golden EM case, which also match VLFeat's own run.
* vl_gmm_get_posteriors afterwards recomputes the final E-step.
* The router-pruned run stays close to the FP64 run from the same
  initialisation, and its report marks the judged iterations."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _model(vl, c, T, dt=np.float32):
    m = vl.GMM(c["D"], c["K"], dt)
    m.set_initialization("custom")
    m.set_max_num_iterations(T)
    m.set_covariance_lower_bound(c["lower_bound"])
    m.set_means(c["means"])
    m.set_covariances(c["covs"])
    m.set_priors(c["priors"])
    return m


@pytest.mark.parametrize("mode", ["exact", "fp32"])
def test_streamed_equals_resident(vl, mode):
    import torch
    from vlfeat_b200 import workloads as W
    c = W.config1(N=120_000, K=256, iters=4)
    x = torch.from_numpy(c["data"]).cuda()
    a = _model(vl, c, 4)
    lla = a.em_device(x, mode)
    b = _model(vl, c, 4)
    llb = b.em_stream_device(x, mode, chunk_rows=30_000)
    assert vl.last_precision() == mode
    tol = 0.0 if mode == "exact" else 5e-6  # FP32: items cut at chunk starts (measured 1.2e-6)
    assert abs(lla - llb) <= 1e-12 * abs(lla) + (tol * abs(lla))
    for got, want in ((b.means, a.means), (b.covariances, a.covariances), (b.priors, a.priors)):
        assert rel_err(got, want) <= tol
    assert len(b.stream_report()) == 5
    # The final E-step's posteriors, recomputed on demand.
    q, _ = vl.get_gmm_data_posteriors(c["data"][:5000], b.priors, b.means, b.covariances) \
        if mode == "exact" else (None, None)
    post = b.posteriors
    assert post.shape == (120_000, 256)
    if q is not None:
        assert np.array_equal(post[:5000], q)
    assert rel_err(post, a.posteriors) <= max(tol, 1e-12) * 10


def test_streamed_restarts_match_vlfeat(vl, golden):
    """The golden EM case restarts an emptied mode at iteration 2: the streamed
    loop re-derives the posteriors chunk by chunk for the restart's M-steps and
    lands on VLFeat's parameters (float run, the exact path's 1e-5)."""
    import torch
    g = golden
    T = int(g["em_T"])
    x = torch.from_numpy(g["em_data"].astype(np.float32)).cuda()
    m = vl.GMM(x.shape[1], int(g["em_means0"].shape[0]), np.float32)
    m.set_initialization("custom")
    m.set_max_num_iterations(T)
    m.set_covariance_lower_bound(g["em_lb"])
    m.set_means(g["em_means0"])
    m.set_covariances(g["em_covs0"])
    m.set_priors(g["em_priors0"])
    ll = m.em_stream_device(x, "exact", chunk_rows=64)
    assert m.num_restarts >= 1
    ref_ll = g["em_ll_f"][T]
    assert abs(ll - ref_ll) <= 1e-5 * abs(ref_ll)
    assert rel_err(m.means, g["em_means_f"][T]) < 1e-5
    assert rel_err(m.covariances, g["em_covs_f"][T]) < 1e-5
    assert rel_err(m.priors, g["em_priors_f"][T]) < 1e-5
    assert rel_err(m.posteriors, g["em_post_f"]) < 1e-5


def test_router_pruned_streamed_em_against_fp64(vl):
    """The large-EM pattern at reduced size: SIFT-like data, D = 128, K = 256,
    10 iterations; BF16 mode with router-pruned E-steps (m = 8, fallback below
    0.99 predicted candidate mass) and a full E-step every 5th iteration.
    Its final parameters and log-likelihood are compared with an FP64 run of
    the full EM from the same initialisation.  The router's missed posterior
    mass (about 1e-3 of each row's mass before its first refit) perturbs every
    pruned M-step, and EM carries the perturbation on: the final means
    measured 3.4e-2 from the FP64 run's (the BF16 mode without router: 5e-5),
    the log-likelihood within 1e-3."""
    import torch
    from vlfeat_b200 import workloads as W
    from vlfeat_b200.router import Router
    c = W.config1(N=300_000, K=256, iters=10)
    x = torch.from_numpy(c["data"]).cuda()
    r = Router(128, 256, hidden=(256, 256), seed=4)
    r.set_input_transform(c["data"].mean(0), 1.0 / np.maximum(c["data"].std(0), 1e-3))
    m = _model(vl, c, 10)
    ll = m.em_stream_device(x, "bf16", chunk_rows=100_000, router=r, m=8, threshold=0.99, judge_every=5)
    rep = m.stream_report()
    assert len(rep) == 11
    assert [row["judged"] for row in rep] == [t % 5 == 0 for t in range(11)]
    assert [row["routed"] for row in rep] == [t % 5 != 0 for t in range(11)]
    for t in (0, 5, 10):
        assert 0.0 <= rep[t]["missed_mass"] < 0.05, rep[t]
    m64 = _model(vl, c, 10, np.float64)
    ll64 = m64.cluster(c["data"].astype(np.float64))
    assert abs(ll - ll64) <= 1e-3 * abs(ll64)
    assert rel_err(m.means, m64.means) < 0.1
    assert rel_err(m.covariances, m64.covariances) < 0.2
    assert rel_err(m.priors, m64.priors) < 0.2
    for t in range(11):
        if rep[t]["routed"]:
            assert 0 <= rep[t]["fallback_rows"] <= 300_000


def test_streamed_restarts_in_fp32_mode_match_resident(vl):
    """Config 0 (restarts fire at iteration 2) in FP32 mode: the streamed loop's
    restarts re-derive the tensor-core E-step's posteriors chunk by chunk and
    land where the resident loop does."""
    import torch
    from vlfeat_b200 import workloads as W
    c = W.config0()
    x = torch.from_numpy(c["data"]).cuda()
    a = _model(vl, c, 6)
    lla = a.em_device(x, "fp32")
    b = _model(vl, c, 6)
    llb = b.em_stream_device(x, "fp32", chunk_rows=10_000)
    assert a.num_restarts == b.num_restarts and a.num_restarts >= 1
    assert abs(lla - llb) <= 1e-6 * abs(lla)
    # Statistics items cut at chunk starts change the fp32 sums' order; the
    # restarts' discontinuous choices carry that on (measured 1.1e-5 priors).
    for got, want in ((b.means, a.means), (b.covariances, a.covariances), (b.priors, a.priors)):
        assert rel_err(got, want) < 5e-5


def _sharded(vl, c, T, x_t, world, mode, dt):
    """EM with the rows of x_t sharded over `world` ranks, run as threads of
    this process on one GPU (each with its own model object and the library's
    per-thread stream); the all-reduce sums through host barriers (bounded),
    so no kernel ever waits for another."""
    import threading
    from vlfeat_b200 import replicas
    N = x_t.shape[0]
    bar = threading.Barrier(world, timeout=60)
    slots = [None] * world
    res, errs = [None] * world, []

    def make_reduce(r):
        def reduce(values):
            slots[r] = values.copy()
            bar.wait()
            total = np.sum(np.stack(slots), axis=0)  # every rank adds in rank order
            bar.wait()
            values[...] = total
        return reduce

    def run(r):
        try:
            r0, r1 = replicas.row_shard(N, r, world)
            m = _model(vl, c, T, dt)
            ll = m.em_sharded_device(x_t[r0:r1], N, make_reduce(r), mode)
            res[r] = (ll, m.means, m.covariances, m.priors, m.num_restarts)
        except BaseException as e:  # noqa: BLE001
            errs.append(e)
            bar.abort()

    th = [threading.Thread(target=run, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=600)
    assert not errs, errs
    return res


@pytest.mark.parametrize("mode,dt,tol", [("exact", np.float64, 1e-10), ("exact", np.float32, 2e-5),
                                         ("fp32", np.float32, 5e-5)])
def test_sharded_em_matches_one_process(vl, mode, dt, tol):
    """Config-0 data (restarts fire at iteration 2) sharded over two ranks:
    every rank ends with the same parameters and log-likelihood, equal to the
    single-process streamed EM's within the precision's summation-order
    tolerance (the ranks' partial sums are added across ranks), with the same
    number of restarts."""
    import torch
    from vlfeat_b200 import workloads as W
    c = W.config0(scale=0.3)
    x = torch.from_numpy(c["data"].astype(dt)).cuda()
    one = _model(vl, c, 5, dt)
    if dt == np.float32:
        ll1 = one.em_stream_device(x, mode)
    else:  # the double model's loop through vl_gmm_cluster (custom initialisation: no init)
        vl.set_precision(mode)
        ll1 = one.cluster(c["data"].astype(dt))
    res = _sharded(vl, c, 5, x, 2, mode, dt)
    (lla, mua, cva, pra, ra), (llb, mub, cvb, prb, rb) = res
    assert lla == llb and ra == rb
    assert np.array_equal(mua, mub) and np.array_equal(cva, cvb) and np.array_equal(pra, prb)
    assert ra == one.num_restarts and ra > 0
    assert abs(lla - ll1) <= tol * abs(ll1)
    for got, want in ((mua, one.means), (cva, one.covariances), (pra, one.priors)):
        assert rel_err(got, want) < tol
