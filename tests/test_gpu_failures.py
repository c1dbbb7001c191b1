"""Failure handling, tested without faulting or hanging the GPU.

* A bounded mbarrier wait that nothing completes runs out after its limit:
  the kernel records its code in the launch's error word and returns, the
  host raises VL_ERR_BAD_ARG with the code, and the CUDA context keeps
  working (the mechanism of every tcgen05 kernel's waits, run by
  vlb200_selftest_bounded_wait on a barrier that nothing arrives on).
* Device allocations that fail (injected on the host by
  vlb200_debug_fail_allocations, as a failed cudaMalloc) surface as
  VL_ERR_ALLOC with the call's error sentinel, and the next call succeeds.
* Non-finite descriptors: the reference's C library does not reject them
  (only its MATLAB binding does, toolbox/gmm/vl_gmm.c:240-262); a NaN or an
  infinite value makes that image's Fisher vector non-finite in VLFeat's
  float code and here, in every arithmetic mode, and leaves the other images
  of a batch unchanged; EM on such data gives a NaN log-likelihood in both."""
import ctypes as C
import os
import threading
import time

import numpy as np
import pytest

from conftest import rel_err
from oracle.oracle import FLAG_IMPROVED

pytestmark = pytest.mark.gpu

VL_ERR_ALLOC, VL_ERR_BAD_ARG = 2, 3


def _decl(lib):
    lib.vlb200_selftest_bounded_wait.restype = C.c_int
    lib.vlb200_selftest_bounded_wait.argtypes = [C.c_double]
    lib.vlb200_debug_fail_allocations.restype = None
    lib.vlb200_debug_fail_allocations.argtypes = [C.c_uint64]


def test_bounded_wait_runs_out_and_context_survives(vl):
    lib = vl.lib()
    _decl(lib)
    t0 = time.perf_counter()
    rc = lib.vlb200_selftest_bounded_wait(50.0)
    dt = time.perf_counter() - t0
    assert rc == VL_ERR_BAD_ARG
    assert b"gave up waiting (code 99)" in lib.vl_get_last_error_message()
    assert 0.05 <= dt < 2.0
    # The context is intact: a tensor-core encode afterwards is correct.
    from vlfeat_b200 import workloads as W
    from oracle.oracle import Restatement
    pr, mu, cv = W.fv_gmm(256, 80, seed=5)
    x = W.pca_like(2000, 80, seed=6)
    vl.set_precision("fp32")
    try:
        enc, _ = vl.fisher_encode(x, mu, cv, pr, FLAG_IMPROVED)
    finally:
        vl.set_precision("exact")
    ref, _ = Restatement().fisher(x.astype(np.float64), mu.astype(np.float64), cv.astype(np.float64),
                                  pr.astype(np.float64), FLAG_IMPROVED)
    assert rel_err(enc, ref) < 2e-5
    lib.vl_set_last_error(0, None)


def test_selftest_rejects_bad_limits(vl):
    lib = vl.lib()
    _decl(lib)
    for bad in (0.0, -1.0, 5000.0):
        assert lib.vlb200_selftest_bounded_wait(bad) == VL_ERR_BAD_ARG
        assert b"limit" in lib.vl_get_last_error_message()
    lib.vl_set_last_error(0, None)


def test_injected_allocation_failure_is_reported_and_recovered(vl):
    """A fresh host thread has empty scratch, so its first encode allocates:
    with one failure injected it returns VL_ERR_ALLOC and 0 terms, as the
    error convention says; the next call on the same thread succeeds."""
    from vlfeat_b200 import workloads as W
    lib = vl.lib()
    _decl(lib)
    pr, mu, cv = W.fv_gmm(64, 32, seed=8)
    x = W.pca_like(1500, 32, seed=9)
    ref, nref = vl.fisher_encode(x, mu, cv, pr, FLAG_IMPROVED)
    res = {}

    def call(enc):
        lib.vl_set_last_error(0, None)
        return lib.vl_fisher_encode(enc.ctypes.data_as(C.c_void_p), 1, mu.ctypes.data_as(C.c_void_p), 32, 64,
                                    cv.ctypes.data_as(C.c_void_p), pr.ctypes.data_as(C.c_void_p),
                                    x.ctypes.data_as(C.c_void_p), x.shape[0], FLAG_IMPROVED)

    def work():
        enc = np.zeros(2 * 64 * 32, np.float32)
        lib.vlb200_debug_fail_allocations(1)
        nt = call(enc)
        res["first"] = (int(nt), lib.vl_get_last_error(), lib.vl_get_last_error_message())
        lib.vlb200_debug_fail_allocations(0)
        nt = call(enc)
        res["second"] = (int(nt), lib.vl_get_last_error(), enc.copy())

    th = threading.Thread(target=work)
    th.start()
    th.join(timeout=120)
    assert not th.is_alive()
    nt, err, msg = res["first"]
    assert nt == 0 and err == VL_ERR_ALLOC, (nt, err, msg)
    assert b"failed" in msg
    nt, err, enc = res["second"]
    assert err == 0 and nt == nref
    assert np.array_equal(enc, ref)


@pytest.fixture(scope="module")
def vlfeat_float():
    from oracle.oracle import Reference
    try:
        return Reference(threads=os.cpu_count() or 1)
    except (FileNotFoundError, OSError):
        return None


@pytest.mark.parametrize("mode", ["exact", "fp32", "bf16"])
def test_nonfinite_descriptors_poison_only_their_image(vl, vlfeat_float, mode):
    import torch
    from vlfeat_b200 import workloads as W
    K, D = 256, 80
    pr, mu, cv = W.fv_gmm(K, D, seed=21)
    counts = np.array([700, 300, 1200, 500])
    offs = np.concatenate([[0], np.cumsum(counts)])
    x = W.pca_like(int(offs[-1]), D, seed=22)
    x[offs[1] + 17, 5] = np.nan      # image 1: one NaN element
    x[offs[2] + 3, 0] = np.inf       # image 2: +inf
    x[offs[2] + 40, 79] = -np.inf    #          and -inf
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    enc = torch.zeros((len(counts), 2 * K * D), device="cuda")
    vl.fisher_encode_batch_device(enc, t(mu), t(cv), t(pr), t(x), offs, FLAG_IMPROVED, mode)
    enc = enc.cpu().numpy()
    clean = W.pca_like(int(offs[-1]), D, seed=22)
    for j in range(len(counts)):
        xj = x[offs[j]:offs[j + 1]]
        if j in (1, 2):
            assert not np.all(np.isfinite(enc[j])), (mode, j)
            if vlfeat_float is not None:
                r, _ = vlfeat_float.fisher(xj, mu, cv, pr, FLAG_IMPROVED)
                assert not np.all(np.isfinite(r)), j
        else:
            e1 = torch.zeros((1, 2 * K * D), device="cuda")
            vl.fisher_encode_batch_device(e1, t(mu), t(cv), t(pr), t(clean[offs[j]:offs[j + 1]]),
                                          np.array([0, counts[j]]), FLAG_IMPROVED, mode)
            assert rel_err(enc[j], e1.cpu().numpy()[0]) < 1e-6, (mode, j)


@pytest.mark.parametrize("mode", ["exact", "fp32"])
def test_em_on_nan_data_gives_nan_loglikelihood(vl, vlfeat_float, mode):
    from vlfeat_b200 import workloads as W
    c = W.config0(scale=0.1)
    data = c["data"].copy()
    data[11, 3] = np.nan
    vl.set_precision(mode)
    try:
        m = vl.GMM(c["D"], c["K"], np.float32)
        m.set_initialization("custom")
        m.set_max_num_iterations(3)
        m.set_covariance_lower_bound(c["lower_bound"])
        m.set_means(c["means"])
        m.set_covariances(c["covs"])
        m.set_priors(c["priors"])
        ll = m.cluster(data)
    finally:
        vl.set_precision("exact")
    assert np.isnan(ll)
    if vlfeat_float is not None:
        r = vlfeat_float.em(data, c["priors"], c["means"], c["covs"], c["lower_bound"], 3)
        assert np.isnan(r["ll"])


def test_misaligned_device_buffers_are_rejected(vl):
    """The tensor-core paths read the data with TMA and bulk copies and store
    row-major posteriors 16 bytes at a time, so device data or posterior
    buffers that do not start 16-byte aligned are refused on the host with
    VL_ERR_BAD_ARG before any launch (never a misaligned access on the GPU);
    the same call on aligned buffers then succeeds, and the exact path, which
    reads and writes element-wise, takes the misaligned buffers."""
    import torch
    from vlfeat_b200 import workloads as W
    K, D, N = 64, 80, 3000
    pr, mu, cv = W.fv_gmm(K, D, seed=21)
    x = W.pca_like(N, D, seed=22)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    P, M, Cv = t(pr), t(mu), t(cv)
    xbuf = torch.zeros(N * D + 4, device="cuda")
    xbuf[1:1 + N * D] = t(x).reshape(-1)
    xm = xbuf[1:1 + N * D].view(N, D)  # starts 4 bytes past a 16-byte boundary
    qbuf = torch.zeros(N * K + 4, device="cuda")
    qm = qbuf[1:1 + N * K].view(N, K)
    q = torch.zeros((N, K), device="cuda")
    with pytest.raises(vl.VLError, match="16-byte aligned"):
        vl.gmm_posteriors_device(q, P, M, Cv, xm, "fp32")
    with pytest.raises(vl.VLError, match="16-byte aligned"):
        vl.gmm_posteriors_device(qm, P, M, Cv, t(x), "fp32")
    ll = vl.gmm_posteriors_device(q, P, M, Cv, t(x), "fp32")
    ref = torch.zeros((N, K), device="cuda")
    ll_exact = vl.gmm_posteriors_device(ref, P, M, Cv, xm, "exact")
    vl.gmm_posteriors_device(qm, P, M, Cv, xm, "exact")
    torch.cuda.synchronize()
    assert np.array_equal(qm.cpu().numpy(), ref.cpu().numpy())
    assert np.max(np.abs(q.cpu().numpy() - ref.cpu().numpy())) < 1e-4
    assert abs(ll - ll_exact) <= 1e-5 * abs(ll_exact)
