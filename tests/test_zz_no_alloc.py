"""GPU test of vlb200_fisher_encode_noalloc, the entry point for callers that
cannot allocate device memory on the call path (services that forbid
allocation after start-up, loops that cannot accept cudaMalloc's implicit
synchronisation, fixed memory budgets).

It is called through the C-ABI and compared with the allocating entry point
vlb200_fisher_encode_device in the same (exact fp32) arithmetic, within the
2e-5 relative tolerance the exact-path tests use, on two calls in a row with
different inputs (the fixed scratch keeps the previous call's contents).
This file is named to run last, so a run that stops at the first failure has
already run every other test; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _bind(lib):
    f = lib.vlb200_fisher_encode_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p,
                  C.c_void_p, C.c_uint64, C.c_int, C.c_void_p, C.c_void_p]
    return f


def _case(seed, K, D, N):
    from vlfeat_b200 import workloads as W
    pr, mu, cv = W.fv_gmm(K, D, seed=seed)
    x = W.pca_like(N, D, seed=seed + 1)
    return pr, mu, cv, x


def test_noalloc_matches_allocating_entry_point(vl):
    import torch
    lib = vl.lib()
    noalloc = _bind(lib)
    stream = torch.cuda.current_stream()
    handle = C.c_void_p(stream.cuda_stream if stream.cuda_stream else 1)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    for seed, (K, D, N), flags in ((1, (64, 32, 3000), vl.FLAG_IMPROVED),
                                   (7, (256, 80, 1234), vl.FLAG_IMPROVED | vl.FLAG_FAST)):
        pr, mu, cv, x = _case(seed, K, D, N)
        mu_t, cv_t, pr_t, x_t = t(mu), t(cv), t(pr), t(x)
        ref = torch.zeros(2 * K * D, device="cuda")
        nt_ref = vl.fisher_encode_device(ref, mu_t, cv_t, pr_t, x_t, flags, "exact", stream)
        enc = torch.full((2 * K * D,), float("nan"), device="cuda")
        nt = torch.zeros(1, dtype=torch.int64, device="cuda")
        rc = noalloc(enc.data_ptr(), mu_t.data_ptr(), D, K, cv_t.data_ptr(), pr_t.data_ptr(),
                     x_t.data_ptr(), N, flags, nt.data_ptr(), handle)
        assert rc == 0, lib.vl_get_last_error_message()
        torch.cuda.synchronize()
        assert rel_err(enc.cpu().numpy(), ref.cpu().numpy()) < 2e-5
        assert int(nt.item()) == nt_ref


def test_noalloc_rejects_oversized_request(vl):
    import torch
    lib = vl.lib()
    noalloc = _bind(lib)
    K, D, N = 64, 32, 5000  # numData above the 4096 limit
    pr, mu, cv, x = _case(3, K, D, N)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    enc = torch.zeros(2 * K * D, device="cuda")
    rc = noalloc(enc.data_ptr(), t(mu).data_ptr(), D, K, t(cv).data_ptr(), t(pr).data_ptr(),
                 t(x).data_ptr(), N, vl.FLAG_IMPROVED, None, None)
    assert rc == 3  # VL_ERR_BAD_ARG
    assert b"exceeds" in lib.vl_get_last_error_message()


def test_noalloc_empty_image_and_null_term_count(vl):
    """numData = 0 gives the zero vector and no terms, as vl/fisher.c:
    383, 450 and 481-484 do (the memset, no prefix, norm floored at 1e-12);
    a NULL numTerms is accepted.  Two calls in a row on the shared scratch."""
    import torch
    lib = vl.lib()
    noalloc = _bind(lib)
    stream = torch.cuda.current_stream()
    handle = C.c_void_p(stream.cuda_stream if stream.cuda_stream else 1)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    K, D = 32, 16
    pr, mu, cv, x = _case(5, K, D, 700)
    mu_t, cv_t, pr_t, x_t = t(mu), t(cv), t(pr), t(x)
    enc = torch.full((2 * K * D,), float("nan"), device="cuda")
    nt = torch.full((1,), 123, dtype=torch.int64, device="cuda")
    rc = noalloc(enc.data_ptr(), mu_t.data_ptr(), D, K, cv_t.data_ptr(), pr_t.data_ptr(),
                 x_t.data_ptr(), 0, vl.FLAG_IMPROVED, nt.data_ptr(), handle)
    assert rc == 0, lib.vl_get_last_error_message()
    torch.cuda.synchronize()
    assert np.array_equal(enc.cpu().numpy(), np.zeros(2 * K * D, np.float32))
    assert int(nt.item()) == 0
    ref = torch.zeros(2 * K * D, device="cuda")
    vl.fisher_encode_device(ref, mu_t, cv_t, pr_t, x_t, vl.FLAG_IMPROVED, "exact", stream)
    enc.fill_(float("nan"))
    rc = noalloc(enc.data_ptr(), mu_t.data_ptr(), D, K, cv_t.data_ptr(), pr_t.data_ptr(),
                 x_t.data_ptr(), x.shape[0], vl.FLAG_IMPROVED, None, handle)
    assert rc == 0, lib.vl_get_last_error_message()
    torch.cuda.synchronize()
    assert rel_err(enc.cpu().numpy(), ref.cpu().numpy()) < 2e-5


def test_noalloc_rejects_sizes_that_wrap_when_signed(vl):
    """Sizes of 2^63 and above are refused before any arithmetic on them."""
    lib = vl.lib()
    noalloc = _bind(lib)
    for n, k, d in ((1 << 63, 8, 8), (16, (1 << 64) - 1, 8), (16, 8, 1 << 63)):
        rc = noalloc(None, None, d, k, None, None, None, n, vl.FLAG_IMPROVED, None, None)
        assert rc == 3  # VL_ERR_BAD_ARG


def test_noalloc_call_is_captured_and_replayed_in_a_cuda_graph(vl):
    """After a first call, the entry point allocates nothing and copies nothing
    from the host: a call captured into a CUDA graph replays on new descriptor
    values and matches the allocating entry point, and a direct call leaves the
    device's free memory unchanged."""
    import torch
    lib = vl.lib()
    noalloc = _bind(lib)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    K, D, N = 128, 64, 2500
    pr, mu, cv, x = _case(11, K, D, N)
    mu_t, cv_t, pr_t, x_t = t(mu), t(cv), t(pr), t(x)
    enc = torch.zeros(2 * K * D, device="cuda")
    nt = torch.zeros(1, dtype=torch.int64, device="cuda")
    flags = vl.FLAG_IMPROVED

    def call(stream):
        return noalloc(enc.data_ptr(), mu_t.data_ptr(), D, K, cv_t.data_ptr(), pr_t.data_ptr(),
                       x_t.data_ptr(), N, flags, nt.data_ptr(), C.c_void_p(stream.cuda_stream))

    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        assert call(side) == 0, lib.vl_get_last_error_message()  # first call: module loading
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    with torch.cuda.stream(side):
        assert call(side) == 0, lib.vl_get_last_error_message()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0

    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        rc = call(torch.cuda.current_stream())
    assert rc == 0, lib.vl_get_last_error_message()
    stream = torch.cuda.current_stream()
    for seed in (12, 13):
        x_t.copy_(t(_case(seed, K, D, N)[3]))
        enc.fill_(float("nan"))
        graph.replay()
        ref = torch.zeros(2 * K * D, device="cuda")
        nt_ref = vl.fisher_encode_device(ref, mu_t, cv_t, pr_t, x_t, flags, "exact", stream)
        torch.cuda.synchronize()
        assert rel_err(enc.cpu().numpy(), ref.cpu().numpy()) < 2e-5
        assert int(nt.item()) == nt_ref
