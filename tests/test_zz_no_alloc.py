"""GPU test of vlb200_fisher_encode_noalloc, the entry point for callers that
cannot allocate device memory on the call path (stream capture, services
that forbid allocation after start-up, fixed memory budgets).

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
