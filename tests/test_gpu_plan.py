"""GPU tests of the batched Fisher plan (vlb200_fisher_plan_*): the batched
tensor-core encoder bound to one batch layout, its tile configurations, the
autotuner and CUDA-graph replay, through the C-ABI.

Reference: the FP64 C restatement (oracle/); tolerances as in the
tensor-core parity tests (relative L2 error per Fisher vector: FP32 mode 1e-4,
BF16 mode 1e-3; term counts within max(2, 1e-3 n))."""
import numpy as np
import pytest

from conftest import rel_err
from oracle.oracle import FLAG_IMPROVED

pytestmark = pytest.mark.gpu

TOL = {"fp32": 1e-4, "bf16": 1e-3}
K, D = 256, 80
COUNTS = np.array([0, 1, 5, 127, 128, 129, 3000, 0, 9000, 17, 20000, 250])


def _t(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


@pytest.fixture(scope="module")
def batch():
    from vlfeat_b200 import workloads as W
    pr, mu, cv = W.fv_gmm(K, D, seed=9)
    offs = np.concatenate([[0], np.cumsum(COUNTS)]).astype(np.int64)
    x = W.pca_like(int(offs[-1]), D, seed=10)
    return pr, mu, cv, offs, x


@pytest.fixture(scope="module")
def refs(batch, restatement):
    pr, mu, cv, offs, x = batch
    out = []
    for j in range(len(COUNTS)):
        e, n = restatement.fisher(x[offs[j]:offs[j + 1]].astype(np.float64), mu.astype(np.float64),
                                  cv.astype(np.float64), pr.astype(np.float64), FLAG_IMPROVED)
        out.append((e, n))
    return out


def _plan(vl, batch, mode):
    pr, mu, cv, offs, x = batch
    p = vl.FisherPlan(D, K, offs, FLAG_IMPROVED, mode)
    g = (_t(mu), _t(cv), _t(pr))
    p.set_gmm(*g)
    return p, g


def _out(n):
    import torch
    return (torch.zeros((n, 2 * K * D), device="cuda"), torch.zeros(n, dtype=torch.int64, device="cuda"))


def _check(enc, nt, refs, mode):
    enc = enc.cpu().numpy()
    nt = nt.cpu().numpy()
    for j, (e, n) in enumerate(refs):
        if COUNTS[j] == 0:
            assert np.all(enc[j] == 0) and nt[j] == 0
        else:
            assert rel_err(enc[j], e) < TOL[mode], j
            assert abs(int(nt[j]) - n) <= max(2, 1e-3 * n), j


@pytest.mark.parametrize("mode", ["fp32", "bf16"])
def test_plan_matches_batch_api(vl, batch, refs, mode):
    """The default configuration runs the same launches as the batched call:
    identical bits."""
    pr, mu, cv, offs, x = batch
    p, g = _plan(vl, batch, mode)
    xt = _t(x)
    enc, nt = _out(len(COUNTS))
    p.execute(enc, xt, nt)
    enc2, nt2 = _out(len(COUNTS))
    vl.fisher_encode_batch_device(enc2, g[0], g[1], g[2], xt, offs, FLAG_IMPROVED, mode, nt2)
    assert p.status() == 0
    assert np.array_equal(enc.cpu().numpy(), enc2.cpu().numpy())
    assert np.array_equal(nt.cpu().numpy(), nt2.cpu().numpy())
    _check(enc, nt, refs, mode)


@pytest.mark.parametrize("mode", ["fp32", "bf16"])
@pytest.mark.parametrize("cfg", [
    dict(item_rows=2048),
    dict(item_rows=4096, stats_mt=1),
    dict(estep_stages=2, stats_stages=2),
    dict(row_budget=4096),          # one E-step launch per few images
    dict(item_rows=128, row_budget=1),  # one image per chunk, 128-row items
])
def test_plan_configs(vl, batch, refs, mode, cfg):
    p, g = _plan(vl, batch, mode)
    p.set_config(**cfg)
    got = p.get_config()
    for k, v in cfg.items():
        assert got[k] == v
    enc, nt = _out(len(COUNTS))
    p.execute(enc, _t(batch[4]), nt)
    assert p.status() == 0
    _check(enc, nt, refs, mode)


def test_plan_graph_replay(vl, batch, refs):
    """A captured encode replays to the same bits as execute, and reads the
    current contents of its bound buffers at every launch."""
    import torch
    pr, mu, cv, offs, x = batch
    p, g = _plan(vl, batch, "bf16")
    s = torch.cuda.Stream()
    xt = _t(x)
    enc, nt = _out(len(COUNTS))
    with torch.cuda.stream(s):
        p.capture(enc, xt, nt, stream=s)
        enc.zero_()
        nt.zero_()
        l0 = vl.launch_count()
        p.launch(stream=s)
        p.launch(stream=s)
        launches = vl.launch_count() - l0
    s.synchronize()
    assert launches > 0 and launches % 2 == 0
    enc_ref, nt_ref = _out(len(COUNTS))
    p.execute(enc_ref, xt, nt_ref)
    torch.cuda.synchronize()
    assert np.array_equal(enc.cpu().numpy(), enc_ref.cpu().numpy())
    assert np.array_equal(nt.cpu().numpy(), nt_ref.cpu().numpy())
    _check(enc, nt, refs, "bf16")
    # New data in the same buffer: the replay encodes it.
    x2 = x[::-1].copy()
    with torch.cuda.stream(s):
        xt.copy_(_t(x2))
        p.launch(stream=s)
    s.synchronize()
    xt2 = _t(x2)
    enc2, nt2 = _out(len(COUNTS))
    p.execute(enc2, xt2, nt2)
    torch.cuda.synchronize()
    assert np.array_equal(enc.cpu().numpy(), enc2.cpu().numpy())
    assert p.status() == 0


def test_plan_autotune(vl, batch, refs):
    pr, mu, cv, offs, x = batch
    p, g = _plan(vl, batch, "fp32")
    enc, nt = _out(len(COUNTS))
    xt = _t(x)
    ms = p.autotune(enc, xt, nt)
    assert ms > 0
    cfg = p.get_config()
    assert cfg["item_rows"] in (4096, 8192, 16384) and cfg["stats_mt"] in (0, 1)
    enc.zero_()
    p.execute(enc, xt, nt)
    assert p.status() == 0
    _check(enc, nt, refs, "fp32")


def test_plan_rejects(vl, batch):
    pr, mu, cv, offs, x = batch
    with pytest.raises(vl.VLError):
        vl.FisherPlan(D, K, offs, FLAG_IMPROVED, "exact")  # the plan is the tensor-core encoder
    with pytest.raises(vl.VLError):
        vl.FisherPlan(96, K, offs, FLAG_IMPROVED, "bf16")  # unsupported dimension
    p = vl.FisherPlan(D, K, offs, FLAG_IMPROVED, "bf16")
    enc, nt = _out(len(COUNTS))
    with pytest.raises(vl.VLError):
        p.execute(enc, _t(x), nt)  # no GMM bound yet
    with pytest.raises(vl.VLError):
        p.set_config(item_rows=100)  # not a multiple of 128
    with pytest.raises(vl.VLError):
        p.launch()  # nothing captured


@pytest.mark.parametrize("pinned", [True, False])
def test_plan_execute_host(vl, batch, refs, pinned):
    """Host buffers in and out, copies overlapped chunk by chunk.  The
    host-buffer layout cuts the batch into more E-step chunks than the device
    execute; the statistics kernel groups rows into MMA k-steps by their
    position in the chunk's posterior image, so the fp32 accumulation order,
    not the arithmetic, changes: results agree to 1e-6 relative, term counts
    exactly."""
    import torch
    pr, mu, cv, offs, x = batch
    p, g = _plan(vl, batch, "bf16")
    xh = torch.from_numpy(x.copy())
    enc_h = torch.zeros((len(COUNTS), 2 * K * D))
    nt_h = torch.zeros(len(COUNTS), dtype=torch.int64)
    if pinned:
        xh, enc_h, nt_h = xh.pin_memory(), enc_h.pin_memory(), nt_h.pin_memory()
    p.execute_host(enc_h, xh, nt_h)
    enc, nt = _out(len(COUNTS))
    p.execute(enc, _t(x), nt)
    torch.cuda.synchronize()
    dev = enc.cpu().numpy()
    for j in range(len(COUNTS)):
        assert rel_err(enc_h.numpy()[j], dev[j]) <= 1e-6, j
    assert np.array_equal(nt_h.numpy(), nt.cpu().numpy())
    # numpy buffers, no term counts, a second call reusing the plan's buffers:
    # the same layout as the first call, so the same bits.
    enc_np = np.zeros((len(COUNTS), 2 * K * D), np.float32)
    p.execute_host(enc_np, np.ascontiguousarray(x))
    assert np.array_equal(enc_np, enc_h.numpy())
    _check(torch.from_numpy(enc_np), nt, refs, "bf16")
