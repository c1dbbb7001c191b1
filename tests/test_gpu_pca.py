"""The recognition app's descriptor prologue on the GPU (PCA learning,
projection, renormalisation and the 'xy' geometric extension,
apps/recognition/trainEncoder.m:150-171, encodeImage.m:91-103) against the
float64 NumPy restatement in oracle.oracle.  The library projects on the
tensor cores in scaled fp16x3 (rows on 16-byte boundaries with a multiple of 4
input dimensions) or on the CUDA cores in fp32: relative error bound 1e-5 per
descriptor either way; the PCA (fp64 covariance, Jacobi
eigenvectors) matches to 1e-6 where the eigenvalues are well separated."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _data(N, D, seed):
    """Descriptors with a known, well-separated spectrum."""
    r = np.random.default_rng(seed)
    lam = 4.0 * 0.93 ** np.arange(D)
    Q, _ = np.linalg.qr(r.standard_normal((D, D)))
    x = (r.standard_normal((N, D)) * np.sqrt(lam)[None, :]) @ Q.T + r.uniform(0, 3, D)[None, :]
    return x.astype(np.float32)


@pytest.mark.parametrize("whitening", [False, True])
def test_pca_learn(vl, whitening):
    import torch
    from oracle.oracle import pca_learn
    x = _data(200_000, 128, seed=1)
    P, c, ev = vl.pca_learn_device(torch.from_numpy(x).cuda(), 80, whitening, 0.01 if whitening else 0.0)
    P64, c64, d64 = pca_learn(x, 80, whitening, 0.01 if whitening else 0.0)
    assert np.abs(c.cpu().numpy() - c64).max() < 1e-6 * np.abs(c64).max()
    assert np.abs(ev - d64).max() < 1e-9 * d64.max()
    Pg = P.cpu().numpy().astype(np.float64)
    err = np.abs(Pg - P64).max(1) / np.abs(P64).max(1)
    assert err.max() < 1e-5


@pytest.mark.parametrize("dims", [(128, 80), (128, 64), (96, 96), (64, 30), (50, 20), (128, 128)])
@pytest.mark.parametrize("renorm", [False, True])
def test_pca_project(vl, dims, renorm):
    import torch
    from oracle.oracle import pca_project
    din, dout = dims
    r = np.random.default_rng(din + dout)
    x = _data(20_000, din, seed=2)
    P = (r.standard_normal((dout, din)) / np.sqrt(din)).astype(np.float32)
    c = r.uniform(0, 2, din).astype(np.float32)
    counts = np.array([5000, 0, 7000, 123, 7877])
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    sizes = np.array([[640, 480], [100, 100], [1024, 768], [33, 17], [500, 500]], np.float32)
    img = np.searchsorted(offs, np.arange(len(x)), side="right") - 1
    frames = (r.uniform(0, 1, (len(x), 2)) * sizes[img]).astype(np.float32)
    want = pca_project(x, P, c, renorm, frames, offs, sizes)
    out = torch.full((len(x), dout + 2), float("nan"), device="cuda")
    vl.pca_project_device(out, torch.from_numpy(x).cuda(), torch.from_numpy(P).cuda(), torch.from_numpy(c).cuda(),
                          renorm, torch.from_numpy(frames).cuda(), offs, torch.from_numpy(sizes).cuda())
    got = out.cpu().numpy().astype(np.float64)
    rel = np.linalg.norm(got[:, :dout] - want[:, :dout], axis=1) / np.linalg.norm(want[:, :dout], axis=1)
    assert rel.max() < 1e-5
    assert np.abs(got[:, dout:] - want[:, dout:]).max() < 1e-6
    # Without frames: only the projected block.
    out2 = torch.empty((len(x), dout), device="cuda")
    vl.pca_project_device(out2, torch.from_numpy(x).cuda(), torch.from_numpy(P).cuda(), torch.from_numpy(c).cuda(),
                          renorm)
    assert np.array_equal(out2.cpu().numpy(), out[:, :dout].cpu().numpy())


def test_pca_prologue_then_fisher(vl, restatement):
    """SIFT-like descriptors -> learned PCA (80 dims, whitened) -> renormalise
    -> xy -> improved Fisher vector (exact path), against the float64
    restatement of the same pipeline."""
    import torch
    from oracle.oracle import FLAG_IMPROVED, pca_learn, pca_project
    from vlfeat_b200 import workloads as W
    x = W.sift_like(60_000, 128, seed=3)
    xt = torch.from_numpy(x).cuda()
    P, c, _ = vl.pca_learn_device(xt, 78, True, 0.01)
    offs = np.array([0, 60_000], np.int64)
    sizes = np.array([[640, 480]], np.float32)
    frames = (np.random.default_rng(4).uniform(0, 1, (60_000, 2)) * sizes[0]).astype(np.float32)
    y = torch.empty((60_000, 80), device="cuda")
    vl.pca_project_device(y, xt, P, c, True, torch.from_numpy(frames).cuda(), offs, torch.from_numpy(sizes).cuda())
    y = y.cpu().numpy()
    y64 = pca_project(x, P.cpu().numpy(), c.cpu().numpy(), True, frames, offs, sizes)
    assert np.abs(y - y64).max() < 1e-5
    pr, mu, cv = W.custom_init(y[:20000].astype(np.float32), 64, seed=5)
    enc, nt = vl.fisher_encode(y[20000:], mu, cv, pr, FLAG_IMPROVED)
    ref, nref = restatement.fisher(y64[20000:], mu.astype(np.float64), cv.astype(np.float64),
                                   pr.astype(np.float64), FLAG_IMPROVED)
    from conftest import rel_err
    assert rel_err(enc, ref) < 1e-4


def test_pca_project_unaligned_rows(vl):
    """Rows that do not start on 16-byte boundaries take the CUDA-core kernel
    (plain loads, fp32); aligned rows take the tensor-core kernel (fp16x3).
    Both are within the 1e-5 per-descriptor bound of the float64 restatement,
    and so within 2e-5 of each other."""
    import torch
    r = np.random.default_rng(9)
    x = _data(5000, 128, seed=10)
    P = torch.from_numpy((r.standard_normal((80, 128)) / 11.3).astype(np.float32)).cuda()
    c = torch.from_numpy(r.uniform(0, 2, 128).astype(np.float32)).cuda()
    flat = torch.empty(x.size + 1, device="cuda")
    flat[1:] = torch.from_numpy(x.ravel()).cuda()
    xu = flat[1:].view(5000, 128)
    assert xu.data_ptr() % 16 != 0
    a = torch.empty((5000, 80), device="cuda")
    b = torch.empty((5000, 80), device="cuda")
    vl.pca_project_device(a, xu, P, c, True)
    vl.pca_project_device(b, torch.from_numpy(x).cuda(), P, c, True)
    from oracle.oracle import pca_project
    want = pca_project(x, P.cpu().numpy(), c.cpu().numpy(), True)[:, :80]
    for got in (a, b):
        g = got.cpu().numpy().astype(np.float64)
        assert (np.linalg.norm(g - want, axis=1) / np.linalg.norm(want, axis=1)).max() < 1e-5
    d = (a - b).double().norm(dim=1) / b.double().norm(dim=1)
    assert float(d.max()) < 2e-5


@pytest.mark.parametrize("xscale,pscale", [(1e-20, 1.0), (1e15, 1.0), (1.0, 1e-15), (1.0, 1e15), (3e5, 7e-4),
                                           (1e36, 1e-27), (1e-30, 1e25)])
def test_pca_project_scales(vl, xscale, pscale):
    """The tensor-core projection scales each row of x - c and the matrix P by
    powers of two into fp16's range, so data far outside it (tiny, huge, or a
    mix with a tiny P) stays within the 1e-5 per-descriptor bound; rows equal to
    the centre give zeros (and renormalise to zeros).  The renormalisation
    squares in single precision as the app's MATLAB code does on single
    descriptors, so norms above about 1.8e19 overflow there as in MATLAB; the
    scales here stay below that."""
    import torch
    from oracle.oracle import pca_project
    r = np.random.default_rng(11)
    x = (_data(3_000, 128, seed=12).astype(np.float64) * xscale).astype(np.float32)
    P = (r.standard_normal((80, 128)) / np.sqrt(128) * pscale).astype(np.float32)
    c = (r.uniform(0, 2, 128) * xscale).astype(np.float32)
    x[7] = c  # a row equal to the centre
    for renorm in (False, True):
        want = pca_project(x, P, c, renorm)[:, :80]
        out = torch.empty((len(x), 80), device="cuda")
        vl.pca_project_device(out, torch.from_numpy(x).cuda(), torch.from_numpy(P).cuda(),
                              torch.from_numpy(c).cuda(), renorm)
        got = out.cpu().numpy().astype(np.float64)
        assert np.all(got[7] == 0.0)
        keep = np.arange(len(x)) != 7
        rel = np.linalg.norm(got[keep] - want[keep], axis=1) / np.linalg.norm(want[keep], axis=1)
        assert rel.max() < 1e-5, (renorm, rel.max())
