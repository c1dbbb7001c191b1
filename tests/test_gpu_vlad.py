"""VLAD encoding on the GPU (vl_vlad_encode, vl/vlad.c:163-242) against the
reference's own encodings: bit-exact for every flag combination, in float
and double, through the drop-in host call and the batched device call.

Checkers: the golden fixtures made by VLFeat's CPU code, the NumPy
restatement oracle.oracle.vlad (pinned to those fixtures on the CPU), and, at
larger sizes, VLFeat's own CPU library where it was built (oracle/_ref)."""
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

NAMES = ["hard", "soft", "empty"]


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint8)


def _case(rng, N, D, K, kind, dt):
    x = (rng.standard_normal((N, D)) * 2.0).astype(dt)
    mu = rng.standard_normal((K, D)).astype(dt)
    if kind == "hard":
        a = np.zeros((N, K), dt)
        a[np.arange(N), rng.integers(0, K, N)] = 1
    else:
        a = rng.dirichlet(np.full(K, 0.5), N).astype(dt)
        a[a < 0.01] = 0
        a[::13, K // 2] = -0.5
    return x, mu, a


@pytest.mark.parametrize("flags", range(16))
@pytest.mark.parametrize("tag", ["f", "d"])
@pytest.mark.parametrize("name", NAMES)
def test_vlad_golden(vl, golden, name, tag, flags):
    dt = np.float32 if tag == "f" else np.float64
    x = golden[f"vlad_{name}_data"].astype(dt)
    mu = golden[f"vlad_{name}_means"].astype(dt)
    a = golden[f"vlad_{name}_assign"].astype(dt)
    got = vl.vlad_encode(x, mu, a, flags)
    want = golden[f"vlad_{name}_enc_{tag}_{flags}"]
    assert got.dtype == want.dtype
    assert np.array_equal(_bits(got), _bits(want))


# Shapes over both kernels.  Streaming kernel (row sizes multiples of 16
# bytes, D <= 128): one or several component blocks per image, whole-row and
# per-row copies, partial last block, 1-4 dimension registers per lane, 16
# and 32 components per warp.  Tile kernel (the other shapes): 1, 2, 4 and 8
# dimensions per thread, ragged, K not a multiple of 8.
SHAPES = [(3000, 80, 256, "hard"), (2000, 128, 64, "soft"), (1500, 64, 300, "hard"),
          (1000, 96, 520, "soft"), (700, 8, 4, "soft"), (2500, 32, 36, "hard"), (900, 112, 132, "hard"),
          (700, 5, 3, "hard"), (900, 130, 13, "soft"), (600, 257, 9, "hard"),
          (400, 600, 21, "soft"), (300, 1024, 8, "hard")]


@pytest.mark.parametrize("flags", [0, 3, 8, 15, 4 | 2])
@pytest.mark.parametrize("tag", ["f", "d"])
@pytest.mark.parametrize("shape", SHAPES)
def test_vlad_restatement(vl, shape, tag, flags):
    from oracle.oracle import vlad
    N, D, K, kind = shape
    dt = np.float32 if tag == "f" else np.float64
    x, mu, a = _case(np.random.default_rng(N + D + K), N, D, K, kind, dt)
    got = vl.vlad_encode(x, mu, a, flags)
    assert np.array_equal(_bits(got), _bits(vlad(x, mu, a, flags)))


@pytest.mark.parametrize("tag", ["f", "d"])
def test_vlad_batch_matches_single(vl, tag):
    """The batched device call over uneven images (one of them empty) writes
    each image's vl_vlad_encode bits."""
    import torch
    dt = np.float32 if tag == "f" else np.float64
    tdt = torch.float32 if tag == "f" else torch.float64
    rng = np.random.default_rng(7)
    D, K = 96, 40
    counts = [311, 0, 57, 1024, 5, 640]
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    x, mu, a = _case(rng, int(offs[-1]), D, K, "soft", dt)
    xt = torch.from_numpy(x).cuda()
    at = torch.from_numpy(a).cuda()
    mt = torch.from_numpy(mu).cuda()
    for flags in (0, 15, 2 | 8):
        enc = torch.full((len(counts), K * D), float("nan"), dtype=tdt, device="cuda")
        vl.vlad_encode_batch_device(enc, mt, xt, at, offs, flags)
        torch.cuda.synchronize()
        got = enc.cpu().numpy()
        for j in range(len(counts)):
            lo, hi = offs[j], offs[j + 1]
            want = vl.vlad_encode(x[lo:hi], mu, a[lo:hi], flags)
            assert np.array_equal(_bits(got[j]), _bits(want)), (flags, j)


REF_SO = os.path.join(ROOT, "oracle", "_ref", "libvl_ref.so")


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="VLFeat's CPU library (oracle/_ref) not built")
@pytest.mark.parametrize("kind", ["hard", "soft"])
def test_vlad_reference_large(vl, kind):
    """SIFT-sized dictionary (D=128, K=256 hard / K=64 soft) and 20,000
    descriptors: the GPU encodings equal VLFeat's CPU encodings bit for bit."""
    from oracle.oracle import Reference
    ref = Reference(threads=os.cpu_count() or 1)
    K = 256 if kind == "hard" else 64
    x, mu, a = _case(np.random.default_rng(99), 20000, 128, K, kind, np.float32)
    for flags in (0, 15, 2 | 1):
        want = ref.vlad(x, mu, a, flags)
        got = vl.vlad_encode(x, mu, a, flags)
        assert np.array_equal(_bits(got), _bits(want)), flags


def test_vlad_properties_full_batch(vl):
    """Size-independent checks at a Fisher-bench-sized batch (512 images,
    D=80, K=256, hard assignments): with all normalisations off, the sum of
    the encodings over images equals the encoding of the whole set up to
    float rounding; with the global norm on, every image has unit norm."""
    import torch
    rng = np.random.default_rng(3)
    counts = rng.integers(1000, 8000, 512)
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    N, D, K = int(offs[-1]), 80, 256
    xt = torch.randn(N, D, device="cuda")
    lab = torch.randint(0, K, (N,), device="cuda")
    at = torch.nn.functional.one_hot(lab, K).float()
    mt = torch.randn(K, D, device="cuda")
    enc = torch.empty(len(counts), K * D, device="cuda")
    vl.vlad_encode_batch_device(enc, mt, xt, at, offs, vl.VLAD_UNNORMALIZED)
    whole = torch.empty(1, K * D, device="cuda")
    vl.vlad_encode_batch_device(whole, mt, xt, at, np.array([0, N], np.int64), vl.VLAD_UNNORMALIZED)
    torch.cuda.synchronize()
    s = enc.double().sum(0)
    assert float((s - whole[0].double()).norm() / whole[0].double().norm()) < 1e-5
    vl.vlad_encode_batch_device(enc, mt, xt, at, offs, 0)
    torch.cuda.synchronize()
    n = enc.double().norm(dim=1)
    assert float((n - 1).abs().max()) < 1e-5
