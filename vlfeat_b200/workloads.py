"""Seeded synthetic workloads with the shapes of the benchmarked configurations.

No public dataset is used: every input here is drawn from NumPy's PCG64
generator with a fixed seed, so the same call returns the same bytes on every
machine.  Layouts follow VLFeat: one descriptor per row (``data[i, d]``),
``means/covs[k, d]``, ``priors[k]`` (vl/gmm.c:711-798).

Generators (sizes are parameters; the defaults are the benchmark sizes):

* :func:`mixture_data` -- K0-component diagonal mixture, means ~ N(0, 4 I),
  per-dimension sigma ~ U[lo, hi] (variance sigma^2), priors ~ Dirichlet(1).
* :func:`sift_like` -- SIFT-shaped descriptors: bins ~ Gamma(0.5, 1),
  L2-normalise, clip at 0.2, renormalise, x512, round, clamp to [0, 255].
* :func:`pca_like` -- N(0, diag(lambda)), lambda_i = (1+i)^-0.8.
* :func:`image_counts` -- per-image descriptor counts ~ lognormal(median, s)
  clipped to [lo, hi].
* :func:`custom_init` -- the custom EM initialisation: K seeded distinct rows
  as means, unbiased global variance (vl/gmm.c:1376-1413) for every
  component, uniform priors.
* :func:`fv_gmm` -- a fixed seeded GMM for Fisher encoding of PCA-like data.
"""
from __future__ import annotations

import numpy as np


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def mixture_params(K0: int, D: int, seed: int, sigma_lo=0.5, sigma_hi=2.0):
    r = _rng(seed)
    means = r.normal(0.0, 2.0, size=(K0, D))
    sigma = r.uniform(sigma_lo, sigma_hi, size=(K0, D))
    priors = r.dirichlet(np.ones(K0))
    return means, sigma, priors


def mixture_data(N: int, D: int, K0: int, seed: int, sigma_lo=0.5, sigma_hi=2.0,
                 params_seed: int | None = None, dtype=np.float32):
    """Draw N points from a seeded K0-component diagonal Gaussian mixture."""
    means, sigma, priors = mixture_params(K0, D, seed if params_seed is None else params_seed,
                                          sigma_lo, sigma_hi)
    r = _rng(seed + 7919)
    comp = r.choice(K0, size=N, p=priors)
    x = means[comp] + sigma[comp] * r.standard_normal((N, D))
    return x.astype(dtype)


def sift_like(N: int, D: int = 128, seed: int = 0, dtype=np.float32):
    r = _rng(seed)
    x = r.gamma(0.5, 1.0, size=(N, D))
    x /= np.maximum(np.linalg.norm(x, axis=1, keepdims=True), 1e-12)
    np.minimum(x, 0.2, out=x)
    x /= np.maximum(np.linalg.norm(x, axis=1, keepdims=True), 1e-12)
    x = np.clip(np.round(x * 512.0), 0, 255)
    return x.astype(dtype)


def pca_lambdas(D: int = 80):
    return (1.0 + np.arange(D)) ** -0.8


def pca_like(N: int, D: int = 80, seed: int = 0, dtype=np.float32):
    r = _rng(seed)
    return (r.standard_normal((N, D)) * np.sqrt(pca_lambdas(D))[None, :]).astype(dtype)


def image_counts(num_images: int, seed: int, median=3000.0, sigma=1.0, lo=200, hi=20000):
    r = _rng(seed)
    c = np.exp(np.log(median) + sigma * r.standard_normal(num_images))
    return np.clip(np.round(c), lo, hi).astype(np.int64)


def custom_init(data: np.ndarray, K: int, seed: int):
    """Means = K seeded distinct rows; covariances = unbiased global variance
    (N-1 denominator, vl/gmm.c:1409) for every component; priors = 1/K."""
    r = _rng(seed)
    N, D = data.shape
    idx = r.choice(N, size=K, replace=False)
    dt = data.dtype
    means = data[idx].astype(dt)
    var = data.astype(np.float64).var(axis=0, ddof=1) if N > 1 else np.zeros(D)
    covs = np.tile(var.astype(dt), (K, 1))
    priors = np.full(K, 1.0 / K, dt)
    return priors, means, covs


def fv_gmm(K: int = 256, D: int = 80, seed: int = 11, dtype=np.float32):
    """Fixed GMM for PCA-like data: means ~ N(0, diag(lambda)/2),
    sigma2_kd = lambda_d * U[0.3, 0.8], priors ~ Dirichlet(2 * 1)."""
    r = _rng(seed)
    lam = pca_lambdas(D)
    means = r.standard_normal((K, D)) * np.sqrt(lam / 2)[None, :]
    covs = lam[None, :] * r.uniform(0.3, 0.8, size=(K, D))
    priors = r.dirichlet(np.full(K, 2.0))
    return priors.astype(dtype), means.astype(dtype), covs.astype(dtype)


# --- benchmarked configurations -------------------------------------------

def config0(scale: float = 1.0):
    """EM + FV, CPU-runnable: N=50,000, D=64, 64-component mixture, K=64,
    10 iterations, improved FV of 2,000 separate descriptors."""
    N = max(64, int(50000 * scale))
    D, K = 64, 64
    data = mixture_data(N, D, 64, seed=100, params_seed=100)
    fv_data = mixture_data(max(1, int(2000 * scale)), D, 64, seed=101, params_seed=100)
    priors, means, covs = custom_init(data, K, seed=102)
    return dict(data=data, fv_data=fv_data, priors=priors, means=means, covs=covs,
                K=K, D=D, iters=10, lower_bound=1e-4)


def config1(N: int = 1_000_000, K: int = 256, iters: int = 20):
    """SIFT-shaped EM at scale; variance floor = 1e-4 x max global variance
    (the scalar bound the reference's recognition app uses,
    apps/recognition/trainEncoder.m:195-199)."""
    data = sift_like(N, 128, seed=200)
    priors, means, covs = custom_init(data, K, seed=201)
    lb = 1e-4 * float(data.astype(np.float64).var(axis=0, ddof=1).max())
    return dict(data=data, priors=priors, means=means, covs=covs, K=K, D=128,
                iters=iters, lower_bound=lb)


def config2_counts(num_images: int = 4096):
    return image_counts(num_images, seed=300)


def config3_params(K: int = 1024, D: int = 80, seed: int = 500):
    """Learned-router configuration: a seeded K-component diagonal mixture with
    the config-0 generator and sigma ~ U[0.3, 1.5] (means ~ N(0, 4 I), priors
    ~ Dirichlet(1)); the GMM of the E-step is the mixture itself.  Returns
    float32 (priors, means, variances)."""
    means, sigma, priors = mixture_params(K, D, seed, 0.3, 1.5)
    return (priors.astype(np.float32), means.astype(np.float32), (sigma ** 2).astype(np.float32))


def config3_data_device(n: int, params, seed: int, device="cuda", chunk: int = 1 << 22):
    """n float32 rows of the config-3 mixture drawn on the GPU with a seeded
    torch generator (component ~ priors, then mean + sigma * N(0, 1))."""
    import torch
    pr, mu, cv = params
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    p = torch.from_numpy(pr.astype(np.float64)).to(device)
    m = torch.from_numpy(mu).to(device)
    s = torch.from_numpy(np.sqrt(cv)).to(device)
    out = torch.empty((n, mu.shape[1]), dtype=torch.float32, device=device)
    for i in range(0, n, chunk):
        b = min(chunk, n - i)
        c = torch.multinomial(p, b, replacement=True, generator=g)
        out[i:i + b] = m[c] + s[c] * torch.randn((b, mu.shape[1]), generator=g, device=device)
    return out


def sift_like_device(n: int, D: int = 128, seed: int = 0, device="cuda", chunk: int = 1 << 21):
    """SIFT-shaped descriptors as :func:`sift_like` (Gamma(0.5, 1) bins,
    L2-normalise, clip at 0.2, renormalise, x512, round, clamp to [0, 255]),
    drawn on the GPU from torch's generator seeded with `seed` (for sizes
    where NumPy on the host is too slow; not the same bytes as sift_like)."""
    import torch
    out = torch.empty((n, D), dtype=torch.float32, device=device)
    torch.cuda.manual_seed(seed)
    conc = torch.full((min(chunk, n), D), 0.5, device=device)
    for i in range(0, n, chunk):
        b = min(chunk, n - i)
        x = torch._standard_gamma(conc[:b])
        x /= x.norm(dim=1, keepdim=True).clamp_min(1e-12)
        x.clamp_(max=0.2)
        x /= x.norm(dim=1, keepdim=True).clamp_min(1e-12)
        out[i:i + b] = (x * 512.0).round_().clamp_(0, 255)
    return out


def custom_init_device(x, K: int, seed: int):
    """:func:`custom_init` for a CUDA tensor: K seeded distinct rows as means,
    the unbiased global variance (N - 1, vl/gmm.c:1409, accumulated in f64)
    for every component, uniform priors.  Returns float32 NumPy arrays and
    the variance floor 1e-4 x the largest global variance."""
    N, D = x.shape
    idx = _rng(seed).choice(N, size=K, replace=False)
    means = x[idx].cpu().numpy().astype(np.float32)
    s1 = np.zeros(D)
    s2 = np.zeros(D)
    step = 1 << 22
    for i in range(0, N, step):
        xb = x[i:i + step].double()
        s1 += xb.sum(0).cpu().numpy()
    mean = s1 / N
    import torch
    mt = torch.from_numpy(mean).to(x.device)
    for i in range(0, N, step):
        s2 += ((x[i:i + step].double() - mt) ** 2).sum(0).cpu().numpy()
    var = s2 / (N - 1)
    covs = np.tile(var.astype(np.float32), (K, 1))
    priors = np.full(K, 1.0 / K, np.float32)
    return priors, means, covs, 1e-4 * float(var.max())
