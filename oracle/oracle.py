"""ctypes bindings for the two CPU checkers of the GMM-EM / Fisher-vector path.

TEST INFRASTRUCTURE ONLY.  Only the tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this module; the product library never
does.

* :class:`Restatement` drives ``oracle/liboracle.so``, the C restatement of the
  reference algorithm (``vlgmm_oracle_impl.h``; every function cites the
  reference lines it follows).
* :class:`Reference` drives ``oracle/_ref/libvl_ref.so``, VLFeat's own CPU
  code compiled from the reference sources by ``oracle/Makefile`` (target
  ``ref``), through VLFeat's unchanged C API (vl/gmm.h:40-145,
  vl/fisher.h:48-54, vl/vlad.h:45-50).  It exists only where that library was
  built.
* :func:`vlad` restates VLAD encoding (vl/vlad.c:163-242) in NumPy.
* :func:`pca_learn` and :func:`pca_project` restate the recognition app's
  descriptor prologue (apps/recognition/trainEncoder.m:150-171,
  encodeImage.m:91-103), MATLAB code with no compiled form here: the
  restatement follows the .m files and is not pinned to outputs of them.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libvl_ref.so")

VL_TYPE_FLOAT = 1
VL_TYPE_DOUBLE = 2
FLAG_SQUARE_ROOT = 1 << 0
FLAG_NORMALIZED = 1 << 1
FLAG_IMPROVED = FLAG_SQUARE_ROOT | FLAG_NORMALIZED
FLAG_FAST = 1 << 2
VLAD_NORMALIZE_COMPONENTS = 1 << 0  # vl/vlad.h:23-26
VLAD_SQUARE_ROOT = 1 << 1
VLAD_UNNORMALIZED = 1 << 2
VLAD_NORMALIZE_MASS = 1 << 3
VL_GMM_KMEANS = 0  # VlGMMKMeans, vl/gmm.h:21-26
VL_GMM_RAND = 1    # VlGMMRand
VL_GMM_CUSTOM = 2  # VlGMMCustom

_vp = C.c_void_p
_sz = C.c_uint64
_dp = C.POINTER(C.c_double)


def _ptr(a):
    return a.ctypes.data_as(_vp) if a is not None else None


def _sfx(dtype):
    return "_f" if np.dtype(dtype) == np.float32 else "_d"


def build(ref: bool = False) -> None:
    """Compile the restatement (and, with ``ref``, the reference library)."""
    subprocess.check_call(["make", "-s", "-C", HERE], stdout=subprocess.DEVNULL)
    if ref:
        subprocess.check_call(["make", "-s", "-C", HERE, "ref"], stdout=subprocess.DEVNULL)


class Restatement:
    """The C restatement (float and double instantiations)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build()
        self.lib = C.CDLL(path)
        for s in ("_f", "_d"):
            f = getattr(self.lib, "orc_posteriors_" + s)
            f.restype = C.c_double
            f.argtypes = [_vp, _sz, _sz, _vp, _vp, _sz, _vp, _vp]
            f = getattr(self.lib, "orc_maximization_" + s)
            f.restype = None
            f.argtypes = [_vp, _vp, _vp, _vp, _vp, _sz, _sz, _sz, _vp]
            f = getattr(self.lib, "orc_restart_empty_modes_" + s)
            f.restype = _sz
            f.argtypes = [_vp, _vp, _vp, _vp, _vp, _sz, _sz, _sz, _vp]
            f = getattr(self.lib, "orc_em_" + s)
            f.restype = C.c_double
            f.argtypes = [_vp, _vp, _vp, _vp, _vp, _sz, _sz, _sz, _vp, _sz,
                          C.POINTER(_sz), C.POINTER(_sz), _vp]
            f = getattr(self.lib, "orc_fisher_" + s)
            f.restype = _sz
            f.argtypes = [_vp, _vp, _sz, _sz, _vp, _vp, _vp, _sz, C.c_int]
            f = getattr(self.lib, "orc_global_variance_" + s)
            f.restype = None
            f.argtypes = [_vp, _vp, _sz, _sz]

    def posteriors(self, data, priors, means, covs):
        dt = data.dtype
        N, D = data.shape
        K = priors.shape[0]
        post = np.zeros((N, K), dt)
        ll = getattr(self.lib, "orc_posteriors_" + _sfx(dt))(
            _ptr(post), K, N, _ptr(np.ascontiguousarray(priors, dt)),
            _ptr(np.ascontiguousarray(means, dt)), D,
            _ptr(np.ascontiguousarray(covs, dt)), _ptr(np.ascontiguousarray(data)))
        return post, ll

    def maximization(self, post, data, priors, means, covs, lb):
        dt = data.dtype
        N, D = data.shape
        K = priors.shape[0]
        pr, mu, cv = priors.astype(dt).copy(), means.astype(dt).copy(), covs.astype(dt).copy()
        lb = np.ascontiguousarray(lb, np.float64)
        getattr(self.lib, "orc_maximization_" + _sfx(dt))(
            _ptr(pr), _ptr(mu), _ptr(cv), _ptr(np.ascontiguousarray(post, dt)),
            _ptr(np.ascontiguousarray(data)), N, D, K, _ptr(lb))
        return pr, mu, cv

    def em(self, data, priors, means, covs, lb, max_iter):
        """EM from a custom initialisation; returns a dict of final state."""
        dt = data.dtype
        N, D = data.shape
        K = priors.shape[0]
        pr, mu, cv = priors.astype(dt).copy(), means.astype(dt).copy(), covs.astype(dt).copy()
        post = np.zeros((N, K), dt)
        lb = np.ascontiguousarray(np.broadcast_to(np.asarray(lb, np.float64), (D,)))
        it, rs = _sz(0), _sz(0)
        trace = np.zeros(max_iter + 2, np.float64)
        ll = getattr(self.lib, "orc_em_" + _sfx(dt))(
            _ptr(pr), _ptr(mu), _ptr(cv), _ptr(post), _ptr(np.ascontiguousarray(data)),
            N, D, K, _ptr(lb), max_iter, C.byref(it), C.byref(rs), _ptr(trace))
        return dict(ll=ll, priors=pr, means=mu, covs=cv, posteriors=post,
                    iterations=int(it.value), restarts=int(rs.value),
                    ll_trace=trace[: int(it.value) + 1])

    def fisher(self, data, means, covs, priors, flags):
        dt = data.dtype
        N, D = data.shape
        K = priors.shape[0]
        enc = np.zeros(2 * K * D, dt)
        nt = getattr(self.lib, "orc_fisher_" + _sfx(dt))(
            _ptr(enc), _ptr(np.ascontiguousarray(means, dt)), D, K,
            _ptr(np.ascontiguousarray(covs, dt)), _ptr(np.ascontiguousarray(priors, dt)),
            _ptr(np.ascontiguousarray(data)), N, int(flags))
        return enc, int(nt)

    def global_variance(self, data):
        N, D = data.shape
        var = np.zeros(D, data.dtype)
        getattr(self.lib, "orc_global_variance_" + _sfx(data.dtype))(
            _ptr(var), _ptr(np.ascontiguousarray(data)), N, D)
        return var


class Reference:
    """VLFeat's own CPU implementation through its unchanged C API."""

    def __init__(self, path: str = REF_SO, threads: int | None = None, simd: bool = True):
        if not os.path.exists(path):
            raise FileNotFoundError(
                f"{path} not built; run `make -C oracle ref` where the reference sources exist")
        self.lib = L = C.CDLL(path)
        L.vl_gmm_new.restype = _vp
        L.vl_gmm_new.argtypes = [C.c_uint32, _sz, _sz]
        L.vl_gmm_delete.argtypes = [_vp]
        for n in ("means", "covariances", "priors"):
            getattr(L, "vl_gmm_set_" + n).argtypes = [_vp, _vp]
            getattr(L, "vl_gmm_get_" + n).argtypes = [_vp]
            getattr(L, "vl_gmm_get_" + n).restype = _vp
        L.vl_gmm_get_posteriors.argtypes = [_vp]
        L.vl_gmm_get_posteriors.restype = _vp
        L.vl_gmm_set_initialization.argtypes = [_vp, C.c_int]
        L.vl_gmm_init_with_kmeans.restype = None
        L.vl_gmm_init_with_kmeans.argtypes = [_vp, _vp, _sz, _vp]
        L.vl_gmm_set_max_num_iterations.argtypes = [_vp, _sz]
        L.vl_gmm_set_num_repetitions.argtypes = [_vp, _sz]
        L.vl_gmm_set_verbosity.argtypes = [_vp, C.c_int]
        L.vl_gmm_set_covariance_lower_bounds.argtypes = [_vp, _vp]
        L.vl_gmm_set_covariance_lower_bound.argtypes = [_vp, C.c_double]
        L.vl_gmm_cluster.restype = C.c_double
        L.vl_gmm_cluster.argtypes = [_vp, _vp, _sz]
        L.vl_gmm_em.restype = C.c_double
        L.vl_gmm_em.argtypes = [_vp, _vp, _sz]
        L.vl_gmm_get_loglikelihood.restype = C.c_double
        L.vl_gmm_get_loglikelihood.argtypes = [_vp]
        L.vl_fisher_encode.restype = _sz
        L.vl_fisher_encode.argtypes = [_vp, C.c_uint32, _vp, _sz, _sz, _vp, _vp, _vp, _sz, C.c_int]
        for s in ("_f", "_d"):
            f = getattr(L, "vl_get_gmm_data_posteriors" + s)
            f.restype = C.c_double
            f.argtypes = [_vp, _sz, _sz, _vp, _vp, _sz, _vp, _vp]
        L.vl_vlad_encode.restype = None
        L.vl_vlad_encode.argtypes = [_vp, C.c_uint32, _vp, _sz, _sz, _vp, _sz, _vp, C.c_int]
        L.vl_set_num_threads.argtypes = [_sz]
        L.vl_get_max_threads.restype = _sz
        L.vl_set_simd_enabled.argtypes = [C.c_int]
        L.vl_get_simd_enabled.restype = C.c_int
        L.vl_get_rand.restype = _vp
        L.vl_rand_seed.argtypes = [_vp, C.c_uint32]
        L.vl_rand_uint32.restype = C.c_uint32
        L.vl_rand_uint32.argtypes = [_vp]
        L.vl_cpu_has_avx.restype = C.c_int
        L.vl_cpu_has_sse2.restype = C.c_int
        if threads is not None:
            self.set_threads(threads)
        L.vl_set_simd_enabled(1 if simd else 0)

    def set_threads(self, n: int) -> None:
        self.lib.vl_set_num_threads(int(n))

    @property
    def threads(self) -> int:
        return int(self.lib.vl_get_max_threads())

    def posteriors(self, data, priors, means, covs):
        dt = data.dtype
        N, D = data.shape
        K = priors.shape[0]
        post = np.zeros((N, K), dt)
        ll = getattr(self.lib, "vl_get_gmm_data_posteriors" + _sfx(dt))(
            _ptr(post), K, N, _ptr(np.ascontiguousarray(priors, dt)),
            _ptr(np.ascontiguousarray(means, dt)), D,
            _ptr(np.ascontiguousarray(covs, dt)), _ptr(np.ascontiguousarray(data)))
        return post, ll

    def em(self, data, priors, means, covs, lb, max_iter, want_posteriors=False):
        """vl_gmm_cluster with VlGMMCustom initialisation (vl/gmm.c:1557-1648)."""
        L = self.lib
        dt = data.dtype
        N, D = data.shape
        K = priors.shape[0]
        typ = VL_TYPE_FLOAT if dt == np.float32 else VL_TYPE_DOUBLE
        g = L.vl_gmm_new(typ, D, K)
        try:
            L.vl_gmm_set_initialization(g, VL_GMM_CUSTOM)
            L.vl_gmm_set_max_num_iterations(g, int(max_iter))
            lbv = np.ascontiguousarray(np.broadcast_to(np.asarray(lb, np.float64), (D,)))
            L.vl_gmm_set_covariance_lower_bounds(g, _ptr(lbv))
            L.vl_gmm_set_means(g, _ptr(np.ascontiguousarray(means, dt)))
            L.vl_gmm_set_covariances(g, _ptr(np.ascontiguousarray(covs, dt)))
            L.vl_gmm_set_priors(g, _ptr(np.ascontiguousarray(priors, dt)))
            dat = np.ascontiguousarray(data)
            ll = L.vl_gmm_cluster(g, _ptr(dat), N)
            ct = C.c_float if dt == np.float32 else C.c_double

            def grab(p, n):
                return np.ctypeslib.as_array(C.cast(p, C.POINTER(ct)), shape=(n,)).copy()

            out = dict(ll=ll, priors=grab(L.vl_gmm_get_priors(g), K),
                       means=grab(L.vl_gmm_get_means(g), K * D).reshape(K, D),
                       covs=grab(L.vl_gmm_get_covariances(g), K * D).reshape(K, D))
            if want_posteriors:
                out["posteriors"] = grab(L.vl_gmm_get_posteriors(g), N * K).reshape(N, K)
            return out
        finally:
            L.vl_gmm_delete(g)

    def seed(self, s: int) -> None:
        """vl_rand_seed on the calling thread's generator (vl/random.c:109-127)."""
        self.lib.vl_rand_seed(self.lib.vl_get_rand(), int(s))

    def rand_init(self, data, K, seed, max_iter=0, lb=1e-4, init=VL_GMM_RAND):
        """vl_gmm_cluster with VlGMMRand (vl/gmm.c:1416-1443) or, with
        init=VL_GMM_KMEANS, VlGMMKMeans initialisation (vl/gmm.c:1315-1370)
        after seeding the thread's generator; max_iter=0 leaves the initial
        parameters (one E-step, no M-step)."""
        L = self.lib
        dt = data.dtype
        N, D = data.shape
        g = L.vl_gmm_new(VL_TYPE_FLOAT if dt == np.float32 else VL_TYPE_DOUBLE, D, K)
        try:
            L.vl_gmm_set_initialization(g, int(init))
            L.vl_gmm_set_max_num_iterations(g, int(max_iter))
            L.vl_gmm_set_covariance_lower_bound(g, float(lb))
            self.seed(seed)
            dat = np.ascontiguousarray(data)
            ll = L.vl_gmm_cluster(g, _ptr(dat), N)
            ct = C.c_float if dt == np.float32 else C.c_double

            def grab(p, n):
                return np.ctypeslib.as_array(C.cast(p, C.POINTER(ct)), shape=(n,)).copy()

            return dict(ll=ll, priors=grab(L.vl_gmm_get_priors(g), K),
                        means=grab(L.vl_gmm_get_means(g), K * D).reshape(K, D),
                        covs=grab(L.vl_gmm_get_covariances(g), K * D).reshape(K, D))
        finally:
            L.vl_gmm_delete(g)

    def kmeans_init(self, data, K, seed, lb=1e-4):
        """vl_gmm_init_with_kmeans (vl/gmm.c:1315-1370) after seeding the
        thread's generator: the GMM parameters of the one-hot M-step, the
        k-means assignment of every row (the one-hot posteriors) and the
        generator's next draw (which shows how many draws the initialisation
        took)."""
        L = self.lib
        dt = data.dtype
        N, D = data.shape
        g = L.vl_gmm_new(VL_TYPE_FLOAT if dt == np.float32 else VL_TYPE_DOUBLE, D, K)
        try:
            L.vl_gmm_set_covariance_lower_bound(g, float(lb))
            self.seed(seed)
            dat = np.ascontiguousarray(data)
            L.vl_gmm_init_with_kmeans(g, _ptr(dat), N, None)
            nxt = int(L.vl_rand_uint32(L.vl_get_rand()))
            ct = C.c_float if dt == np.float32 else C.c_double

            def grab(p, n):
                return np.ctypeslib.as_array(C.cast(p, C.POINTER(ct)), shape=(n,)).copy()

            post = grab(L.vl_gmm_get_posteriors(g), N * K).reshape(N, K)
            return dict(priors=grab(L.vl_gmm_get_priors(g), K),
                        means=grab(L.vl_gmm_get_means(g), K * D).reshape(K, D),
                        covs=grab(L.vl_gmm_get_covariances(g), K * D).reshape(K, D),
                        assign=np.argmax(post, axis=1).astype(np.int64), next_draw=nxt)
        finally:
            L.vl_gmm_delete(g)

    def distance_lanes(self) -> int:
        """Lanes of the reference's squared-L2 kernel on this host for float
        data (vl/mathop.c:489-510): 8 (AVX), 4 (SSE2) or 1."""
        if not self.lib.vl_get_simd_enabled():
            return 1
        return 8 if self.lib.vl_cpu_has_avx() else (4 if self.lib.vl_cpu_has_sse2() else 1)

    def fisher(self, data, means, covs, priors, flags):
        dt = data.dtype
        N, D = data.shape
        K = priors.shape[0]
        typ = VL_TYPE_FLOAT if dt == np.float32 else VL_TYPE_DOUBLE
        enc = np.zeros(2 * K * D, dt)
        nt = self.lib.vl_fisher_encode(
            _ptr(enc), typ, _ptr(np.ascontiguousarray(means, dt)), D, K,
            _ptr(np.ascontiguousarray(covs, dt)), _ptr(np.ascontiguousarray(priors, dt)),
            _ptr(np.ascontiguousarray(data)), N, int(flags))
        return enc, int(nt)


    def vlad(self, data, means, assignments, flags):
        """vl_vlad_encode (vl/vlad.h:45-50): K x D encoding of data's dtype."""
        dt = data.dtype
        N, D = data.shape
        K = means.shape[0]
        typ = VL_TYPE_FLOAT if dt == np.float32 else VL_TYPE_DOUBLE
        enc = np.zeros(K * D, dt)
        self.lib.vl_vlad_encode(
            _ptr(enc), typ, _ptr(np.ascontiguousarray(means, dt)), D, K,
            _ptr(np.ascontiguousarray(data)), N,
            _ptr(np.ascontiguousarray(assignments, dt)), int(flags))
        return enc


def vlad(data, means, assignments, flags):
    """VLAD encoding restated (vl/vlad.c:163-242) in the data type's scalar
    arithmetic, vectorised over components and dimensions only: every
    accumulation keeps the reference's order.

    * enc_k += a_ik x_i for rows in order where a_ik > 0, each step computed
      in double and rounded to the data type (vl/vlad.c:180-188); the mass
      sum_i a_ik is a double;
    * mass > 0: enc_k = enc_k / mass - mu_k (NORMALIZE_MASS, the divide in
      double, the subtraction in the data type) or enc_k - mass mu_k in
      double (vl/vlad.c:191-202);
    * signed square root (vl/vlad.c:204-213);
    * per-component and global L2 norms: sums of squares in the data type in
      element order, square root, floored at 1e-12 in double
      (vl/vlad.c:215-240).
    """
    T = data.dtype.type
    x = np.asarray(data)
    a = np.asarray(assignments, x.dtype)
    mu = np.asarray(means, x.dtype)
    N, D = x.shape
    K = mu.shape[0]
    enc = np.zeros((K, D), x.dtype)
    mass = np.zeros(K, np.float64)
    for i in range(N):
        m = a[i] > 0
        if not m.any():
            continue
        q = a[i, m].astype(np.float64)
        mass[m] = mass[m] + q
        enc[m] = (enc[m].astype(np.float64) + q[:, None] * x[i].astype(np.float64)[None, :]).astype(x.dtype)
    pos = mass > 0
    if flags & VLAD_NORMALIZE_MASS:
        enc[pos] = (enc[pos].astype(np.float64) / mass[pos, None]).astype(x.dtype)
        enc[pos] = enc[pos] - mu[pos]
    else:
        enc[pos] = (enc[pos].astype(np.float64) - mass[pos, None] * mu[pos].astype(np.float64)).astype(x.dtype)
    if flags & VLAD_SQUARE_ROOT:
        enc = np.where(enc >= 0, np.sqrt(np.abs(enc)), -np.sqrt(np.abs(enc))).astype(x.dtype)

    def floor(n):
        return np.where(n.astype(np.float64) > 1e-12, n, T(1e-12)).astype(x.dtype)

    if flags & VLAD_NORMALIZE_COMPONENTS:
        n = np.zeros(K, x.dtype)
        for d in range(D):
            n = n + enc[:, d] * enc[:, d]
        n = floor(np.sqrt(n))
        enc = enc / n[:, None]
    enc = enc.ravel()
    if not flags & VLAD_UNNORMALIZED:
        n = T(0)
        for z in enc:
            n = T(n + T(z * z))
        n = floor(np.sqrt(np.asarray(n, x.dtype)))
        enc = enc / n
    return enc


def pca_learn(descrs, num_pca, whitening=False, regul=0.0):
    """PCA learning of apps/recognition/trainEncoder.m:150-171 restated in
    float64: center = mean, X = x x^T / n, eigenvalues sorted decreasing,
    d += regul * max(d), projection = first eigenvectors as rows (scaled by
    1/sqrt(d) when whitening).  descrs: n x D (one descriptor per row).
    Eigenvector signs are fixed as the library fixes them: the entry of
    largest magnitude is positive."""
    x = np.asarray(descrs, np.float64)
    c = x.mean(0)
    xc = x - c
    X = xc.T @ xc / x.shape[0]
    d, V = np.linalg.eigh(X)
    perm = np.argsort(-d, kind="stable")
    d, V = d[perm], V[:, perm]
    d = d + regul * d.max()
    m = min(num_pca, x.shape[1])
    V = V[:, :m]
    am = np.abs(V).argmax(0)
    V = V * np.where(V[am, np.arange(m)] < 0, -1.0, 1.0)[None, :]
    P = (V / np.sqrt(d[:m])[None, :]).T if whitening else V.T
    return P, c, d[:m]


def pca_project(descrs, P, c, renormalize=True, frames=None, offsets=None, sizes=None):
    """Descriptor prologue of apps/recognition/encodeImage.m:91-103 in float64:
    y = P (x - c), y / max(1e-12, |y|) per descriptor when renormalising, then
    the 'xy' extension (extendDescriptorsWithGeometry.m:19-21) with frames
    normalised by their image's size: (f - [w, h]/2) / [w, h]."""
    y = (np.asarray(descrs, np.float64) - np.asarray(c, np.float64)) @ np.asarray(P, np.float64).T
    if renormalize:
        y = y / np.maximum(1e-12, np.sqrt((y * y).sum(1)))[:, None]
    if frames is None:
        return y
    f = np.asarray(frames, np.float64)
    img = np.searchsorted(np.asarray(offsets), np.arange(len(f)), side="right") - 1
    wh = np.asarray(sizes, np.float64)[img]
    return np.concatenate([y, (f - wh / 2) / wh], 1)


def simple_fisher(data, means, covs, priors, flags):
    """Straight FP64 NumPy statement of the Fisher vector, written from the
    formulas of vl/fisher.c:19-130 (the same role as the ``simple_fisher``
    helper of toolbox/xtest/vl_test_fisher.m:57-78).  Small inputs only."""
    x = np.asarray(data, np.float64)
    mu = np.asarray(means, np.float64)
    s2 = np.asarray(covs, np.float64)
    pi = np.asarray(priors, np.float64)
    N, D = x.shape
    K = pi.shape[0]
    logw = np.where(pi < 1e-6, -np.inf, np.log(np.maximum(pi, 1e-300)))
    diff = x[:, None, :] - mu[None, :, :]
    lp = (logw[None, :] - 0.5 * D * np.log(2 * np.pi) - 0.5 * np.log(s2).sum(1)[None, :]
          - 0.5 * (diff ** 2 / s2[None]).sum(2))
    m = lp.max(1, keepdims=True)
    q = np.exp(lp - m)
    q /= q.sum(1, keepdims=True)
    if flags & FLAG_FAST:
        q = (np.arange(K)[None, :] == q.argmax(1)[:, None]).astype(np.float64)
    q = np.where(q < 1e-6, 0.0, q)
    q[:, pi < 1e-6] = 0.0
    z = diff / np.sqrt(s2)[None]
    u = np.einsum("nk,nkd->kd", q, z)
    v = np.einsum("nk,nkd->kd", q, z ** 2 - 1)
    if N > 0:
        with np.errstate(divide="ignore"):
            u = u / (N * np.sqrt(pi))[:, None]
            v = v / (N * np.sqrt(2 * pi))[:, None]
        u[pi < 1e-6] = 0
        v[pi < 1e-6] = 0
    enc = np.concatenate([u.ravel(), v.ravel()])
    if flags & FLAG_SQUARE_ROOT:
        enc = np.sign(enc) * np.sqrt(np.abs(enc))
    if flags & FLAG_NORMALIZED:
        enc = enc / max(np.linalg.norm(enc), 1e-12)
    return enc


# ------------------------------------------------------- Rand initialisation
class MT19937:
    """MT19937 (Matsumoto and Nishimura, 1998; 2002 initialisation) as
    VLFeat's vl/random.c uses it: unseeded state seeds itself with 5489
    (vl/random.c:202-203); vl_rand_uindex is a draw modulo the range
    (vl/random.h:64-73), vl_rand_real1 a draw times 1/(2^32 - 1)
    (vl/random.h:116-120)."""

    def __init__(self, seed=None):
        self.mt = [0] * 624
        self.mti = 625
        if seed is not None:
            self.seed(seed)

    def seed(self, s):
        mt = self.mt
        mt[0] = s & 0xFFFFFFFF
        for i in range(1, 624):
            mt[i] = (1812433253 * (mt[i - 1] ^ (mt[i - 1] >> 30)) + i) & 0xFFFFFFFF
        self.mti = 624

    def uint32(self):
        mt = self.mt
        if self.mti >= 624:
            if self.mti == 625:
                self.seed(5489)
            for k in range(624):
                y = (mt[k] & 0x80000000) | (mt[(k + 1) % 624] & 0x7FFFFFFF)
                mt[k] = mt[(k + 397) % 624] ^ (y >> 1) ^ (0x9908B0DF if y & 1 else 0)
            self.mti = 0
        y = mt[self.mti]
        self.mti += 1
        y ^= y >> 11
        y ^= (y << 7) & 0x9D2C5680
        y ^= (y << 15) & 0xEFC60000
        y ^= y >> 18
        return y & 0xFFFFFFFF

    def uindex(self, n):
        return self.uint32() % n

    def real1(self):
        return self.uint32() * (1.0 / 4294967295.0)


def _l2_ordered(a, b, lanes, T):
    """Squared L2 distance in the summation order of the reference's kernel:
    `lanes` accumulators over consecutive element groups, the SIMD horizontal
    sum (AVX float: ((v0+v1)+(v4+v5)) + ((v2+v3)+(v6+v7)); 4 lanes:
    (v0+v2)+(v1+v3); 2 lanes: v0+v1), then the remaining elements in order
    (vl/mathop_avx.c:44-108, vl/mathop_sse2.c:44-140, vl/mathop.c)."""
    D = a.shape[0]
    v = [T(0)] * lanes
    i = 0
    while i + lanes <= D:
        for l in range(lanes):
            d = T(a[i + l] - b[i + l])
            v[l] = T(v[l] + T(d * d))
        i += lanes
    if lanes == 8:
        acc = T(T(T(v[0] + v[1]) + T(v[4] + v[5])) + T(T(v[2] + v[3]) + T(v[6] + v[7])))
    elif lanes == 4:
        acc = T(T(v[0] + v[2]) + T(v[1] + v[3]))
    elif lanes == 2:
        acc = T(v[0] + v[1])
    else:
        acc = v[0]
    while i < D:
        d = T(a[i] - b[i])
        acc = T(acc + T(d * d))
        i += 1
    return acc


def rand_init(data, K, rng, lanes):
    """VlGMMRand initialisation restated (vl/gmm.c:1376-1443 and
    vl/kmeans.c:588-649) with the data type's scalar arithmetic, for small
    cases: uniform priors, every covariance the global variance (mean and
    squared deviations summed over the rows in order, / N and / (N - 1)),
    means by k-means++ seeding with `rng` (an MT19937)."""
    T = data.dtype.type
    N, D = data.shape
    priors = np.full(K, T(1.0 / K), data.dtype)
    sigma = np.zeros(D, data.dtype)
    if N > 1:
        for d in range(D):
            m = T(0)
            for i in range(N):
                m = T(m + data[i, d])
            m = T(m / T(N))
            ss = T(0)
            for i in range(N):
                df = T(data[i, d] - m)
                ss = T(ss + T(df * df))
            sigma[d] = T(ss / T(N - 1))
    covs = np.tile(sigma, (K, 1))
    centers = np.zeros((K, D), data.dtype)
    mind = [T(np.inf)] * N
    x = rng.uindex(N)
    c = 0
    while True:
        thresh = T(rng.real1())
        centers[c] = data[x]
        c += 1
        if c == K:
            break
        energy = T(0)
        for i in range(N):
            dist = _l2_ordered(centers[c - 1], data[i], lanes, T)
            mind[i] = mind[i] if mind[i] < dist else dist
            energy = T(energy + mind[i])
        t = T(thresh * energy)
        acc = T(0)
        x = 0
        while x < N - 1:
            acc = T(acc + mind[x])
            if acc >= t:
                break
            x += 1
    return dict(priors=priors, means=centers, covs=covs)


# ----------------------------------------------------- KMeans initialisation
def _l2_rows(q, C, lanes, T):
    """_l2_ordered of q against every row of C, vectorised over the rows (each
    NumPy operation rounds to T, so every element follows the scalar order)."""
    K, D = C.shape
    q = np.asarray(q, T)
    v = [np.zeros(K, T) for _ in range(lanes)]
    i = 0
    while i + lanes <= D:
        for l in range(lanes):
            d = (q[i + l] - C[:, i + l]).astype(T)
            v[l] = (v[l] + (d * d).astype(T)).astype(T)
        i += lanes
    if lanes == 8:
        acc = ((v[0] + v[1]) + (v[4] + v[5])) + ((v[2] + v[3]) + (v[6] + v[7]))
    elif lanes == 4:
        acc = (v[0] + v[2]) + (v[1] + v[3])
    elif lanes == 2:
        acc = v[0] + v[1]
    else:
        acc = v[0]
    acc = acc.astype(T)
    while i < D:
        d = (q[i] - C[:, i]).astype(T)
        acc = (acc + (d * d).astype(T)).astype(T)
        i += 1
    return acc


def _kd_tree(C, rng):
    """One kd-tree of a one-tree forest over the rows of C with median
    thresholds (vl/kdtree.c:165-325, 491-576; vl/kmeans.c:723-726).  Nodes are
    [lowerChild, upperChild, splitDimension, threshold, lowerBound,
    upperBound]; entries [index, value].  Draws from rng as the reference."""
    K, D = C.shape
    nodes, ent = [], [[k, 0.0] for k in range(K)]

    def new():
        nodes.append([0, 0, 0, 0.0, 0.0, 0.0])
        return len(nodes) - 1

    def build(n, b, e):
        if e - b <= 1:
            nodes[n][0], nodes[n][1] = -b - 1, -e - 1
            return
        have, bd, bv = False, 0, 0.0
        for d in range(D):
            full = e - b <= 1024
            ns = e - b if full else 1024
            mean = sec = 0.0
            for i in range(ns):
                si = i if full else rng.uint32() % 1024
                datum = float(C[ent[b + si][0], d])
                mean += datum
                sec += datum * datum
            mean /= ns
            sec /= ns
            var = sec - mean * mean
            if var <= 0:
                continue
            if not have or bv < var:
                have, bd, bv = True, d, var
        if not have:
            nodes[n][0], nodes[n][1] = -b - 1, -e - 1
            return
        rng.uint32()  # the dice over the kept dimensions (one tree: one)
        nodes[n][2] = bd
        for i in range(b, e):
            ent[i][1] = float(C[ent[i][0], bd])
        ent[b:e] = sorted(ent[b:e], key=lambda t: t[1])
        med = (b + e - 1) // 2
        nodes[n][3] = ent[med][1]
        lc = new()
        nodes[n][0] = lc
        build(lc, b, med + 1)
        uc = new()
        nodes[n][1] = uc
        build(uc, med + 1, e)

    build(new(), 0, K)
    sb = [-np.inf, np.inf] * D

    def bounds(n):
        i, t = nodes[n][2], nodes[n][3]
        nodes[n][4], nodes[n][5] = sb[2 * i], sb[2 * i + 1]
        if nodes[n][0] > 0:
            sb[2 * i + 1] = t
            bounds(nodes[n][0])
            sb[2 * i + 1] = nodes[n][5]
        if nodes[n][1] > 0:
            sb[2 * i] = t
            bounds(nodes[n][1])
            sb[2 * i] = nodes[n][4]

    bounds(0)
    return nodes, [e[0] for e in ent]


def _kd_query(q, dists, nodes, ent, max_comp):
    """Best-bin-first search for one neighbour (vl/kdtree.c:583-725,
    774-840) with the binary heap of vl/heap-def.h; dists[k] is the distance
    of the query to centre k.  Returns (distance, index)."""
    exact = max_comp == 0
    heap = [(0.0, 0)]
    comps, have, best, bi = 0, False, 0.0, 0
    while exact or comps < max_comp:
        if not heap:
            break
        n = len(heap) - 1
        heap[0], heap[n] = heap[n], heap[0]
        top = heap.pop()
        i = 0
        while True:  # vl/heap-def.h up()
            l, r = 2 * i + 1, 2 * i + 2
            if l >= len(heap):
                break
            if r >= len(heap):
                if heap[i][0] > heap[l][0]:
                    heap[i], heap[l] = heap[l], heap[i]
                break
            c = l if heap[l][0] < heap[r][0] else r
            if heap[i][0] > heap[c][0]:
                heap[i], heap[c] = heap[c], heap[i]
                i = c
            else:
                break
        lb, node = top
        if have and best < lb:
            break
        dist = lb
        while True:
            lo, up, dim, x2, x1, x3 = nodes[node]
            if lo < 0:
                for it in range(-lo - 1, -up - 1):
                    if not (exact or comps < max_comp):
                        break
                    di = ent[it]
                    dd = float(dists[di])
                    comps += 1
                    if not have:
                        have, best, bi = True, dd, di
                    elif best > dd:
                        best, bi = dd, di
                break
            x = float(q[dim])
            delta = x - x2
            save = dist + delta * delta
            if x <= x2:
                nxt, sv = lo, up
                if x <= x1:
                    delta = x - x1
                    save -= delta * delta
            else:
                nxt, sv = up, lo
                if x > x3:
                    delta = x - x3
                    save -= delta * delta
            if not have or best > save:
                heap.append((save, sv))
                j = len(heap) - 1
                while j > 0:  # vl/heap-def.h down()
                    p = (j - 1) // 2
                    if heap[j][0] < heap[p][0]:
                        heap[j], heap[p] = heap[p], heap[j]
                        j = p
                    else:
                        break
            node = nxt
    return best, bi


def kmeans_init(data, K, rng, lanes):
    """The k-means of VlGMMKMeans restated (vl/gmm.c:1336-1364 with
    vl/kmeans.c:528-582, 708-771, 1003-1150, 656-702) for small cases:
    random-selection seeding, ANN refinement (one tree, max(N/4, 10)
    comparisons, 5 iterations), exact quantisation.  Returns the centres, the
    assignment of every row and the energy."""
    T = data.dtype.type
    N, D = data.shape
    perm = list(range(N))
    n = N
    while n > 1:  # vl/shuffle-def.h:82-91
        k = rng.uindex(n)
        n -= 1
        perm[n], perm[k] = perm[k], perm[n]
    C = np.zeros((K, D), data.dtype)
    k = i = 0
    while k < K:
        if K - k < N - i and k > 0:
            d = np.array([_l2_rows(data[perm[i]], C[j:j + 1], lanes, T)[0] for j in range(k)])
            if np.any(d == 0):
                i += 1
                continue
        C[k] = data[perm[i]]
        k += 1
        i += 1
    max_comp = max(N // 4, 10)
    assign = np.zeros(N, np.int64)
    dist = np.zeros(N, data.dtype)
    energy = prev = initial = np.inf
    it = 0
    while True:
        nodes, ent = _kd_tree(C, rng)
        for x in range(N):
            dd = _l2_rows(data[x], C, lanes, T)
            nd, ni = _kd_query(data[x], dd, nodes, ent, max_comp)
            if it == 0:
                dist[x], assign[x] = T(nd), ni
            else:
                pd = dd[assign[x]]
                if pd > T(nd):
                    dist[x], assign[x] = T(nd), ni
                else:
                    dist[x] = pd
        energy = 0.0
        for x in range(N):
            energy += float(dist[x])
        if it >= 5 or energy == prev:
            break
        if it == 0:
            initial = energy
        elif (prev - energy) / (initial - energy) < 1e-4:
            break
        prev = energy
        mass = np.bincount(assign, minlength=K)
        acc = np.zeros((K, D), data.dtype)
        for x in range(N):
            acc[assign[x]] = (acc[assign[x]] + data[x]).astype(T)
        for c in range(K):
            if mass[c] > 0:
                C[c] = (acc[c] / T(mass[c])).astype(T)
            else:
                C[c] = data[rng.uindex(N)]
        it += 1
    final = np.zeros(N, np.int64)
    for x in range(N):
        dd = _l2_rows(data[x], C, lanes, T)
        best, bi = T(np.inf), 0
        for c in range(K):
            if dd[c] < best:
                best, bi = dd[c], c
        final[x] = bi
    return dict(centers=C, assign=final, energy=energy)
