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
VL_GMM_RAND = 1    # VlGMMRand, vl/gmm.h:21-26
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

    def rand_init(self, data, K, seed, max_iter=0, lb=1e-4):
        """vl_gmm_cluster with VlGMMRand initialisation (vl/gmm.c:1416-1443)
        after seeding the thread's generator; max_iter=0 leaves the initial
        parameters (one E-step, no M-step)."""
        L = self.lib
        dt = data.dtype
        N, D = data.shape
        g = L.vl_gmm_new(VL_TYPE_FLOAT if dt == np.float32 else VL_TYPE_DOUBLE, D, K)
        try:
            L.vl_gmm_set_initialization(g, VL_GMM_RAND)
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
