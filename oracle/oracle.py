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
  vl/fisher.h:48-54).  It exists only where that library was built.
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
VL_GMM_CUSTOM = 2  # VlGMMCustom, vl/gmm.h:21-26

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
        L.vl_set_num_threads.argtypes = [_sz]
        L.vl_get_max_threads.restype = _sz
        L.vl_set_simd_enabled.argtypes = [C.c_int]
        L.vl_get_simd_enabled.restype = C.c_int
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
