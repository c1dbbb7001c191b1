"""Python mirror of VLFeat's GMM / Fisher-vector C API over the B200 library.

Everything here calls ``vlfeat_b200/lib/libvl.so`` through ctypes: the
reference's own entry points (vl/gmm.h, vl/fisher.h) with host arrays, and
the ``vlb200_*`` extensions with device tensors.  There is no CPU fallback:
if the library is missing, :func:`lib` raises; if a call fails on the GPU,
the library's last-error message is raised as :class:`VLError`.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libvl.so")

VL_TYPE_FLOAT = 1
VL_TYPE_DOUBLE = 2
FLAG_SQUARE_ROOT = 1 << 0
FLAG_NORMALIZED = 1 << 1
FLAG_IMPROVED = FLAG_SQUARE_ROOT | FLAG_NORMALIZED
FLAG_FAST = 1 << 2
# VLAD flags, vl/vlad.h:23-26
VLAD_NORMALIZE_COMPONENTS = 1 << 0
VLAD_SQUARE_ROOT = 1 << 1
VLAD_UNNORMALIZED = 1 << 2
VLAD_NORMALIZE_MASS = 1 << 3
INIT_KMEANS, INIT_RAND, INIT_CUSTOM = 0, 1, 2  # VlGMMInitialization, vl/gmm.h:21-26

PREC_DEFAULT, PREC_EXACT, PREC_FP32, PREC_BF16, PREC_BF16_ROUTER = 0, 1, 2, 3, 4
PRECISIONS = {"default": 0, "exact": 1, "fp32": 2, "bf16": 3, "bf16_router": 4}

_vp = C.c_void_p
_sz = C.c_uint64


class VLError(RuntimeError):
    pass


_LIB = None

# vlb200_allreduce_fn: void (*)(double *values, vl_size count, void *context)
ALLREDUCE_FN = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.c_size_t, C.c_void_p)


def _decl(L):
    def f(name, res, *args):
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = list(args)

    f("vl_gmm_new", _vp, C.c_uint32, _sz, _sz)
    f("vl_gmm_new_copy", _vp, _vp)
    f("vl_gmm_delete", None, _vp)
    f("vl_gmm_reset", None, _vp)
    f("vl_gmm_cluster", C.c_double, _vp, _vp, _sz)
    f("vl_gmm_em", C.c_double, _vp, _vp, _sz)
    f("vl_gmm_init_with_rand_data", None, _vp, _vp, _sz)
    f("vl_gmm_init_with_kmeans", None, _vp, _vp, _sz, _vp)
    for n in ("means", "covariances", "priors"):
        f("vl_gmm_set_" + n, None, _vp, _vp)
        f("vl_gmm_get_" + n, _vp, _vp)
    f("vl_gmm_get_posteriors", _vp, _vp)
    f("vl_gmm_set_num_repetitions", None, _vp, _sz)
    f("vl_gmm_set_max_num_iterations", None, _vp, _sz)
    f("vl_gmm_set_verbosity", None, _vp, C.c_int)
    f("vl_gmm_set_initialization", None, _vp, C.c_int)
    f("vl_gmm_set_kmeans_init_object", None, _vp, _vp)
    f("vl_gmm_set_covariance_lower_bounds", None, _vp, _vp)
    f("vl_gmm_set_covariance_lower_bound", None, _vp, C.c_double)
    f("vl_gmm_get_data_type", C.c_uint32, _vp)
    for n in ("dimension", "num_repetitions", "num_data", "num_clusters", "max_num_iterations"):
        f("vl_gmm_get_" + n, _sz, _vp)
    f("vl_gmm_get_loglikelihood", C.c_double, _vp)
    f("vl_gmm_get_verbosity", C.c_int, _vp)
    f("vl_gmm_get_initialization", C.c_int, _vp)
    f("vl_gmm_get_kmeans_init_object", _vp, _vp)
    f("vl_gmm_get_covariance_lower_bounds", _vp, _vp)
    for s in ("_f", "_d"):
        f("vl_get_gmm_data_posteriors" + s, C.c_double, _vp, _sz, _sz, _vp, _vp, _sz, _vp, _vp)
    f("vl_fisher_encode", _sz, _vp, C.c_uint32, _vp, _sz, _sz, _vp, _vp, _vp, _sz, C.c_int)
    f("vl_vlad_encode", None, _vp, C.c_uint32, _vp, _sz, _sz, _vp, _sz, _vp, C.c_int)
    f("vlb200_vlad_encode_batch_device", C.c_int, _vp, C.c_uint32, _vp, _sz, _sz, _vp, _vp, _vp, _sz,
      C.c_int, _vp)
    f("vlb200_pca_project_device", C.c_int, _vp, _sz, _vp, _sz, _sz, _vp, _vp, C.c_int, _vp, _vp, _vp, _sz, _vp)
    f("vlb200_pca_learn_device", C.c_int, _vp, _vp, _sz, _vp, _sz, _sz, C.c_int, C.c_double, _vp, _vp)
    f("vl_get_last_error", C.c_int)
    f("vl_get_last_error_message", C.c_char_p)
    f("vl_set_last_error", C.c_int, C.c_int, C.c_char_p)
    f("vl_set_num_threads", None, _sz)
    f("vl_get_max_threads", _sz)
    f("vl_get_version_string", C.c_char_p)
    f("vlb200_version", C.c_char_p)
    f("vlb200_device_ok", C.c_int)
    f("vlb200_set_precision", C.c_int, C.c_int)
    f("vlb200_get_precision", C.c_int)
    f("vlb200_last_precision", C.c_int)
    f("vlb200_launch_count", C.c_uint64)
    f("vlb200_profile_enable", None, C.c_int)
    f("vlb200_profile_reset", None)
    f("vlb200_profile_read", C.c_int, C.c_char_p, _sz, _vp, _vp, _sz)
    f("vlb200_gmm_posteriors_device", C.c_int, _vp, _sz, _sz, _vp, _vp, _sz, _vp, _vp, C.c_int,
      C.POINTER(C.c_double), _vp)
    f("vlb200_gmm_em_device", C.c_double, _vp, _vp, _sz, C.c_int)
    f("vlb200_gmm_get_ll_trace", _sz, _vp, _vp, _sz)
    f("vlb200_gmm_get_num_restarts", _sz, _vp)
    f("vlb200_gmm_set_param_trace", None, _vp, C.c_int)
    f("vlb200_gmm_em_stream_device", C.c_double, _vp, _vp, _sz, C.c_int, _sz, _vp, _sz, C.c_float, _sz)
    f("vlb200_gmm_em_sharded_device", C.c_double, _vp, _vp, _sz, _sz, C.c_int, _sz, ALLREDUCE_FN, _vp)
    f("vlb200_gmm_get_stream_report", _sz, _vp, _vp, _sz)
    f("vlb200_gmm_get_param_trace", _sz, _vp, _sz, _vp, _vp, _vp)
    f("vlb200_fisher_encode_device", C.c_int, _vp, _vp, _sz, _sz, _vp, _vp, _vp, _sz, C.c_int,
      C.c_int, C.POINTER(C.c_uint64), _vp)
    f("vlb200_fisher_encode_batch_device", C.c_int, _vp, _vp, _sz, _sz, _vp, _vp, _vp, _vp, _sz,
      C.c_int, C.c_int, _vp, _vp)
    f("vl_get_rand", _vp)
    f("vl_rand_seed", None, _vp, C.c_uint32)
    f("vl_rand_uint32", C.c_uint32, _vp)
    f("vl_rand_init", None, _vp)
    f("vl_cpu_has_avx", C.c_int)
    f("vl_cpu_has_sse2", C.c_int)
    f("vl_gmm_init_with_rand_data", None, _vp, _vp, _sz)
    f("vlb200_fisher_plan_new", _vp, _sz, _sz, _vp, _sz, C.c_int, C.c_int)
    f("vlb200_fisher_plan_delete", None, _vp)
    f("vlb200_fisher_plan_set_gmm", C.c_int, _vp, _vp, _vp, _vp)
    f("vlb200_fisher_plan_execute", C.c_int, _vp, _vp, _vp, _vp, _vp)
    f("vlb200_fisher_plan_execute_host", C.c_int, _vp, _vp, _vp, _vp, _vp)
    f("vlb200_fisher_plan_autotune", C.c_int, _vp, _vp, _vp, _vp, _vp, C.POINTER(C.c_double))
    f("vlb200_fisher_plan_get_config", C.c_int, _vp, _vp)
    f("vlb200_fisher_plan_set_config", C.c_int, _vp, _vp, _vp)
    f("vlb200_fisher_plan_capture", C.c_int, _vp, _vp, _vp, _vp, _vp)
    f("vlb200_fisher_plan_launch", C.c_int, _vp, _vp)
    f("vlb200_fisher_plan_status", C.c_int, _vp, _vp)


def lib(path: str = LIB_PATH):
    """Load the library (once).  Raises if it has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(path):
            raise VLError(f"{path} is missing: build it with `python -m vlfeat_b200.build`")
        L = C.CDLL(path)
        _decl(L)
        _LIB = L
    return _LIB


def _raise_last(what: str):
    L = lib()
    msg = L.vl_get_last_error_message().decode(errors="replace")
    raise VLError(f"{what}: {msg} (code {L.vl_get_last_error()})")


def _clear():
    lib().vl_set_last_error(0, None)


def _np_ptr(a):
    return a.ctypes.data_as(_vp)


def _dt(dtype):
    dt = np.dtype(dtype)
    if dt == np.float32:
        return VL_TYPE_FLOAT
    if dt == np.float64:
        return VL_TYPE_DOUBLE
    raise TypeError("data must be float32 or float64")


def _prec(p) -> int:
    return PRECISIONS[p] if isinstance(p, str) else int(p)


def set_precision(p) -> None:
    if lib().vlb200_set_precision(_prec(p)):
        _raise_last("vlb200_set_precision")


def get_precision() -> int:
    return int(lib().vlb200_get_precision())


def last_precision() -> str:
    """Arithmetic the calling thread's last encode / E-step / EM iteration
    actually ran ("exact", "fp32", "bf16", "bf16_router"; "" before any)."""
    v = int(lib().vlb200_last_precision())
    return {k: n for n, k in PRECISIONS.items() if n != "default"}.get(v, "")


def device_ok() -> bool:
    return bool(lib().vlb200_device_ok())


def launch_count() -> int:
    return int(lib().vlb200_launch_count())


def profile_enable(on: bool = True) -> None:
    lib().vlb200_profile_enable(1 if on else 0)


def profile_reset() -> None:
    lib().vlb200_profile_reset()


def profile_read(max_entries: int = 64):
    """{kernel name: (launches, total device ms)} since the last reset."""
    stride = 64
    names = C.create_string_buffer(stride * max_entries)
    ms = np.zeros(max_entries, np.float64)
    cnt = np.zeros(max_entries, np.uint64)
    n = lib().vlb200_profile_read(names, stride, _np_ptr(ms), _np_ptr(cnt), max_entries)
    out = {}
    for i in range(min(n, max_entries)):
        nm = names.raw[i * stride:(i + 1) * stride].split(b"\0", 1)[0].decode()
        out[nm] = (int(cnt[i]), float(ms[i]))
    return out


# ------------------------------------------------------------------ GMM
class GMM:
    """``VlGMM`` (vl/gmm.h) on the GPU.  Arrays are NumPy, row-major:
    data (N, D), means/covariances (K, D), priors (K,)."""

    def __init__(self, dimension: int, num_clusters: int, dtype=np.float32):
        self.dtype = np.dtype(dtype)
        self.D, self.K = int(dimension), int(num_clusters)
        _clear()
        self._h = lib().vl_gmm_new(_dt(self.dtype), self.D, self.K)
        if not self._h:
            _raise_last("vl_gmm_new")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _LIB is not None:
            _LIB.vl_gmm_delete(h)
            self._h = None

    def _arr(self, a, shape):
        a = np.ascontiguousarray(a, self.dtype)
        if a.shape != shape:
            raise ValueError(f"expected shape {shape}, got {a.shape}")
        return a

    def set_means(self, m):
        lib().vl_gmm_set_means(self._h, _np_ptr(self._arr(m, (self.K, self.D))))

    def set_covariances(self, c):
        lib().vl_gmm_set_covariances(self._h, _np_ptr(self._arr(c, (self.K, self.D))))

    def set_priors(self, p):
        lib().vl_gmm_set_priors(self._h, _np_ptr(self._arr(p, (self.K,))))

    def set_initialization(self, init):
        init = {"kmeans": INIT_KMEANS, "rand": INIT_RAND, "custom": INIT_CUSTOM}.get(init, init)
        lib().vl_gmm_set_initialization(self._h, int(init))

    def set_max_num_iterations(self, n):
        lib().vl_gmm_set_max_num_iterations(self._h, int(n))

    def set_num_repetitions(self, n):
        lib().vl_gmm_set_num_repetitions(self._h, int(n))

    def set_verbosity(self, v):
        lib().vl_gmm_set_verbosity(self._h, int(v))

    def set_covariance_lower_bound(self, b):
        lb = np.asarray(b, np.float64)
        if lb.ndim == 0:
            lib().vl_gmm_set_covariance_lower_bound(self._h, float(lb))
        else:
            lb = np.ascontiguousarray(lb, np.float64).reshape(self.D)
            lib().vl_gmm_set_covariance_lower_bounds(self._h, _np_ptr(lb))

    def _data(self, data):
        data = np.ascontiguousarray(data, self.dtype)
        if data.ndim != 2 or data.shape[1] != self.D:
            raise ValueError("data must be (N, D)")
        return data

    def cluster(self, data) -> float:
        data = self._data(data)
        _clear()
        ll = lib().vl_gmm_cluster(self._h, _np_ptr(data), data.shape[0])
        if lib().vl_get_last_error():
            _raise_last("vl_gmm_cluster")
        return ll

    def em(self, data) -> float:
        data = self._data(data)
        _clear()
        ll = lib().vl_gmm_em(self._h, _np_ptr(data), data.shape[0])
        if lib().vl_get_last_error():
            _raise_last("vl_gmm_em")
        return ll

    def em_device(self, data_t, precision="default") -> float:
        """EM on a (N, D) float32 CUDA tensor (vlb200_gmm_em_device)."""
        _clear()
        ll = lib().vlb200_gmm_em_device(self._h, data_t.data_ptr(), data_t.shape[0], _prec(precision))
        if lib().vl_get_last_error():
            _raise_last("vlb200_gmm_em_device")
        return ll

    def em_stream_device(self, data_t, precision="default", chunk_rows=0, router=None, m=8,
                         threshold=0.99, judge_every=5) -> float:
        """Streamed EM on a (N, D) float32 CUDA tensor, posteriors never
        resident (vlb200_gmm_em_stream_device); `router` a router.Router or
        None.  `data_t` must stay alive while the posteriors may be read."""
        _clear()
        ll = lib().vlb200_gmm_em_stream_device(self._h, data_t.data_ptr(), data_t.shape[0], _prec(precision),
                                               int(chunk_rows), router._h if router is not None else None,
                                               int(m), float(threshold), int(judge_every))
        if lib().vl_get_last_error():
            _raise_last("vlb200_gmm_em_stream_device")
        return ll

    def em_sharded_device(self, data_t, total_rows, allreduce, precision="default", chunk_rows=0) -> float:
        """EM over rows sharded across ranks (vlb200_gmm_em_sharded_device):
        `data_t` this rank's (n, D) CUDA tensor of the model's dtype, at least
        one row, of `total_rows` in all; `allreduce(values)` sums a float64
        NumPy array in place over all ranks (replicas.allreduce_sum builds one
        on a torch.distributed group).  Returns the log-likelihood over all
        rows, the same on every rank."""
        err = []

        def cb(ptr, count, _ctx):
            # Every call is passed on, also after a failure, so that the ranks
            # keep making the same collective calls; the first error is
            # raised once the library call returns.
            try:
                allreduce(np.ctypeslib.as_array(ptr, shape=(int(count),)))
            except BaseException as e:  # noqa: BLE001
                err.append(e)

        fn = ALLREDUCE_FN(cb)
        _clear()
        ll = lib().vlb200_gmm_em_sharded_device(self._h, data_t.data_ptr(), data_t.shape[0], int(total_rows),
                                                 _prec(precision), int(chunk_rows), fn, None)
        if err:
            raise err[0]
        if lib().vl_get_last_error():
            _raise_last("vlb200_gmm_em_sharded_device")
        return ll

    def stream_report(self):
        """Per E-step of the last streamed EM: dicts of log-likelihood,
        judged, routed, missed_mass, fallback_rows, ms."""
        buf = np.zeros((4096, 6), np.float64)
        n = int(lib().vlb200_gmm_get_stream_report(self._h, _np_ptr(buf), 4096))
        keys = ("loglikelihood", "judged", "routed", "missed_mass", "fallback_rows", "ms")
        return [{k: (bool(v) if k in ("judged", "routed") else float(v)) for k, v in zip(keys, row)}
                for row in buf[:n]]

    def _get(self, fn, n):
        ct = C.c_float if self.dtype == np.float32 else C.c_double
        p = fn(self._h)
        if not p:
            _raise_last("getter")
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(ct)), shape=(n,)).copy()

    @property
    def means(self):
        return self._get(lib().vl_gmm_get_means, self.K * self.D).reshape(self.K, self.D)

    @property
    def covariances(self):
        return self._get(lib().vl_gmm_get_covariances, self.K * self.D).reshape(self.K, self.D)

    @property
    def priors(self):
        return self._get(lib().vl_gmm_get_priors, self.K)

    @property
    def posteriors(self):
        n = int(lib().vl_gmm_get_num_data(self._h))
        return self._get(lib().vl_gmm_get_posteriors, n * self.K).reshape(n, self.K)

    @property
    def loglikelihood(self) -> float:
        return float(lib().vl_gmm_get_loglikelihood(self._h))

    @property
    def num_data(self) -> int:
        return int(lib().vl_gmm_get_num_data(self._h))

    @property
    def ll_trace(self):
        buf = np.zeros(4096, np.float64)
        n = lib().vlb200_gmm_get_ll_trace(self._h, _np_ptr(buf), buf.size)
        return buf[:n].copy()

    @property
    def num_restarts(self) -> int:
        return int(lib().vlb200_gmm_get_num_restarts(self._h))

    def set_param_trace(self, on: bool = True) -> None:
        """Keep every EM iteration's parameters (vlb200_gmm_set_param_trace)."""
        lib().vlb200_gmm_set_param_trace(self._h, 1 if on else 0)

    def param_trace(self):
        """[(means, covariances, priors)] as float64, entry t after t M-steps."""
        out = []
        n = int(lib().vlb200_gmm_get_param_trace(self._h, 1 << 62, None, None, None))
        for t in range(n):
            mu = np.zeros((self.K, self.D)); cv = np.zeros((self.K, self.D)); pr = np.zeros(self.K)
            lib().vlb200_gmm_get_param_trace(self._h, t, _np_ptr(mu), _np_ptr(cv), _np_ptr(pr))
            out.append((mu, cv, pr))
        return out


def get_gmm_data_posteriors(data, priors, means, covariances):
    """vl_get_gmm_data_posteriors_{f,d} (vl/gmm.h:94-112) -> (posteriors, LL)."""
    data = np.ascontiguousarray(data)
    dt = data.dtype
    N, D = data.shape
    K = len(priors)
    post = np.zeros((N, K), dt)
    fn = lib().vl_get_gmm_data_posteriors_f if dt == np.float32 else lib().vl_get_gmm_data_posteriors_d
    _dt(dt)
    _clear()
    ll = fn(_np_ptr(post), K, N, _np_ptr(np.ascontiguousarray(priors, dt)),
            _np_ptr(np.ascontiguousarray(means, dt)), D,
            _np_ptr(np.ascontiguousarray(covariances, dt)), _np_ptr(data))
    if lib().vl_get_last_error():
        _raise_last("vl_get_gmm_data_posteriors")
    return post, ll


def fisher_encode(data, means, covariances, priors, flags=FLAG_IMPROVED):
    """vl_fisher_encode (vl/fisher.h:48-54) -> (enc of 2KD, numTerms)."""
    data = np.ascontiguousarray(data)
    dt = data.dtype
    typ = _dt(dt)
    N, D = data.shape
    K = len(priors)
    enc = np.zeros(2 * K * D, dt)
    _clear()
    nt = lib().vl_fisher_encode(_np_ptr(enc), typ, _np_ptr(np.ascontiguousarray(means, dt)), D, K,
                                _np_ptr(np.ascontiguousarray(covariances, dt)),
                                _np_ptr(np.ascontiguousarray(priors, dt)), _np_ptr(data), N,
                                int(flags))
    if lib().vl_get_last_error():
        _raise_last("vl_fisher_encode")
    return enc, int(nt)


def vlad_encode(data, means, assignments, flags=0):
    """vl_vlad_encode (vl/vlad.h:45-50) -> enc of K*D elements of data's dtype.
    assignments: N x K weights (hard or soft)."""
    data = np.ascontiguousarray(data)
    dt = data.dtype
    N, D = data.shape
    K = np.asarray(means).shape[0]
    enc = np.zeros(K * D, dt)
    _clear()
    lib().vl_vlad_encode(_np_ptr(enc), _dt(dt), _np_ptr(np.ascontiguousarray(means, dt)), D, K,
                         _np_ptr(data), N, _np_ptr(np.ascontiguousarray(assignments, dt)), int(flags))
    if lib().vl_get_last_error():
        _raise_last("vl_vlad_encode")
    return enc


def rand_seed(s: int) -> None:
    """vl_rand_seed on the calling thread's generator (vl_get_rand)."""
    lib().vl_rand_seed(lib().vl_get_rand(), int(s))


def rand_uint32() -> int:
    return int(lib().vl_rand_uint32(lib().vl_get_rand()))


def _stream(stream):
    """Stream handle for the library: the given stream, or torch's current
    stream when None.  A handle of 0 (the legacy default stream) is passed as
    cudaStreamLegacy (0x1), since 0 would select the library's own stream."""
    if stream is None:
        import torch  # device calls take torch tensors: order with torch's stream
        stream = torch.cuda.current_stream()
    h = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
    return C.c_void_p(h if h else 1)


def gmm_posteriors_device(post_t, priors_t, means_t, covs_t, data_t, precision="default",
                          stream=None) -> float:
    ll = C.c_double(0)
    N, D = data_t.shape
    K = priors_t.shape[0]
    _clear()
    rc = lib().vlb200_gmm_posteriors_device(post_t.data_ptr(), K, N, priors_t.data_ptr(),
                                            means_t.data_ptr(), D, covs_t.data_ptr(),
                                            data_t.data_ptr(), _prec(precision), C.byref(ll),
                                            _stream(stream))
    if rc:
        _raise_last("vlb200_gmm_posteriors_device")
    return ll.value


def fisher_encode_device(enc_t, means_t, covs_t, priors_t, data_t, flags=FLAG_IMPROVED,
                         precision="default", stream=None) -> int:
    N, D = data_t.shape
    K = priors_t.shape[0]
    nt = C.c_uint64(0)
    _clear()
    rc = lib().vlb200_fisher_encode_device(enc_t.data_ptr(), means_t.data_ptr(), D, K,
                                           covs_t.data_ptr(), priors_t.data_ptr(),
                                           data_t.data_ptr(), N, int(flags), _prec(precision),
                                           C.byref(nt), _stream(stream))
    if rc:
        _raise_last("vlb200_fisher_encode_device")
    return int(nt.value)


def fisher_encode_batch_device(enc_t, means_t, covs_t, priors_t, data_t, offsets,
                               flags=FLAG_IMPROVED, precision="default", nterms_t=None,
                               stream=None) -> None:
    """Encode len(offsets)-1 images in one call; enc_t is (numImages, 2KD)."""
    offs = np.ascontiguousarray(offsets, np.int64)
    D = data_t.shape[1]
    K = priors_t.shape[0]
    _clear()
    rc = lib().vlb200_fisher_encode_batch_device(
        enc_t.data_ptr(), means_t.data_ptr(), D, K, covs_t.data_ptr(), priors_t.data_ptr(),
        data_t.data_ptr(), _np_ptr(offs), len(offs) - 1, int(flags), _prec(precision),
        nterms_t.data_ptr() if nterms_t is not None else None, _stream(stream))
    if rc:
        _raise_last("vlb200_fisher_encode_batch_device")


def vlad_encode_batch_device(enc_t, means_t, data_t, assign_t, offsets, flags=0, stream=None) -> None:
    """VLAD of len(offsets)-1 images in one call (torch CUDA tensors of one
    dtype, float32 or float64); enc_t is (numImages, K*D)."""
    import torch
    offs = np.ascontiguousarray(offsets, np.int64)
    K, D = means_t.shape
    typ = VL_TYPE_FLOAT if data_t.dtype == torch.float32 else VL_TYPE_DOUBLE
    _clear()
    rc = lib().vlb200_vlad_encode_batch_device(enc_t.data_ptr(), typ, means_t.data_ptr(), D, K,
                                               data_t.data_ptr(), assign_t.data_ptr(), _np_ptr(offs),
                                               len(offs) - 1, int(flags), _stream(stream))
    if rc:
        _raise_last("vlb200_vlad_encode_batch_device")


def pca_learn_device(data_t, num_pca_dimensions, whitening=False, whitening_regul=0.0, stream=None):
    """PCA of a descriptor sample (vlb200_pca_learn_device): returns
    (projection (m x D) and center (D) as torch CUDA tensors, eigenvalues)."""
    import torch
    N, D = data_t.shape
    m = int(num_pca_dimensions)
    P = torch.empty((m, D), dtype=torch.float32, device=data_t.device)
    c = torch.empty(D, dtype=torch.float32, device=data_t.device)
    ev = np.zeros(m, np.float64)
    _clear()
    rc = lib().vlb200_pca_learn_device(P.data_ptr(), c.data_ptr(), m, data_t.data_ptr(), D, N, int(bool(whitening)),
                                       float(whitening_regul), _np_ptr(ev), _stream(stream))
    if rc:
        _raise_last("vlb200_pca_learn_device")
    return P, c, ev


def pca_project_device(out_t, data_t, projection_t, center_t, renormalize=True, frames_t=None, offsets=None,
                       image_sizes_t=None, stream=None):
    """The app's descriptor prologue (vlb200_pca_project_device): out_t is
    N x (m + 2 if frames_t is given)."""
    N, D = data_t.shape
    m = projection_t.shape[0]
    offs = np.ascontiguousarray(offsets if offsets is not None else [0, N], np.int64)
    _clear()
    rc = lib().vlb200_pca_project_device(
        out_t.data_ptr(), m, data_t.data_ptr(), D, N, projection_t.data_ptr(), center_t.data_ptr(),
        int(bool(renormalize)), frames_t.data_ptr() if frames_t is not None else None, _np_ptr(offs),
        image_sizes_t.data_ptr() if image_sizes_t is not None else None, len(offs) - 1, _stream(stream))
    if rc:
        _raise_last("vlb200_pca_project_device")


class FisherPlan:
    """vlb200_fisher_plan_*: the batched tensor-core encoder bound to one batch
    layout, with autotuned tile shapes and CUDA-graph replay.  The GMM and the
    data/output buffers are torch CUDA tensors that must outlive their use."""

    CONFIG_KEYS = ("item_rows", "stats_mt", "stats_stages", "estep_stages", "row_budget")

    def __init__(self, D, K, offsets, flags=FLAG_IMPROVED, precision="bf16"):
        self.offsets = np.ascontiguousarray(offsets, np.int64)
        _clear()
        h = lib().vlb200_fisher_plan_new(D, K, _np_ptr(self.offsets), len(self.offsets) - 1,
                                         int(flags), _prec(precision))
        if not h:
            _raise_last("vlb200_fisher_plan_new")
        self._h = h
        self._keep = ()

    def close(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.vlb200_fisher_plan_delete(self._h)
        self._h = None

    def __del__(self):
        self.close()

    def _check(self, rc, what):
        if rc:
            _raise_last(what)

    def set_gmm(self, means_t, covs_t, priors_t):
        self._gmm = (means_t, covs_t, priors_t)
        _clear()
        self._check(lib().vlb200_fisher_plan_set_gmm(self._h, means_t.data_ptr(), covs_t.data_ptr(),
                                                     priors_t.data_ptr()), "vlb200_fisher_plan_set_gmm")

    def execute(self, enc_t, data_t, nterms_t=None, stream=None):
        _clear()
        self._check(lib().vlb200_fisher_plan_execute(
            self._h, enc_t.data_ptr(), data_t.data_ptr(),
            nterms_t.data_ptr() if nterms_t is not None else None, _stream(stream)),
            "vlb200_fisher_plan_execute")

    def execute_host(self, enc, data, nterms=None, stream=None):
        """Host buffers (numpy arrays or CPU torch tensors; page-locked ones let
        the copies overlap the encode).  Returns when the results are written."""
        def ptr(a):
            if a is None:
                return None
            return a.data_ptr() if hasattr(a, "data_ptr") else _np_ptr(a)
        _clear()
        self._check(lib().vlb200_fisher_plan_execute_host(self._h, ptr(enc), ptr(data), ptr(nterms),
                                                          _stream(stream)),
                    "vlb200_fisher_plan_execute_host")

    def autotune(self, enc_t, data_t, nterms_t=None, stream=None) -> float:
        ms = C.c_double(0)
        _clear()
        self._check(lib().vlb200_fisher_plan_autotune(
            self._h, enc_t.data_ptr(), data_t.data_ptr(),
            nterms_t.data_ptr() if nterms_t is not None else None, _stream(stream), C.byref(ms)),
            "vlb200_fisher_plan_autotune")
        return ms.value

    def get_config(self) -> dict:
        c = np.zeros(5, np.int64)
        self._check(lib().vlb200_fisher_plan_get_config(self._h, _np_ptr(c)),
                    "vlb200_fisher_plan_get_config")
        return dict(zip(self.CONFIG_KEYS, (int(v) for v in c)))

    def set_config(self, stream=None, **kw):
        cur = self.get_config()
        cur.update(kw)
        c = np.array([cur[k] for k in self.CONFIG_KEYS], np.int64)
        _clear()
        self._check(lib().vlb200_fisher_plan_set_config(self._h, _np_ptr(c), _stream(stream)),
                    "vlb200_fisher_plan_set_config")

    def capture(self, enc_t, data_t, nterms_t=None, stream=None):
        self._keep = (enc_t, data_t, nterms_t)
        _clear()
        self._check(lib().vlb200_fisher_plan_capture(
            self._h, enc_t.data_ptr(), data_t.data_ptr(),
            nterms_t.data_ptr() if nterms_t is not None else None, _stream(stream)),
            "vlb200_fisher_plan_capture")

    def launch(self, stream=None):
        self._check(lib().vlb200_fisher_plan_launch(self._h, _stream(stream)),
                    "vlb200_fisher_plan_launch")

    def status(self, stream=None) -> int:
        return int(lib().vlb200_fisher_plan_status(self._h, _stream(stream)))
