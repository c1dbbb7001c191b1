"""Python interface to the learned E-step router (``vlb200_router_*``).

The router is an MLP (ReLU, bf16 weights, fp32 accumulation) that predicts
each descriptor's top-m mixture components.  Training, inference, the exact
posteriors on the candidates and the full-E-step fallback all run in the
library's own CUDA kernels; this module only binds them.  Data arguments are
CUDA tensors; parameters move as host NumPy vectors.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi

_vp = C.c_void_p
_sz = C.c_uint64
_DECLARED = False


def _lib():
    global _DECLARED
    L = capi.lib()
    if not _DECLARED:
        def f(name, res, *args):
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = list(args)
        f("vlb200_router_new", _vp, _sz, _sz, _vp, _sz, C.c_uint32)
        f("vlb200_router_delete", None, _vp)
        f("vlb200_router_num_params", _sz, _vp)
        f("vlb200_router_get_params", C.c_int, _vp, _vp)
        f("vlb200_router_set_params", C.c_int, _vp, _vp)
        f("vlb200_router_set_input_transform", C.c_int, _vp, _vp, _vp)
        f("vlb200_router_targets", C.c_int, _vp, _sz, _sz, _vp, _vp)
        f("vlb200_router_loss_grad", C.c_int, _vp, _vp, _sz, _vp, _vp, C.POINTER(C.c_double), _vp)
        f("vlb200_router_train", C.c_int, _vp, _vp, _sz, _vp, _vp, _sz, _sz, C.c_float,
          C.POINTER(C.c_double))
        f("vlb200_router_posteriors", C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _sz, _sz, C.c_float,
          C.POINTER(C.c_uint64), _vp)
        f("vlb200_router_missed_mass", C.c_int, _vp, _vp, _sz, _sz, C.POINTER(C.c_double))
        f("vlb200_router_set_default", C.c_int, _vp, _sz, C.c_float)
        f("vlb200_router_set_tensor_core_inference", C.c_int, _vp, C.c_int)
        f("vlb200_router_logits", C.c_int, _vp, _vp, _sz, _vp, _vp)
        f("vlb200_router_candidates", C.c_int, _vp, _vp, _sz, _sz, _vp, _vp, C.c_int, _vp)
        _DECLARED = True
    return L


def _check(rc, what):
    if rc:
        capi._raise_last(what)


class Router:
    def __init__(self, dimension: int, num_clusters: int, hidden=(256, 256), seed: int = 0):
        L = _lib()
        self.D, self.K = int(dimension), int(num_clusters)
        self.sizes = [self.D, *[int(h) for h in hidden], self.K]
        h = np.ascontiguousarray(hidden, np.uint64)
        capi._clear()
        self._h = L.vlb200_router_new(self.D, self.K, h.ctypes.data_as(_vp), len(hidden), seed)
        if not self._h:
            capi._raise_last("vlb200_router_new")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and capi._LIB is not None:
            capi._LIB.vlb200_router_set_default(None, 8, 0.99)
            capi._LIB.vlb200_router_delete(h)
            self._h = None

    @property
    def num_params(self) -> int:
        return int(_lib().vlb200_router_num_params(self._h))

    def get_params(self):
        out = np.zeros(self.num_params, np.float32)
        _check(_lib().vlb200_router_get_params(self._h, out.ctypes.data_as(_vp)), "get_params")
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        _check(_lib().vlb200_router_set_params(self._h, p.ctypes.data_as(_vp)), "set_params")

    def layers(self):
        """Split a parameter vector into [(W, b), ...] (W: out x in)."""
        p, out, o = self.get_params(), [], 0
        for i in range(len(self.sizes) - 1):
            n_in, n_out = self.sizes[i], self.sizes[i + 1]
            W = p[o:o + n_out * n_in].reshape(n_out, n_in)
            o += n_out * n_in
            b = p[o:o + n_out]
            o += n_out
            out.append((W, b))
        return out

    def set_input_transform(self, centre, scale):
        c = np.ascontiguousarray(centre, np.float32)
        s = np.ascontiguousarray(scale, np.float32)
        _check(_lib().vlb200_router_set_input_transform(self._h, c.ctypes.data_as(_vp),
                                                        s.ctypes.data_as(_vp)), "set_input_transform")

    def loss_grad(self, x_t, tidx_t, tw_t, want_grad=True):
        B = x_t.shape[0]
        loss = C.c_double(0)
        g = np.zeros(self.num_params, np.float32) if want_grad else None
        _check(_lib().vlb200_router_loss_grad(self._h, x_t.data_ptr(), B, tidx_t.data_ptr(),
                                              tw_t.data_ptr(), C.byref(loss),
                                              g.ctypes.data_as(_vp) if want_grad else None),
               "loss_grad")
        return loss.value, g

    def train(self, x_t, tidx_t, tw_t, epochs=3, batch=2048, lr=1e-3):
        loss = C.c_double(0)
        _check(_lib().vlb200_router_train(self._h, x_t.data_ptr(), x_t.shape[0], tidx_t.data_ptr(),
                                          tw_t.data_ptr(), epochs, batch, lr, C.byref(loss)), "train")
        return loss.value

    def posteriors(self, post_t, priors_t, means_t, covs_t, x_t, m=8, threshold=0.99):
        fb = C.c_uint64(0)
        _check(_lib().vlb200_router_posteriors(self._h, post_t.data_ptr(), priors_t.data_ptr(),
                                               means_t.data_ptr(), covs_t.data_ptr(), x_t.data_ptr(),
                                               x_t.shape[0], m, threshold, C.byref(fb),
                                               capi._stream(None)), "router_posteriors")
        return int(fb.value)

    def set_tensor_core_inference(self, on=True):
        _check(_lib().vlb200_router_set_tensor_core_inference(self._h, 1 if on else 0),
               "set_tensor_core_inference")

    def logits(self, logits_t, x_t):
        _check(_lib().vlb200_router_logits(self._h, x_t.data_ptr(), x_t.shape[0], logits_t.data_ptr(),
                                           capi._stream(None)), "logits")

    def candidates(self, cand_t, mass_t, x_t, m=8, fused=True):
        _check(_lib().vlb200_router_candidates(self._h, x_t.data_ptr(), x_t.shape[0], m, cand_t.data_ptr(),
                                               mass_t.data_ptr(), 1 if fused else 0, capi._stream(None)),
               "candidates")

    def set_default(self, m=8, threshold=0.99):
        _check(_lib().vlb200_router_set_default(self._h, m, threshold), "set_default")


def targets(post_t, tidx_t, tw_t):
    N, K = post_t.shape
    _check(_lib().vlb200_router_targets(post_t.data_ptr(), N, K, tidx_t.data_ptr(), tw_t.data_ptr()),
           "targets")


def missed_mass(qfull_t, qc_t) -> float:
    N, K = qfull_t.shape
    out = C.c_double(0)
    _check(_lib().vlb200_router_missed_mass(qfull_t.data_ptr(), qc_t.data_ptr(), N, K,
                                            C.byref(out)), "missed_mass")
    return out.value
