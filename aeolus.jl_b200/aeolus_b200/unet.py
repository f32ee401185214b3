"""The learned U-Net preconditioner (include/aeolus_b200_unet.h).

    net = UNet((nx, ny, nz), seed=0)
    net.set_mask(fluid)               # 1 fluid, 0 solid (nz, ny, nx)
    net.set_out_scale(s)              # error scale (see `error_scale`)
    loss = net.train_step(r, e, lr)   # one Adam step on a residual -> error pair
    z = net.apply(r)                  # z ~ A^-1 r

Fields are interior-only float64 numpy arrays [k, j, i].  The network's
forward and backward passes and Adam run on the GPU (tcgen05 convolutions);
there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L

ACTIVATIONS = ("x", "e1a", "e1", "p1", "e2a", "e2", "p2", "e3a", "e3", "u2", "d2", "u1", "d1", "z")
LAYERS = (("e1a", 16, 16), ("e1", 16, 16), ("e2a", 16, 32), ("e2", 32, 32), ("e3a", 32, 32), ("e3", 32, 32),
          ("d2", 32, 16), ("d1", 16, 16), ("out", 16, 16))
_LEVEL = {"x": 0, "e1a": 0, "e1": 0, "p1": 1, "e2a": 1, "e2": 1, "p2": 2, "e3a": 2, "e3": 2, "u2": 1, "d2": 1,
          "u1": 0, "d1": 0, "z": 0}
_CH = {"x": 16, "e1a": 16, "e1": 16, "p1": 16, "e2a": 32, "e2": 32, "p2": 32, "e3a": 32, "e3": 32, "u2": 32,
       "d2": 16, "u1": 16, "d1": 16, "z": 1}

_D = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)


def _pd(a):
    return a.ctypes.data_as(_D)


def _pf(a):
    return a.ctypes.data_as(_F)


def split_params(flat):
    """{layer: (W[27, co, ci], b[co])} views of a flat parameter array."""
    out, o = {}, 0
    for name, ci, co in LAYERS:
        w = 27 * ci * co
        out[name] = (flat[o:o + w].reshape(27, co, ci), flat[o + w:o + w + co])
        o += w + co
    return out


def join_params(P):
    return np.concatenate([np.concatenate([P[n][0].ravel(), P[n][1].ravel()]) for n, _, _ in LAYERS]).astype(np.float32)


class UNet:
    def __init__(self, shape, seed=0, device=0):
        lib = L.load()
        nx, ny, nz = (int(v) for v in shape)
        self.shape = (nz, ny, nx)
        h = C.c_void_p()
        L.check(lib.aeo_unet_create(nx, ny, nz, int(seed), int(device), C.byref(h)), None, unet=True)
        self._h = h
        self.nparams = int(lib.aeo_unet_param_count())
        self.out_scale = 1.0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            L.load().aeo_unet_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def _chk(self, s):
        L.check(s, self._h, unet=True)

    def _arr(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.shape != self.shape:
            raise ValueError(f"array shape {a.shape} != {self.shape}")
        return a

    def params(self):
        p = np.empty(self.nparams, dtype=np.float32)
        self._chk(L.load().aeo_unet_get_params(self._h, _pf(p), None))
        return p

    def grads(self):
        g = np.empty(self.nparams, dtype=np.float32)
        self._chk(L.load().aeo_unet_get_params(self._h, None, _pf(g)))
        return g

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.nparams:
            raise ValueError("wrong parameter count")
        self._chk(L.load().aeo_unet_set_params(self._h, _pf(p)))

    def set_mask(self, fluid):
        m = np.ascontiguousarray(fluid, dtype=np.float32)
        if m.shape != self.shape:
            raise ValueError("mask shape")
        self._chk(L.load().aeo_unet_set_mask(self._h, _pf(m)))

    def set_out_scale(self, s):
        self._chk(L.load().aeo_unet_set_out_scale(self._h, float(s)))
        self.out_scale = float(s)

    def apply(self, r):
        r = self._arr(r)
        z = np.empty(self.shape)
        self._chk(L.load().aeo_unet_apply(self._h, _pd(r), _pd(z)))
        return z

    def gradients(self, r, e):
        r, e = self._arr(r), self._arr(e)
        loss = C.c_double()
        self._chk(L.load().aeo_unet_gradients(self._h, _pd(r), _pd(e), C.byref(loss)))
        return loss.value

    def train_step(self, r, e, lr=1e-3):
        r, e = self._arr(r), self._arr(e)
        loss = C.c_double()
        self._chk(L.load().aeo_unet_train_step(self._h, _pd(r), _pd(e), float(lr), C.byref(loss)))
        return loss.value

    def activation(self, name):
        lev = _LEVEL[name]
        nz, ny, nx = (v >> lev for v in self.shape)
        c = _CH[name]
        out = np.empty((nz, ny, nx, c) if c > 1 else (nz, ny, nx), dtype=np.float32)
        self._chk(L.load().aeo_unet_activation(self._h, ACTIVATIONS.index(name), _pf(out)))
        return out

    def profile(self, what="forward", reps=10):
        code = {"forward": 0, "train": 1, "conv": 2, "wgrad": 3}[what]
        ms = C.c_double()
        self._chk(L.load().aeo_unet_profile(self._h, code, int(reps), C.byref(ms)))
        return ms.value


def error_scale(pairs):
    """The RMS ratio |e| / |r| over training pairs: the output scale that
    makes the network's targets O(1)."""
    return float(np.mean([np.sqrt(np.mean(e ** 2)) / max(np.sqrt(np.mean(r ** 2)), 1e-300) for r, e in pairs]))
