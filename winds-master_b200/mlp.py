"""ctypes binding of ``include/winds_mlp.h``: the bound-circulation MLP
(BF16 tensor-core GEMMs with FP32 accumulation, Adam training on the GPU)
that gives the Kutta-Joukowski iteration its initial guess."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .bs import _check, lib


class MlpConfigC(C.Structure):
    _fields_ = [("n_in", C.c_int), ("seed", C.c_ulonglong)]


class MlpTrainC(C.Structure):
    _fields_ = [("epochs", C.c_int), ("batch", C.c_int), ("lr", C.c_float), ("beta1", C.c_float),
                ("beta2", C.c_float), ("eps", C.c_float), ("weight_decay", C.c_float),
                ("seed", C.c_ulonglong)]


def _bind():
    L = lib()
    if not hasattr(L, "_mlp_bound"):
        L.winds_mlp_create.argtypes = [C.POINTER(MlpConfigC), C.POINTER(C.c_void_p)]
        L.winds_mlp_param_count.argtypes = [C.c_void_p]
        L.winds_mlp_param_count.restype = C.c_longlong
        L.winds_mlp_get_params.argtypes = [C.c_void_p, C.c_void_p]
        L.winds_mlp_set_params.argtypes = [C.c_void_p, C.c_void_p]
        L.winds_mlp_set_scaling.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float]
        L.winds_mlp_get_scaling.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_float)]
        L.winds_mlp_set_base.argtypes = [C.c_void_p, C.c_int]
        L.winds_mlp_get_base.argtypes = [C.c_void_p]
        L.winds_mlp_forward_host.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p]
        L.winds_mlp_loss_grad_host.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong,
                                               C.POINTER(C.c_double), C.c_void_p]
        L.winds_mlp_train_host.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong,
                                           C.POINTER(MlpTrainC), C.c_void_p]
        L.winds_mlp_train_stats.argtypes = [C.c_void_p, C.POINTER(C.c_double),
                                            C.POINTER(C.c_longlong)]
        L.winds_mlp_destroy.argtypes = [C.c_void_p]
        L._mlp_bound = True
    return L


def _f32(a, cols=None):
    x = np.ascontiguousarray(a, dtype=np.float32)
    if cols is not None and (x.ndim != 2 or x.shape[1] != cols):
        raise ValueError(f"expected rows of {cols} features, got {x.shape}")
    return x


class Mlp:
    """The network on the current device. ``n_in`` features per row."""

    def __init__(self, n_in: int, seed: int = 0):
        L = _bind()
        h = C.c_void_p()
        _check(L.winds_mlp_create(C.byref(MlpConfigC(int(n_in), int(seed))), C.byref(h)))
        self.h = h
        self.n_in = int(n_in)
        self.n_param = int(L.winds_mlp_param_count(h))

    @property
    def params(self) -> np.ndarray:
        th = np.zeros(self.n_param, dtype=np.float32)
        _check(_bind().winds_mlp_get_params(self.h, th.ctypes.data))
        return th

    @params.setter
    def params(self, theta):
        th = _f32(theta)
        if th.size != self.n_param:
            raise ValueError("parameter vector length")
        _check(_bind().winds_mlp_set_params(self.h, th.ctypes.data))

    def set_scaling(self, shift, scale, out_scale=1.0):
        sh, sc = _f32(shift), _f32(scale)
        _check(_bind().winds_mlp_set_scaling(self.h, sh.ctypes.data, sc.ctypes.data, float(out_scale)))

    BASES = {"previous": 0, "extrapolated": 1}

    def set_base(self, base="previous"):
        """What the wake engine adds the scaled output to: the previous step's
        converged bound circulation, or its linear extrapolation over the last
        two steps (``"extrapolated"``: the network then learns the residual)."""
        _check(_bind().winds_mlp_set_base(self.h, self.BASES[base]))

    @property
    def base(self) -> str:
        k = int(_bind().winds_mlp_get_base(self.h))
        return {v: n for n, v in self.BASES.items()}[k]

    def scaling(self):
        sh = np.zeros(self.n_in, np.float32)
        sc = np.zeros(self.n_in, np.float32)
        o = C.c_float()
        _check(_bind().winds_mlp_get_scaling(self.h, sh.ctypes.data, sc.ctypes.data, C.byref(o)))
        return sh, sc, o.value

    def forward(self, x) -> np.ndarray:
        x = _f32(x, self.n_in)
        y = np.zeros(x.shape[0], dtype=np.float32)
        _check(_bind().winds_mlp_forward_host(self.h, x.ctypes.data, x.shape[0], y.ctypes.data))
        return y

    def loss_grad(self, x, t):
        x = _f32(x, self.n_in)
        t = _f32(t)
        g = np.zeros(self.n_param, dtype=np.float32)
        loss = C.c_double()
        _check(_bind().winds_mlp_loss_grad_host(self.h, x.ctypes.data, t.ctypes.data, x.shape[0],
                                                C.byref(loss), g.ctypes.data))
        return loss.value, g

    def train(self, x, t, epochs=10, batch=4096, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8,
              weight_decay=0.0, seed=0) -> np.ndarray:
        x = _f32(x, self.n_in)
        t = _f32(t)
        p = MlpTrainC(int(epochs), int(batch), float(lr), float(beta1), float(beta2), float(eps),
                      float(weight_decay), int(seed))
        el = np.zeros(max(1, int(epochs)), dtype=np.float32)
        _check(_bind().winds_mlp_train_host(self.h, x.ctypes.data, t.ctypes.data, x.shape[0],
                                            C.byref(p), el.ctypes.data))
        return el[:epochs]

    def train_stats(self):
        ms, n = C.c_double(), C.c_longlong()
        _check(_bind().winds_mlp_train_stats(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def close(self):
        if getattr(self, "h", None):
            _bind().winds_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
