"""Python binding of the learned noise-PSD model (fft3d_psd_* in
include/fft3d_b200.h): a 544 -> 512 -> 512 -> 544 GELU MLP that predicts each
32x32 block's per-frequency noise power from its log power spectrum, trained on
the GPU from coloured-noise blocks the GPU generates. All work runs in the
library's sm_100a kernels; without a CUDA device every call raises.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .engine import FFT3DError, _check, lib

BINS, FEATURES, HIDDEN, OUTPUTS, INFO = 544, 576, 512, 640, 12
INFO_FIELDS = ("sigma", "a0", "a1", "a2", "a3", "rising", "gain", "frame", "x0", "y0", "sumh2", "pad")


class TrainCfg(ctypes.Structure):
    _fields_ = [("blocks", ctypes.c_longlong), ("batch", ctypes.c_int), ("epochs", ctypes.c_int),
                ("lr", ctypes.c_float), ("lr_final", ctypes.c_float), ("seed", ctypes.c_ulonglong),
                ("clean_frames", ctypes.c_int), ("width", ctypes.c_int), ("height", ctypes.c_int),
                ("sigma_min", ctypes.c_float), ("sigma_max", ctypes.c_float), ("knot_min", ctypes.c_float)]


_bound = False


def _bind():
    global _bound
    L = lib()
    if not _bound:
        vp, ci, ll, fp = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.POINTER(ctypes.c_float)
        cfgp = ctypes.POINTER(TrainCfg)
        L.fft3d_psd_train_default.argtypes = [cfgp]
        L.fft3d_psd_create.argtypes = [ci, ctypes.c_ulonglong, ci, ci, ci, ctypes.POINTER(vp)]
        L.fft3d_psd_destroy.argtypes = [vp]
        L.fft3d_psd_param_count.restype = ll
        L.fft3d_psd_get_params.argtypes = [vp, vp, ll]
        L.fft3d_psd_set_params.argtypes = [vp, vp, ll]
        L.fft3d_psd_train.argtypes = [vp, cfgp, vp, ci, fp]
        L.fft3d_psd_generate.argtypes = [vp, cfgp, ll, ll, vp, vp, vp, vp, vp]
        L.fft3d_psd_gradients.argtypes = [vp, vp, vp, ci, vp, fp]
        L.fft3d_psd_forward.argtypes = [vp, vp, ci, vp]
        L.fft3d_psd_train_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        _bound = True
    return L


def train_cfg(**kw) -> TrainCfg:
    """Training configuration: the library defaults (2^21 blocks, batch 4096,
    3 epochs, Adam 1e-3 -> 5e-5, 16 clean 1920x1080 frames, sigma 2..10,
    knots 0.1..1) with keyword overrides."""
    c = TrainCfg()
    _bind().fft3d_psd_train_default(ctypes.byref(c))
    for k, v in kw.items():
        if not hasattr(c, k):
            raise TypeError(f"unknown training setting {k!r}")
        setattr(c, k, v)
    return c


def _ptr(a):
    return None if a is None else a.ctypes.data


class PsdModel:
    """Learned noise-PSD model on one CUDA device, for 32x32 blocks with the
    analysis window of (ow, oh, wintype)."""

    def __init__(self, device: int = 0, seed: int = 1, ow: int = 16, oh: int = 16, wintype: int = 0):
        L = _bind()
        h = ctypes.c_void_p()
        _check(L.fft3d_psd_create(device, seed, ow, oh, wintype, ctypes.byref(h)))
        self.h = h
        self.nparam = int(L.fft3d_psd_param_count())

    def params(self) -> np.ndarray:
        out = np.empty(self.nparam, np.float32)
        _check(_bind().fft3d_psd_get_params(self.h, out.ctypes.data, self.nparam))
        return out

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        if p.size != self.nparam:
            raise FFT3DError(f"expected {self.nparam} parameters, got {p.size}")
        _check(_bind().fft3d_psd_set_params(self.h, p.ctypes.data, self.nparam))

    def train(self, cfg: TrainCfg | None = None, curve_len: int = 16, **kw):
        """Generate the training blocks on the GPU and train; returns
        (loss curve, held-out loss)."""
        cfg = cfg or train_cfg(**kw)
        curve = np.zeros(curve_len, np.float32)
        val = ctypes.c_float()
        _check(_bind().fft3d_psd_train(self.h, ctypes.byref(cfg), curve.ctypes.data, curve_len, ctypes.byref(val)))
        return curve, float(val.value)

    def train_stats(self) -> dict:
        """Device timing of the last train(): generation and training ms,
        steps, GEMM flops per step."""
        out = (ctypes.c_double * 4)()
        _check(_bind().fft3d_psd_train_stats(self.h, out))
        return dict(generate_ms=out[0], train_ms=out[1], steps=int(out[2]), gemm_flops_per_step=out[3])

    def generate(self, first: int, count: int, cfg: TrainCfg | None = None, **kw) -> dict:
        """The generator's blocks first .. first+count-1 (host copies)."""
        cfg = cfg or train_cfg(**kw)
        out = dict(features=np.empty((count, FEATURES), np.float32), target=np.empty((count, BINS), np.float32),
                   info=np.empty((count, INFO), np.float32), clean=np.empty((count, 32, 32), np.float32),
                   noisy=np.empty((count, 32, 32), np.uint8))
        _check(_bind().fft3d_psd_generate(self.h, ctypes.byref(cfg), first, count, *[_ptr(out[k]) for k in
                                          ("features", "target", "info", "clean", "noisy")]))
        return out

    def gradients(self, features: np.ndarray, target: np.ndarray):
        """(loss, gradient in the parameter layout) of one forward/backward pass."""
        x = np.ascontiguousarray(features, np.float32)
        t = np.ascontiguousarray(target, np.float32)
        g = np.empty(self.nparam, np.float32)
        loss = ctypes.c_float()
        _check(_bind().fft3d_psd_gradients(self.h, x.ctypes.data, t.ctypes.data, x.shape[0], g.ctypes.data,
                                           ctypes.byref(loss)))
        return float(loss.value), g

    def forward(self, features: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(features, np.float32)
        out = np.empty((x.shape[0], BINS), np.float32)
        _check(_bind().fft3d_psd_forward(self.h, x.ctypes.data, x.shape[0], out.ctypes.data))
        return out

    def close(self):
        if getattr(self, "h", None):
            _bind().fft3d_psd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
