"""ctypes binding of the CPU restatement (oracle/lib/liboracle.so).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from neo_fft3d_b200.params import FFT3DParams, PlaneDesc, make_params, plane_descs, processed_planes

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "liboracle.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle not built ({LIB_PATH}); run make -C oracle restate")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.oracle_create.restype = vp
        L.oracle_create.argtypes = [ctypes.c_int, ctypes.POINTER(FFT3DParams), ctypes.POINTER(PlaneDesc)]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_filter.restype = ctypes.c_int
        L.oracle_filter.argtypes = [vp, ctypes.c_int, ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_int), vp,
                                    ctypes.c_int]
        L.oracle_geometry.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
        L.oracle_spectrum.argtypes = [vp, vp, ctypes.c_int, vp]
        L.oracle_last_filtered.argtypes = [vp, vp]
        L.oracle_gridsample.argtypes = [vp, vp]
        L.oracle_estimate_pattern.argtypes = [vp, vp, ctypes.c_int]
        L.oracle_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


class OraclePlane:
    """One plane engine of the restatement (float: dbl=False, FP64: dbl=True)."""

    def __init__(self, params: FFT3DParams, desc: PlaneDesc, dbl: bool = False):
        self.params, self.desc, self.dbl = params, desc, dbl
        self.h = lib().oracle_create(1 if dbl else 0, ctypes.byref(params), ctypes.byref(desc))
        if not self.h:
            raise ValueError(lib().oracle_last_error().decode())
        g = (ctypes.c_int * 8)()
        lib().oracle_geometry(self.h, g)
        self.nox, self.noy, self.coverw, self.coverh, self.outwidth, self.nblocks, self.ow, self.oh = list(g)
        self.bw, self.bh = params.bw, params.bh

    def spec_shape(self):
        return (self.nblocks, self.bh, self.outwidth)

    def filter(self, n: int, window, out: np.ndarray):
        """window: list of 5 arrays (or None) = frames n-2..n+2; out: plane array."""
        ptrs = (ctypes.c_void_p * 5)()
        strides = (ctypes.c_int * 5)()
        keep = []
        for i, a in enumerate(window):
            if a is not None:
                a = np.ascontiguousarray(a)
                keep.append(a)
                ptrs[i] = a.ctypes.data
                strides[i] = a.strides[0]
        rc = lib().oracle_filter(self.h, n, ptrs, strides, out.ctypes.data, out.strides[0])
        if rc != 0:
            raise RuntimeError(f"oracle_filter failed: {rc}")
        return out

    def spectrum(self, frame: np.ndarray) -> np.ndarray:
        frame = np.ascontiguousarray(frame)
        buf = np.empty(self.spec_shape() + (2,), np.float64)
        lib().oracle_spectrum(self.h, frame.ctypes.data, frame.strides[0], buf.ctypes.data)
        return buf[..., 0] + 1j * buf[..., 1]

    def last_filtered(self) -> np.ndarray:
        buf = np.empty(self.spec_shape() + (2,), np.float64)
        lib().oracle_last_filtered(self.h, buf.ctypes.data)
        return buf[..., 0] + 1j * buf[..., 1]

    def gridsample(self) -> np.ndarray:
        buf = np.empty((self.bh, self.outwidth, 2), np.float64)
        lib().oracle_gridsample(self.h, buf.ctypes.data)
        return buf[..., 0] + 1j * buf[..., 1]

    def estimate_pattern(self, frame: np.ndarray):
        frame = np.ascontiguousarray(frame)
        lib().oracle_estimate_pattern(self.h, frame.ctypes.data, frame.strides[0])

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_destroy(self.h)
            self.h = None


def window_of(plane: np.ndarray, n: int):
    """Frames n-2..n+2 of a [F,H,W] plane (None outside the clip)."""
    F = plane.shape[0]
    return [plane[n + d] if 0 <= n + d < F else None for d in range(-2, 3)]


def filter_clip(planes, dbl: bool = False, frames=None, bits=None, **kw):
    """Filter a whole clip (list of [F,H,W] planes) with the restatement, the
    way the plugin does: one engine per processed plane, frames in order,
    unprocessed planes copied. Returns the output planes."""
    F = planes[0].shape[0]
    if bits is None:
        bits = 8 if planes[0].dtype == np.uint8 else (32 if planes[0].dtype == np.float32 else 16)
    p = make_params(**kw)
    descs = plane_descs([a.shape[1:] for a in planes], bits, F)
    proc = processed_planes(len(planes), kw.get("planes"), kw.get("y"), kw.get("u"), kw.get("v"))
    frames = range(F) if frames is None else frames
    outs = []
    for i, a in enumerate(planes):
        o = np.empty((len(frames),) + a.shape[1:], a.dtype)
        if not proc[i]:
            o[:] = a[list(frames)]
            outs.append(o)
            continue
        eng = OraclePlane(p, descs[i], dbl)
        for j, n in enumerate(frames):
            eng.filter(n, window_of(a, n), o[j])
        outs.append(o)
    return outs
