"""Python binding of the C ABI in include/fft3d_b200.h (lib/libfft3d_b200.so).

This is a thin ctypes layer: all work runs in the sm_100a kernels of the
library. There is no CPU fallback; if the library or a CUDA device is missing,
every call raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .params import FFT3DParams, PlaneDesc, make_params, plane_descs, processed_planes

_HERE = os.path.dirname(os.path.abspath(__file__))
# NEO_FFT3D_LIB: another build of the same library (A/B measurements)
LIB_PATH = os.environ.get("NEO_FFT3D_LIB") or os.path.join(_HERE, "lib", "libfft3d_b200.so")
_lib = None

SYMBOLS = ("fft3d_params_default", "fft3d_plane_create", "fft3d_plane_filter", "fft3d_plane_filter_device",
           "fft3d_plane_cached", "fft3d_plane_spectrum", "fft3d_plane_geometry", "fft3d_plane_set_pattern_frame",
           "fft3d_plane_reset", "fft3d_plane_destroy", "fft3d_last_error", "fft3d_kernel_launches",
           "fft3d_plane_set_timing", "fft3d_plane_timing", "fft3d_plane_device_bytes", "fft3d_plane_synchronize",
           "fft3d_plane_debug_set_error_flag")
KERNELS = ("forward", "filter_inverse", "overlap_add", "fused", "filter_bins")


class FFT3DError(RuntimeError):
    pass


def lib():
    """Load the native library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FFT3DError(f"neo_fft3d_b200 native library not built: {LIB_PATH}")
        L = ctypes.CDLL(LIB_PATH)
        vp, ci = ctypes.c_void_p, ctypes.c_int
        L.fft3d_params_default.argtypes = [ctypes.POINTER(FFT3DParams)]
        L.fft3d_plane_create.argtypes = [ctypes.POINTER(FFT3DParams), ctypes.POINTER(PlaneDesc), ci,
                                         ctypes.POINTER(vp)]
        L.fft3d_plane_filter.argtypes = [vp, ci, ctypes.POINTER(vp), ctypes.POINTER(ci), vp, ci]
        L.fft3d_plane_filter_device.argtypes = [vp, ci, ctypes.POINTER(vp), ctypes.POINTER(ci), vp, ci, vp]
        L.fft3d_plane_filter_frames_device.argtypes = [vp, ci, ci, ctypes.POINTER(vp), ctypes.POINTER(ci),
                                                       ctypes.POINTER(vp), ctypes.POINTER(ci), vp]
        L.fft3d_plane_filter_frames.argtypes = [vp, ci, ci, ctypes.POINTER(vp), ctypes.POINTER(ci),
                                                ctypes.POINTER(vp), ctypes.POINTER(ci)]
        L.fft3d_plane_cached.argtypes = [vp, ci]
        L.fft3d_plane_spectrum.argtypes = [vp, ci, vp]
        L.fft3d_plane_geometry.argtypes = [vp, ctypes.POINTER(ci)]
        L.fft3d_plane_set_pattern_frame.argtypes = [vp, vp, ci]
        L.fft3d_plane_reset.argtypes = [vp]
        L.fft3d_plane_destroy.argtypes = [vp]
        L.fft3d_last_error.restype = ctypes.c_char_p
        L.fft3d_kernel_launches.restype = ctypes.c_uint64
        L.fft3d_plane_device_bytes.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64)]
        L.fft3d_plane_synchronize.argtypes = [vp]
        L.fft3d_plane_debug_set_error_flag.argtypes = [vp, ci]
        L.fft3d_plane_set_timing.argtypes = [vp, ci]
        L.fft3d_plane_timing.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        L.fft3d_plane_set_psd.argtypes = [vp, vp, ci, ctypes.c_float]
        L.fft3d_batch_create.argtypes = [ci, ctypes.POINTER(vp)]
        L.fft3d_batch_destroy.argtypes = [vp]
        L.fft3d_batch_set_tuning.argtypes = [vp, ci]
        L.fft3d_batch_step.argtypes = [vp, ci, ctypes.POINTER(vp), ctypes.POINTER(ci), ctypes.POINTER(vp),
                                       ctypes.POINTER(ci), ctypes.POINTER(vp), ctypes.POINTER(ci), vp]
        L.fft3d_batch_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        L.fft3d_batch_set_timing.argtypes = [vp, ci]
        L.fft3d_batch_timing.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        _lib = L
    return _lib


def _check(rc: int):
    if rc != 0:
        raise FFT3DError(f"{lib().fft3d_last_error().decode()} (status {rc})")


def kernel_launches() -> int:
    return int(lib().fft3d_kernel_launches())


class PlaneEngine:
    """One GPU plane engine (the counterpart of the reference's FFT3DEngine)."""

    def __init__(self, params: FFT3DParams, desc: PlaneDesc, device: int = 0):
        self.params, self.desc = params, desc
        h = ctypes.c_void_p()
        _check(lib().fft3d_plane_create(ctypes.byref(params), ctypes.byref(desc), device, ctypes.byref(h)))
        self.h = h
        g = (ctypes.c_int * 8)()
        _check(lib().fft3d_plane_geometry(self.h, g))
        self.nox, self.noy, self.coverw, self.coverh, self.outwidth, self.nblocks, self.ow, self.oh = list(g)

    def filter(self, n: int, window, out: np.ndarray) -> np.ndarray:
        """Filter frame n from host arrays. window: frames n-2..n+2 (None where
        absent or already cached); out: the output plane (written in place)."""
        ptrs = (ctypes.c_void_p * 5)()
        strides = (ctypes.c_int * 5)()
        keep = []
        for i, a in enumerate(window):
            if a is not None:
                a = np.ascontiguousarray(a)
                keep.append(a)
                ptrs[i] = a.ctypes.data
                strides[i] = a.strides[0]
        _check(lib().fft3d_plane_filter(self.h, n, ptrs, strides, out.ctypes.data, out.strides[0]))
        return out

    def filter_device(self, n: int, ptrs, strides, dst_ptr: int, dst_stride: int, stream: int = 0):
        """Filter frame n from device pointers (ints); queued on `stream`."""
        p = (ctypes.c_void_p * 5)(*[x or None for x in ptrs])
        s = (ctypes.c_int * 5)(*strides)
        _check(lib().fft3d_plane_filter_device(self.h, n, p, s, ctypes.c_void_p(dst_ptr), dst_stride,
                                               ctypes.c_void_p(stream) if stream else None))

    def filter_frames_device(self, n0: int, ptrs, strides, dst_ptrs, dst_strides, stream: int = 0):
        """Filter frames n0 .. n0 + len(dst_ptrs) - 1 in one call (a frame
        group): ptrs[j] / strides[j] are frame n0 - 2 + j (len(dst_ptrs) + 4
        entries, 0 outside the clip); queued on `stream`."""
        count = len(dst_ptrs)
        if len(ptrs) != count + 4 or len(strides) != count + 4 or len(dst_strides) != count:
            raise ValueError("filter_frames_device: ptrs/strides need count + 4 entries, dst_strides count")
        p = (ctypes.c_void_p * (count + 4))(*[x or None for x in ptrs])
        s = (ctypes.c_int * (count + 4))(*strides)
        d = (ctypes.c_void_p * count)(*dst_ptrs)
        ds = (ctypes.c_int * count)(*dst_strides)
        _check(lib().fft3d_plane_filter_frames_device(self.h, n0, count, p, s, d, ds,
                                                      ctypes.c_void_p(stream) if stream else None))

    def filter_frames(self, n0: int, srcs, dsts):
        """Filter frames n0 .. n0 + len(dsts) - 1 from host frames in one call
        (a frame group): srcs[j] is frame n0 - 2 + j (len(dsts) + 4 entries,
        None outside the clip or when cached), dsts[j] receives frame n0 + j
        (2D arrays, rows contiguous)."""
        count = len(dsts)
        if len(srcs) != count + 4:
            raise ValueError("filter_frames: srcs needs len(dsts) + 4 entries")
        p = (ctypes.c_void_p * (count + 4))(*[None if a is None else a.ctypes.data for a in srcs])
        s = (ctypes.c_int * (count + 4))(*[0 if a is None else a.strides[0] for a in srcs])
        d = (ctypes.c_void_p * count)(*[a.ctypes.data for a in dsts])
        ds = (ctypes.c_int * count)(*[a.strides[0] for a in dsts])
        _check(lib().fft3d_plane_filter_frames(self.h, n0, count, p, s, d, ds))

    def cached(self, n: int) -> bool:
        return bool(lib().fft3d_plane_cached(self.h, n))

    def spectrum(self, n: int) -> np.ndarray:
        buf = np.empty((self.nblocks, self.params.bh, self.outwidth, 2), np.float32)
        _check(lib().fft3d_plane_spectrum(self.h, n, buf.ctypes.data))
        return buf[..., 0] + 1j * buf[..., 1].astype(np.complex64)

    def set_pattern_frame(self, frame: np.ndarray):
        frame = np.ascontiguousarray(frame)
        _check(lib().fft3d_plane_set_pattern_frame(self.h, frame.ctypes.data, frame.strides[0]))

    def set_psd(self, model, pooled: bool = False, strength: float = 3.0):
        """Take the Wiener/Kalman noise power from a learned PSD model
        (neo_fft3d_b200.psd.PsdModel), times `strength`, instead of sigma;
        None returns to sigma."""
        _check(lib().fft3d_plane_set_psd(self.h, model.h if model is not None else None, 1 if pooled else 0,
                                         strength))
        self._psd_model = model  # the model must outlive its use by this plane

    def set_timing(self, enable: bool):
        _check(lib().fft3d_plane_set_timing(self.h, 1 if enable else 0))

    def timing(self) -> dict:
        """{kernel: (launches, milliseconds, algorithmic bytes)}; resets the counters."""
        out = (ctypes.c_double * 15)()
        _check(lib().fft3d_plane_timing(self.h, out))
        return {k: (out[3 * i], out[3 * i + 1], out[3 * i + 2]) for i, k in enumerate(KERNELS)}

    def reset(self):
        _check(lib().fft3d_plane_reset(self.h))

    def device_bytes(self) -> int:
        out = ctypes.c_uint64()
        _check(lib().fft3d_plane_device_bytes(self.h, ctypes.byref(out)))
        return int(out.value)

    def synchronize(self):
        """Wait for the plane's queued work; raises on a device-side wait that ran out."""
        _check(lib().fft3d_plane_synchronize(self.h))

    def close(self):
        if getattr(self, "h", None):
            lib().fft3d_plane_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Batched multi-plane scheduler (fft3d_batch_*): one step filters one
    frame of each of many planes with batched, tuned, graph-captured launches."""

    def __init__(self, device: int = 0, tuning: bool = True):
        h = ctypes.c_void_p()
        _check(lib().fft3d_batch_create(device, ctypes.byref(h)))
        self.h = h
        _check(lib().fft3d_batch_set_tuning(self.h, 1 if tuning else 0))

    class Prepared(tuple):
        """C arrays of a step's items (Batch.prepare)."""

    @staticmethod
    def prepare(items):
        """The C arrays of a step's items, for repeated steps over fixed buffers."""
        k = len(items)
        return Batch.Prepared((k, (ctypes.c_void_p * k)(*[it[0].h.value for it in items]),
                               (ctypes.c_int * k)(*[it[1] for it in items]),
                               (ctypes.c_void_p * (5 * k))(*[p or None for it in items for p in it[2]]),
                               (ctypes.c_int * (5 * k))(*[x for it in items for x in it[3]]),
                               (ctypes.c_void_p * k)(*[it[4] for it in items]),
                               (ctypes.c_int * k)(*[it[5] for it in items])))

    def step(self, items, stream: int = 0):
        """items: list of (PlaneEngine, n, src_ptrs[5], src_strides[5], dst_ptr, dst_stride),
        or the result of prepare(items). A plane may appear with consecutive
        frames n, n + 1, ... (a frame group; not for Kalman planes)."""
        k, planes, ns, src, sst, dst, dstr = items if isinstance(items, Batch.Prepared) else self.prepare(items)
        _check(lib().fft3d_batch_step(self.h, k, planes, ns, src, sst, dst, dstr,
                                      ctypes.c_void_p(stream) if stream else None))

    def set_timing(self, enable: bool = True):
        """Per-phase kernel timing of tuned steps (they then run without their graph)."""
        _check(lib().fft3d_batch_set_timing(self.h, 1 if enable else 0))

    def timing(self) -> dict:
        """{phase: (launches, ms, algorithmic bytes)} since creation (waits for the timed launches)."""
        out = (ctypes.c_double * 12)()
        _check(lib().fft3d_batch_timing(self.h, out))
        names = ("forward", "filter_inverse", "copy", "overlap_add")
        return {k: (int(out[3 * i]), out[3 * i + 1], out[3 * i + 2]) for i, k in enumerate(names)}

    def stats(self) -> dict:
        out = (ctypes.c_double * 8)()
        _check(lib().fft3d_batch_stats(self.h, out))
        return dict(steps=int(out[0]), graph_launches=int(out[1]), tuning_steps=int(out[2]),
                    kernels_last_step=int(out[4]), step_shapes=int(out[5]), wave_budget_mib=int(out[6]),
                    host_ms_planning=out[3], host_ms_steps=out[7])

    def close(self):
        if getattr(self, "h", None):
            lib().fft3d_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def filter_clip(planes, frames=None, bits=None, device: int = 0, psd=None, psd_pooled=False, psd_strength=3.0, **kw):
    """FFT3D(clip, **kw) on the GPU for a clip given as a list of [F,H,W] host
    planes, the way the plugin drives its engines: one engine per processed
    plane, frames in order, unprocessed planes copied. Returns output planes.
    psd: a learned noise-PSD model used in place of sigma (PlaneEngine.set_psd),
    with psd_pooled / psd_strength as there."""
    F = planes[0].shape[0]
    if bits is None:
        bits = 8 if planes[0].dtype == np.uint8 else (32 if planes[0].dtype == np.float32 else 16)
    p = make_params(**kw)
    descs = plane_descs([a.shape[1:] for a in planes], bits, F)
    proc = processed_planes(len(planes), kw.get("planes"), kw.get("y"), kw.get("u"), kw.get("v"))
    frames = list(range(F)) if frames is None else list(frames)
    outs = []
    for i, a in enumerate(planes):
        o = np.empty((len(frames),) + a.shape[1:], a.dtype)
        if not proc[i]:
            o[:] = a[frames]
            outs.append(o)
            continue
        eng = PlaneEngine(p, descs[i], device)
        if psd is not None:
            eng.set_psd(psd, psd_pooled, psd_strength)
        if p.pfactor != 0:
            eng.set_pattern_frame(a[min(max(p.pframe, 0), F - 1)])
        for j, n in enumerate(frames):
            win = [a[n + d] if 0 <= n + d < F else None for d in range(-2, 3)]
            eng.filter(n, win, o[j])
        eng.close()
        outs.append(o)
    return outs
