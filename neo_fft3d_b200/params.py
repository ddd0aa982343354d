"""Parameter surface of neo_fft3d, as ctypes mirrors of include/fft3d_b200.h.

Names, meanings and defaults are the reference plugin's (src/fft3d.hpp:29-106):
``FFT3D(clip, sigma, beta, planes, bw, bh, bt, ow, oh, kratio, sharpen,
scutoff, svr, smin, smax, measure, interlaced, wintype, pframe, px, py, pshow,
pcutoff, pfactor, sigma2, sigma3, sigma4, degrid, dehalo, hr, ht, l, t, r, b,
opt, ncpu, mt)``; sigma2..4 default to sigma (src/fft3d.hpp:77-97).
"""
from __future__ import annotations

import ctypes

_FLOAT = ("sigma", "beta", "kratio", "sharpen", "scutoff", "svr", "smin", "smax", "pcutoff", "pfactor",
          "sigma2", "sigma3", "sigma4", "degrid", "dehalo", "hr", "ht")


class FFT3DParams(ctypes.Structure):
    _fields_ = [
        ("sigma", ctypes.c_float), ("beta", ctypes.c_float),
        ("bw", ctypes.c_int), ("bh", ctypes.c_int), ("bt", ctypes.c_int), ("ow", ctypes.c_int), ("oh", ctypes.c_int),
        ("kratio", ctypes.c_float), ("sharpen", ctypes.c_float), ("scutoff", ctypes.c_float), ("svr", ctypes.c_float),
        ("smin", ctypes.c_float), ("smax", ctypes.c_float),
        ("measure", ctypes.c_int), ("interlaced", ctypes.c_int), ("wintype", ctypes.c_int),
        ("pframe", ctypes.c_int), ("px", ctypes.c_int), ("py", ctypes.c_int), ("pshow", ctypes.c_int),
        ("pcutoff", ctypes.c_float), ("pfactor", ctypes.c_float),
        ("sigma2", ctypes.c_float), ("sigma3", ctypes.c_float), ("sigma4", ctypes.c_float),
        ("degrid", ctypes.c_float), ("dehalo", ctypes.c_float), ("hr", ctypes.c_float), ("ht", ctypes.c_float),
        ("l", ctypes.c_int), ("t", ctypes.c_int), ("r", ctypes.c_int), ("b", ctypes.c_int),
        ("opt", ctypes.c_int), ("ncpu", ctypes.c_int), ("mt", ctypes.c_int),
    ]


class PlaneDesc(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int), ("height", ctypes.c_int), ("bits", ctypes.c_int),
                ("is_chroma", ctypes.c_int), ("ssw", ctypes.c_int), ("ssh", ctypes.c_int),
                ("num_frames", ctypes.c_int), ("rgb", ctypes.c_int)]


DEFAULTS = dict(sigma=2.0, beta=1.0, bw=32, bh=32, bt=3, ow=-1, oh=-1, kratio=2.0, sharpen=0.0, scutoff=0.3,
                svr=1.0, smin=4.0, smax=20.0, measure=1, interlaced=0, wintype=0, pframe=0, px=0, py=0, pshow=0,
                pcutoff=0.1, pfactor=0.0, sigma2=None, sigma3=None, sigma4=None, degrid=1.0, dehalo=0.0, hr=2.0,
                ht=50.0, l=0, t=0, r=0, b=0, opt=0, ncpu=2, mt=0)


def make_params(**kw) -> FFT3DParams:
    """Resolve keyword arguments against the reference defaults. Unknown names
    raise TypeError; sigma2..4 fall back to sigma; crop values below 0 become 0
    (src/fft3d.hpp:135-138)."""
    unknown = set(kw) - set(DEFAULTS) - {"planes", "y", "u", "v"}
    if unknown:
        raise TypeError(f"unknown FFT3D argument(s): {sorted(unknown)}")
    v = dict(DEFAULTS)
    v.update({k: kw[k] for k in kw if k in DEFAULTS})
    for k in ("sigma2", "sigma3", "sigma4"):
        if v[k] is None:
            v[k] = v["sigma"]
    for k in ("l", "t", "r", "b"):
        v[k] = max(int(v[k]), 0)
    p = FFT3DParams()
    for name, _ in FFT3DParams._fields_:
        val = v[name]
        setattr(p, name, float(val) if name in _FLOAT else int(val))
    return p


def plane_descs(planes_shapes, bits: int, num_frames: int, yuv: bool = True):
    """PlaneDesc for every plane of a clip given [(h, w), ...] plane shapes."""
    h0, w0 = planes_shapes[0]
    out = []
    for i, (h, w) in enumerate(planes_shapes):
        ssw = 0 if i == 0 else max(0, (w0 // w).bit_length() - 1)
        ssh = 0 if i == 0 else max(0, (h0 // h).bit_length() - 1)
        out.append(PlaneDesc(w, h, bits, 1 if (yuv and 0 < i < 3) else 0, ssw, ssh, num_frames, 0 if yuv else 1))
    return out


def processed_planes(nplanes: int, planes=None, y=None, u=None, v=None):
    """Which planes are filtered: VapourSynth ``planes`` list (default all
    three), or AviSynth y/u/v modes (3 process, 2 copy), src/fft3d.hpp:149-169."""
    if planes is not None:
        sel = [p for p in (planes if isinstance(planes, (list, tuple)) else [planes]) if p < nplanes]
        return [i in sel for i in range(nplanes)]
    if y is not None or u is not None or v is not None:
        modes = [3 if y is None else y, 3 if u is None else u, 3 if v is None else v, 2]
        return [modes[i] == 3 for i in range(nplanes)]
    return [i < 3 for i in range(nplanes)]
