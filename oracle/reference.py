"""Run the UNMODIFIED reference plugin (oracle/_ref) on a clip.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py). The plugin is built from
the reference's own sources by ``make -C oracle ref`` and driven through the
headless VapourSynth host exactly as ``core.neo_fft3d.FFT3D(clip, ...)``.
"""
from __future__ import annotations

import os

from neo_fft3d_b200 import vshost

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(_HERE, "_ref", "libneo_fft3d_ref.so")
SHIM_SO = os.path.join(_HERE, "_ref", "libfftw3f_threads.so")

_core = None


def available() -> bool:
    return os.path.exists(REF_SO) and os.path.exists(SHIM_SO) and os.path.exists(vshost.LIB_PATH)


def core():
    global _core
    if _core is None:
        if not available():
            raise RuntimeError("reference plugin not built (make -C oracle ref)")
        c = vshost.Core()
        c.load_plugin(REF_SO, preload=[SHIM_SO])
        _core = c
    return _core


def run(clip_planes, threads: int = 1, first: int = 0, count=None, bits=None, **kw):
    """core.neo_fft3d.FFT3D(clip, **kw) rendered over frames [first, first+count).
    ``bits``: bit depth of uint16 planes (default 16)."""
    c = core()
    clip = c.clip(clip_planes, bits=bits)
    out = c.invoke("neo_fft3d", "FFT3D", clip, **kw)
    return out.render(first=first, count=count, threads=threads)
