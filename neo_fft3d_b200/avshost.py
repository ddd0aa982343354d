"""Python binding of the headless AviSynth+ host (csrc/avshost.cpp).

It loads any AviSynth+ plugin (``AvisynthPluginInit3``), invokes a registered
function with named arguments exactly as an AviSynth+ script would
(``neo_fft3d(clip, sigma=3, bt=5)``) and renders frames into numpy planes. Used
to run the AviSynth+ plugin shell of this package without an AviSynth+ install.
"""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np

from . import synth

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libfft3d_avshost.so")
PLUGIN_PATH = os.path.join(_HERE, "lib", "libneo_fft3d_avs.so")

FAMILY_Y, FAMILY_YUV, FAMILY_RGB, FAMILY_YUVA = 0, 1, 2, 3
MT_NICE_FILTER, MT_MULTI_INSTANCE, MT_SERIALIZED = 1, 2, 3

_lib = None


class AvisynthError(RuntimeError):
    """An error the plugin raised through IScriptEnvironment::ThrowError."""


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"headless AviSynth+ host not built: {LIB_PATH}")
        L = ctypes.CDLL(LIB_PATH)
        vp, cp, ci = ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int
        L.avsh_error.restype = cp
        L.avsh_create.restype = vp
        L.avsh_destroy.argtypes = [vp]
        L.avsh_pixel_type.argtypes = [ci, ci, ci, ci]
        L.avsh_load_plugin.argtypes = [vp, cp]
        L.avsh_function.argtypes = [vp, ci, ctypes.POINTER(cp), ctypes.POINTER(cp)]
        L.avsh_clip.restype = vp
        L.avsh_clip.argtypes = [vp, ci, ci, ci, ci, vp, ctypes.c_longlong]
        L.avsh_clip_free.argtypes = [vp]
        L.avsh_clip_info.argtypes = [vp, ctypes.POINTER(ci)]
        L.avsh_invoke.argtypes = [vp, cp, vp, ci, ctypes.POINTER(cp), cp, ctypes.POINTER(ci),
                                  ctypes.POINTER(ctypes.c_double), ctypes.POINTER(vp), ctypes.POINTER(ci)]
        L.avsh_get_frame.argtypes = [vp, vp, ci, ctypes.POINTER(vp), ctypes.POINTER(ci)]
        _lib = L
    return _lib


def available() -> bool:
    return os.path.exists(LIB_PATH) and os.path.exists(PLUGIN_PATH)


def param_slots(params: str):
    """(name, type) per slot of an AviSynth+ parameter string; unnamed slots
    have name None."""
    return [(m.group(1), m.group(2)) for m in re.finditer(r"(?:\[([^\]]*)\])?([a-z.*+])", params)]


class Clip:
    """A clip of the host: a source clip or a function's result."""

    def __init__(self, env, handle, shapes, mt_mode=None, keep=None):
        self.env, self.handle, self.shapes, self.mt_mode, self._keep = env, handle, shapes, mt_mode, keep

    def info(self):
        out = (ctypes.c_int * 4)()
        lib().avsh_clip_info(self.handle, out)
        return dict(width=out[0], height=out[1], pixel_type=out[2], frames=out[3])

    def frame(self, n: int):
        """Frame n as a list of [H, W] planes."""
        planes = [np.empty(s[1:], dtype=dt) for s, dt in self.shapes]
        ptrs = (ctypes.c_void_p * len(planes))(*[p.ctypes.data for p in planes])
        strides = (ctypes.c_int * len(planes))(*[p.strides[0] for p in planes])
        if lib().avsh_get_frame(self.env.handle, self.handle, n, ptrs, strides):
            raise AvisynthError(lib().avsh_error().decode())
        return planes

    def render(self, first=0, count=None, order=None):
        """Frames [first, first+count) in increasing order (or in ``order``,
        a list of frame numbers), as a list of [count, H, W] planes."""
        frames = self.shapes[0][0][0]
        if order is None:
            count = frames - first if count is None else count
            order = list(range(first, first + count))
        out = [np.empty((len(order),) + s[1:], dtype=dt) for s, dt in self.shapes]
        for i, n in enumerate(order):
            for o, p in zip(out, self.frame(n)):
                o[i] = p
        return out

    def __del__(self):
        if self.handle and _lib is not None:
            _lib.avsh_clip_free(self.handle)
            self.handle = None


class Env:
    """A headless AviSynth+ script environment with its loaded plugins."""

    def __init__(self):
        self.handle = lib().avsh_create()
        self._clips = []

    def load_plugin(self, path: str = PLUGIN_PATH, preload=()):
        """Load an AviSynth+ plugin; ``preload`` lists libraries loaded first
        with RTLD_GLOBAL (e.g. an FFTW-API library the plugin dlopen()s)."""
        for p in preload:
            ctypes.CDLL(p, mode=ctypes.RTLD_GLOBAL)
        if lib().avsh_load_plugin(self.handle, path.encode()):
            raise RuntimeError(f"cannot load plugin {path}: {lib().avsh_error().decode()}")

    def functions(self):
        """{name: parameter string} of every function the plugins registered."""
        out, k = {}, 0
        name, params = ctypes.c_char_p(), ctypes.c_char_p()
        while lib().avsh_function(self.handle, k, ctypes.byref(name), ctypes.byref(params)) == 0:
            out[name.value.decode()] = params.value.decode()
            k += 1
        return out

    def clip(self, planes, *, family=None, bits=None, ssw=None, ssh=None) -> Clip:
        """A source clip of numpy planes [F, H, W] (Y U V [A] or R G B [A])."""
        y = planes[0]
        frames, height, width = y.shape
        if bits is None:
            bits = 8 if y.dtype == np.uint8 else (32 if y.dtype == np.float32 else 16)
        if family is None:
            family = FAMILY_Y if len(planes) == 1 else (FAMILY_YUVA if len(planes) == 4 else FAMILY_YUV)
        if ssw is None:
            ssw = int(round(np.log2(width / planes[1].shape[2]))) if family in (FAMILY_YUV, FAMILY_YUVA) else 0
        if ssh is None:
            ssh = int(round(np.log2(height / planes[1].shape[1]))) if family in (FAMILY_YUV, FAMILY_YUVA) else 0
        pt = lib().avsh_pixel_type(family, bits, ssw, ssh)
        if pt == -1:
            raise ValueError(f"no AviSynth+ format for family {family}, {bits} bits, subsampling {ssw}/{ssh}")
        buf = synth.pack(planes)
        h = lib().avsh_clip(self.handle, width, height, pt, frames, buf.ctypes.data, buf.size // frames)
        return Clip(self, h, [(p.shape, p.dtype) for p in planes])

    def invoke(self, name: str, clip: Clip, **kwargs) -> Clip:
        """name(clip, **kwargs): ints, floats and bools by the function's
        parameter types (an int given for a float parameter is passed as a
        float, as the AviSynth+ parser does)."""
        slots = dict(param_slots(self.functions()[name]))
        n = len(kwargs)
        names = (ctypes.c_char_p * max(n, 1))()
        kinds = ctypes.create_string_buffer(max(n, 1))
        ints = (ctypes.c_int * max(n, 1))()
        floats = (ctypes.c_double * max(n, 1))()
        for i, (k, v) in enumerate(kwargs.items()):
            names[i] = k.encode()
            t = slots.get(k, "i")
            if t == "b" or isinstance(v, bool):
                kinds[i], ints[i] = b"b", int(bool(v))
            elif t == "f":
                kinds[i], floats[i] = b"f", float(v)
            else:
                if not float(v).is_integer():
                    raise TypeError(f"{name}: {k} is an int parameter")
                kinds[i], ints[i] = b"i", int(v)
        out, mt = ctypes.c_void_p(), ctypes.c_int()
        if lib().avsh_invoke(self.handle, name.encode(), clip.handle, n, names, kinds.raw, ints, floats,
                             ctypes.byref(out), ctypes.byref(mt)):
            raise AvisynthError(lib().avsh_error().decode())
        return Clip(self, out.value, clip.shapes, mt_mode=mt.value, keep=clip)

    def __del__(self):
        if self.handle and _lib is not None:
            _lib.avsh_destroy(self.handle)
            self.handle = None
