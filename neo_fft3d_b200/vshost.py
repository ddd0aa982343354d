"""Python binding of the headless VapourSynth API v3.6 host (csrc/vshost.cpp).

It loads any VapourSynth plugin, invokes a registered filter with keyword
arguments exactly as a VapourSynth script would (``core.ns.Func(clip, ...)``)
and renders frames into numpy planes. Used to run the GPU plugin shell of this
package without a VapourSynth install.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import synth

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libfft3d_vshost.so")

CM_GRAY, CM_RGB, CM_YUV = 1000000, 2000000, 3000000
ST_INTEGER, ST_FLOAT = 0, 1

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"headless VS host not built: {LIB_PATH}")
        L = ctypes.CDLL(LIB_PATH)
        vp, cp, ci = ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int
        L.vsh_core_new.restype = vp
        L.vsh_core_free.argtypes = [vp]
        L.vsh_load_plugin.restype = vp
        L.vsh_load_plugin.argtypes = [vp, cp]
        L.vsh_last_error.restype = cp
        L.vsh_plugin_namespace.restype = cp
        L.vsh_plugin_namespace.argtypes = [vp]
        L.vsh_function_args.restype = cp
        L.vsh_function_args.argtypes = [vp, cp]
        L.vsh_map_new.restype = vp
        L.vsh_map_free.argtypes = [vp]
        L.vsh_map_set_int.argtypes = [vp, cp, ctypes.c_int64, ci]
        L.vsh_map_set_float.argtypes = [vp, cp, ctypes.c_double, ci]
        L.vsh_map_set_node.argtypes = [vp, cp, vp]
        L.vsh_map_error.restype = cp
        L.vsh_map_error.argtypes = [vp]
        L.vsh_map_get_node.restype = vp
        L.vsh_map_get_node.argtypes = [vp, cp]
        L.vsh_invoke.restype = vp
        L.vsh_invoke.argtypes = [vp, vp, cp, vp]
        L.vsh_clip_new.restype = vp
        L.vsh_clip_new.argtypes = [vp, ci, ci, ci, ci, ci, ci, ci, ci, vp]
        L.vsh_node_free.argtypes = [vp]
        L.vsh_node_info.argtypes = [vp, ctypes.POINTER(ci)]
        L.vsh_render.restype = ci
        L.vsh_render.argtypes = [vp, ci, ci, ci, vp]
        _lib = L
    return _lib


class Clip:
    """A node of the headless host (source clip or filter output)."""

    def __init__(self, core, handle, keep=None):
        self.core, self.handle, self._keep = core, handle, keep

    def info(self):
        out = (ctypes.c_int * 8)()
        lib().vsh_node_info(self.handle, out)
        w, h, n, cf, bits, ssw, ssh, planes = list(out)
        return dict(width=w, height=h, frames=n, color_family=cf, bits=bits, ssw=ssw, ssh=ssh, planes=planes)

    def plane_shapes(self):
        i = self.info()
        dt = np.uint8 if i["bits"] <= 8 else (np.uint16 if i["bits"] <= 16 else np.float32)
        shapes = []
        for p in range(i["planes"]):
            w = i["width"] >> i["ssw"] if p else i["width"]
            h = i["height"] >> i["ssh"] if p else i["height"]
            shapes.append(((i["frames"], h, w), dt))
        return shapes

    def render(self, first=0, count=None, threads=1):
        """Render frames [first, first+count) and return them as a list of planes."""
        shapes = self.plane_shapes()
        total = shapes[0][0][0]
        count = total - first if count is None else count
        shapes = [((count,) + s[1:], dt) for s, dt in shapes]
        fb = sum(int(np.prod(s[1:])) * np.dtype(dt).itemsize for s, dt in shapes)
        buf = np.empty(fb * count, np.uint8)
        rc = lib().vsh_render(self.handle, first, count, threads, buf.ctypes.data)
        if rc != 0:
            raise RuntimeError(lib().vsh_last_error().decode())
        return synth.unpack(buf, shapes)

    def __del__(self):
        try:
            if self.handle:
                lib().vsh_node_free(self.handle)
        except Exception:
            pass
        self.handle = None


class Core:
    """A headless VapourSynth core with its loaded plugins."""

    def __init__(self):
        self.handle = lib().vsh_core_new()
        self.plugins = {}

    def load_plugin(self, path: str, preload=()):
        """Load a VS plugin .so; ``preload`` lists libraries loaded first with
        RTLD_GLOBAL (e.g. an FFTW-API library the plugin dlopen()s by name)."""
        for p in preload:
            ctypes.CDLL(p, mode=ctypes.RTLD_GLOBAL)
        h = lib().vsh_load_plugin(self.handle, path.encode())
        if not h:
            raise RuntimeError(f"cannot load plugin {path}: {lib().vsh_last_error().decode()}")
        ns = lib().vsh_plugin_namespace(h).decode()
        self.plugins[ns] = h
        return ns

    def function_args(self, ns: str, name: str):
        a = lib().vsh_function_args(self.plugins[ns], name.encode())
        return a.decode() if a else None

    def clip(self, planes, *, color_family=CM_YUV, bits=None, ssw=None, ssh=None) -> Clip:
        """Wrap numpy planes [F,H,W] (list) as a source clip (the buffer is kept alive)."""
        y = planes[0]
        frames, height, width = y.shape
        if bits is None:
            bits = 8 if y.dtype == np.uint8 else (32 if y.dtype == np.float32 else 16)
        st = ST_FLOAT if y.dtype == np.float32 else ST_INTEGER
        if len(planes) == 1:
            color_family, ssw, ssh = CM_GRAY, 0, 0
        if ssw is None:
            ssw = int(round(np.log2(width / planes[1].shape[2])))
        if ssh is None:
            ssh = int(round(np.log2(height / planes[1].shape[1])))
        buf = synth.pack(planes)
        h = lib().vsh_clip_new(self.handle, color_family, st, bits, ssw, ssh, width, height, frames, buf.ctypes.data)
        return Clip(self, h, keep=buf)

    def invoke(self, ns: str, name: str, clip: Clip, **kwargs) -> Clip:
        """core.<ns>.<name>(clip, **kwargs). Lists become array arguments; bools
        become ints (VapourSynth has no boolean type)."""
        L = lib()
        m = L.vsh_map_new()
        try:
            L.vsh_map_set_node(m, b"clip", clip.handle)
            for k, v in kwargs.items():
                vals = v if isinstance(v, (list, tuple)) else [v]
                for i, x in enumerate(vals):
                    app = 1 if i else 0
                    if isinstance(x, (bool, np.bool_)):
                        L.vsh_map_set_int(m, k.encode(), int(x), app)
                    elif isinstance(x, (int, np.integer)):
                        L.vsh_map_set_int(m, k.encode(), int(x), app)
                    else:
                        L.vsh_map_set_float(m, k.encode(), float(x), app)
            out = L.vsh_invoke(self.handle, self.plugins[ns], name.encode(), m)
            try:
                err = L.vsh_map_error(out)
                if err:
                    raise RuntimeError(err.decode())
                node = L.vsh_map_get_node(out, b"clip")
                return Clip(self, node, keep=clip)
            finally:
                L.vsh_map_free(out)
        finally:
            L.vsh_map_free(m)
