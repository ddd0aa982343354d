"""Sample formats beyond 8/10-bit YUV through the VapourSynth plugin shell,
against the reference plugin in the same headless host: Gray, planar RGB
(no chroma offset, full-size planes), 12- and 16-bit YUV420 and 32-bit float
YUV444 (the reference clamps every float plane to [0, 1])."""
import os

import numpy as np
import pytest

from neo_fft3d_b200 import synth, vshost
from oracle import reference

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PLUGIN = os.path.join(ROOT, "neo_fft3d_b200", "lib", "libneo_fft3d_vs.so")

needs_ref = pytest.mark.skipif(not reference.available(), reason="reference plugin not built")


def _clip(fmt):
    if fmt in ("rgb8", "yuv444ps"):
        p = synth.make_clip(160, 128, 6, noise_sigma=5, seed=99, ssw=0, ssh=0)
    else:
        p = synth.make_clip(160, 128, 6, noise_sigma=5, seed=99)
    if fmt == "gray8":
        return [p[0]], dict(color_family=vshost.CM_GRAY), None
    if fmt == "rgb8":
        return p, dict(color_family=vshost.CM_RGB), None
    if fmt == "yuv420p12":
        return [a.astype(np.uint16) << 4 for a in p], dict(bits=12), 12
    if fmt == "yuv420p16":
        return [a.astype(np.uint16) * 257 for a in p], dict(bits=16), 16
    return [a.astype(np.float32) / 255.0 for a in p], dict(), None


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("fmt", ["gray8", "rgb8", "yuv420p12", "yuv420p16", "yuv444ps"])
@pytest.mark.parametrize("kw", [dict(sigma=2.0, bt=3), dict(sigma=2.0, bt=1, sharpen=0.4)], ids=["bt3", "bt1_sharpen"])
def test_format_matches_reference(gpu, fmt, kw):
    planes, ckw, _ = _clip(fmt)
    outs = []
    c = vshost.Core()
    c.load_plugin(PLUGIN)
    outs.append(c.invoke("neo_fft3d", "FFT3D", c.clip(planes, **ckw), **kw).render())
    r = reference.core()
    outs.append(r.invoke("neo_fft3d", "FFT3D", r.clip(planes, **ckw), opt=1, **kw).render())
    for i, (g, w) in enumerate(zip(*outs)):
        if g.dtype == np.float32:
            d = np.abs(g.astype(np.float64) - w)
            assert d.max() <= 2e-3 and (d <= 1 / 255).mean() >= 0.999, (fmt, i, d.max())
        else:
            d = np.abs(g.astype(np.int64) - w.astype(np.int64))
            assert (d <= 1).mean() >= 0.999 and d.max() <= 3, (fmt, i, d.max())
