"""The VapourSynth plugin shell (lib/libneo_fft3d_vs.so) as a drop-in for the
reference plugin: same namespace, function and argument string, same error
messages, and (GPU) the same frames through the headless VapourSynth host."""
import os

import numpy as np
import pytest

from neo_fft3d_b200 import synth, vshost
from oracle import reference

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PLUGIN = os.path.join(ROOT, "neo_fft3d_b200", "lib", "libneo_fft3d_vs.so")

needs_ref = pytest.mark.skipif(not reference.available(), reason="reference plugin not built")


def ours():
    c = vshost.Core()
    ns = c.load_plugin(PLUGIN)
    assert ns == "neo_fft3d"
    return c


@needs_ref
def test_same_registration_as_reference():
    assert ours().function_args("neo_fft3d", "FFT3D") == reference.core().function_args("neo_fft3d", "FFT3D")


@needs_ref
@pytest.mark.parametrize("kw", [dict(bw=32, ow=20), dict(bt=7), dict(beta=0.5), dict(l=100, r=100)])
def test_same_creation_errors(kw):
    planes = synth.make_clip(128, 96, 3, seed=3)
    msgs = []
    for core in (ours(), reference.core()):
        with pytest.raises(RuntimeError) as e:
            core.invoke("neo_fft3d", "FFT3D", core.clip(planes), **kw)
        msgs.append(str(e.value))
    assert msgs[0] == msgs[1]


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("kw", [dict(sigma=3.0, bt=5, sharpen=0.3), dict(sigma=2.0, bt=3, planes=[0, 2]),
                                dict(sigma=3.0, bt=0), dict(sigma=2.0, bt=3, l=8, t=4, r=8, b=6),
                                dict(sigma=2.0, bt=3, pfactor=1.0, pframe=1)],
                         ids=["wiener5", "planes02", "kalman", "crop", "pattern"])
def test_plugin_matches_reference(gpu, kw):
    planes = synth.make_clip(176, 144, 8, noise_sigma=5, seed=41)
    c = ours()
    got = c.invoke("neo_fft3d", "FFT3D", c.clip(planes), **kw).render(threads=1)
    want = reference.run(planes, opt=1, **kw)
    for g, w in zip(got, want):
        d = np.abs(g.astype(np.int64) - w.astype(np.int64))
        assert (d <= 1).mean() >= 0.999, (kw, d.max())


@pytest.mark.gpu
def test_plugin_parallel_render_matches_serial(gpu):
    planes = synth.make_clip(176, 144, 10, noise_sigma=5, seed=42)
    c = ours()
    a = c.invoke("neo_fft3d", "FFT3D", c.clip(planes), sigma=3.0, bt=5).render(threads=1)
    b = c.invoke("neo_fft3d", "FFT3D", c.clip(planes), sigma=3.0, bt=5).render(threads=4)
    for x, y in zip(a, b):
        assert np.abs(x.astype(int) - y.astype(int)).max() <= 1


@pytest.mark.gpu
def test_plugin_frame_groups_match_one_frame_per_call(gpu, monkeypatch):
    """With NEO_FFT3D_FRAME_GROUP set, the VapourSynth plugin filters Wiener
    3D clips in frame groups (each request computes its aligned group once,
    the group's other requests are served from the group): the same frames as
    one frame per call, rendered by parallel workers and in reverse order."""
    planes = synth.make_clip(176, 144, 21, noise_sigma=5, seed=47)
    outs = []
    for g, threads in (("1", 1), ("8", 4), ("3", 3), ("16", 1)):
        monkeypatch.setenv("NEO_FFT3D_FRAME_GROUP", g)
        c = ours()
        outs.append(c.invoke("neo_fft3d", "FFT3D", c.clip(planes), sigma=3.0, bt=5, sharpen=0.2).render(threads=threads))
    for o in outs[1:]:
        for a, b in zip(outs[0], o):
            assert np.array_equal(a, b)
    monkeypatch.setenv("NEO_FFT3D_FRAME_GROUP", "8")
    c = ours()
    node = c.invoke("neo_fft3d", "FFT3D", c.clip(planes), sigma=3.0, bt=5, sharpen=0.2)
    for n in reversed(range(21)):
        got = node.render(first=n, count=1)
        for a, b in zip(outs[0], got):
            assert np.array_equal(a[n], b[0])
