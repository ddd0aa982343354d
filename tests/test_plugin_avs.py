"""The AviSynth+ plugin shell (lib/libneo_fft3d_avs.so) as a drop-in for the
reference plugin's AviSynth+ entry, both loaded into the headless AviSynth+
host (csrc/avshost.cpp): the same function name and parameter string, the same
creation errors and MT mode, the same frames for copy-only plane modes (CPU),
and (GPU) the same filtered frames as the reference plugin and as this
package's VapourSynth shell."""
import os

import numpy as np
import pytest

from neo_fft3d_b200 import avshost, synth, vshost
from oracle import reference

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
VS_PLUGIN = os.path.join(ROOT, "neo_fft3d_b200", "lib", "libneo_fft3d_vs.so")

needs_host = pytest.mark.skipif(not avshost.available(), reason="AviSynth+ host or plugin not built")
needs_ref = pytest.mark.skipif(not (reference.available() and avshost.available()),
                               reason="reference plugin not built")


def ours():
    env = avshost.Env()
    env.load_plugin(avshost.PLUGIN_PATH)
    return env


def ref():
    env = avshost.Env()
    env.load_plugin(reference.REF_SO, preload=[reference.SHIM_SO])
    return env


def both():
    return [ours()] + ([ref()] if reference.available() else [])


@needs_host
def test_parameter_string_slots():
    params = ours().functions()["neo_fft3d"]
    slots = avshost.param_slots(params)
    assert slots[0] == (None, "c")
    names = [n for n, _ in slots[1:]]
    assert "planes" not in names and {"y", "u", "v"} <= set(names)
    kinds = dict(slots[1:])
    assert kinds["measure"] == kinds["interlaced"] == kinds["pshow"] == kinds["mt"] == "b"
    assert kinds["sigma"] == "f" and kinds["bt"] == "i"


@needs_ref
def test_same_registration_as_reference():
    assert ours().functions() == ref().functions()


@needs_ref
@pytest.mark.parametrize("kw", [dict(bw=32, ow=20), dict(bh=32, oh=17), dict(bt=7), dict(bt=-2), dict(beta=0.5),
                                dict(l=100, r=100), dict(t=48, b=48), dict(l=200, y=2, u=2, v=2)])
def test_same_creation_errors(kw):
    planes = synth.make_clip(128, 96, 3, seed=3)
    msgs = []
    for env in (ours(), ref()):
        with pytest.raises(avshost.AvisynthError) as e:
            env.invoke("neo_fft3d", env.clip(planes), **kw)
        msgs.append(str(e.value))
    assert msgs[0] == msgs[1]
    assert msgs[0].startswith("neo_fft3d: ")


@needs_host
def test_unknown_argument_is_refused():
    env = ours()
    with pytest.raises(avshost.AvisynthError, match="planes"):
        env.invoke("neo_fft3d", env.clip(synth.make_clip(64, 48, 2, seed=1)), planes=1)


@needs_host
@pytest.mark.parametrize("bt,mode", [(0, avshost.MT_SERIALIZED), (3, avshost.MT_NICE_FILTER),
                                     (-1, avshost.MT_NICE_FILTER)])
def test_copy_modes_and_mt_mode_without_gpu(bt, mode):
    """y = u = v = 2 filters no plane: no GPU work, the source frames come
    back, and the MT mode still follows bt."""
    planes = synth.make_clip(96, 64, 4, noise_sigma=4, seed=5)
    for env in both():
        out = env.invoke("neo_fft3d", env.clip(planes), sigma=3.0, bt=bt, y=2, u=2, v=2)
        assert out.mt_mode == mode
        got = out.render()
        for g, w in zip(got, planes):
            np.testing.assert_array_equal(g, w)


def _compare(got, want, tol_frac=0.999):
    for g, w in zip(got, want):
        d = np.abs(g.astype(np.int64) - w.astype(np.int64))
        assert (d <= 1).mean() >= tol_frac, d.max()


CASES = [
    ("wiener5", dict(sigma=3.0, bt=5, sharpen=0.3), {}),
    ("yuv_modes", dict(sigma=2.0, bt=3, u=2), {}),
    ("kalman", dict(sigma=3.0, bt=0), {}),
    ("crop", dict(sigma=2.0, bt=3, l=8, t=4, r=8, b=6), {}),
    ("pattern", dict(sigma=2.0, bt=3, pfactor=1.0, pframe=1), {}),
    ("wiener2d_dehalo", dict(sigma=2.5, bt=1, dehalo=0.4, measure=False), {}),
    ("yuv444_10bit", dict(sigma=8.0, bt=4, bw=48, bh=48, ow=16, oh=16), dict(bits=10, ssw=0, ssh=0)),
]


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("name,kw,clip", CASES, ids=[c[0] for c in CASES])
def test_plugin_matches_reference(gpu, name, kw, clip):
    bits = clip.get("bits", 8)
    planes = synth.make_clip(176, 144, 8, noise_sigma=5 * (4 if bits == 10 else 1), seed=43, bits=bits,
                             ssw=clip.get("ssw", 1), ssh=clip.get("ssh", 1))
    outs = []
    for env in (ours(), ref()):
        c = env.clip(planes, bits=bits)
        outs.append(env.invoke("neo_fft3d", c, **kw).render())
    _compare(outs[0], outs[1])
    if name == "yuv_modes":  # u = 2 copies the plane
        np.testing.assert_array_equal(outs[0][1], planes[1])


@pytest.mark.gpu
@needs_host
def test_avs_shell_matches_vs_shell(gpu):
    """The two shells drive the same planes of libfft3d_b200: identical frames."""
    planes = synth.make_clip(200, 136, 7, noise_sigma=5, seed=44)
    env = ours()
    a = env.invoke("neo_fft3d", env.clip(planes), sigma=3.0, bt=5, sharpen=0.2).render()
    core = vshost.Core()
    core.load_plugin(VS_PLUGIN)
    b = core.invoke("neo_fft3d", "FFT3D", core.clip(planes), sigma=3.0, bt=5, sharpen=0.2).render(threads=1)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


@pytest.mark.gpu
@needs_host
def test_random_access_matches_sequential(gpu):
    """Frames requested out of order (a seek, then backwards) give the frames
    of a sequential render: the cached spectra never stand in for other
    frames."""
    planes = synth.make_clip(160, 128, 12, noise_sigma=5, seed=45)
    env = ours()
    seq = env.invoke("neo_fft3d", env.clip(planes), sigma=3.0, bt=5).render()
    order = [7, 3, 4, 11, 0, 6, 5, 10, 1, 2, 9, 8]
    rnd = env.invoke("neo_fft3d", env.clip(planes), sigma=3.0, bt=5).render(order=order)
    for s, r in zip(seq, rnd):
        np.testing.assert_array_equal(s[order], r)
