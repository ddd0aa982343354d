"""pshow (src/fft3d_engine.h:505-565): with pfactor != 0 each output frame is
the noise pattern's block alone on a flat background, the block found on that
frame (or fixed by px, py), with the reference's switch to constant windows
after the first frame. Checked against the reference plugin itself (built
from its sources, run through the headless VapourSynth host, one thread so
that the frames come in order)."""
import numpy as np
import pytest

from neo_fft3d_b200 import engine, synth
from oracle import reference

needs_ref = pytest.mark.skipif(not reference.available(), reason="reference plugin not built")

CASES = [("found", dict(sigma=2.0, bt=3, pfactor=1.0, pshow=1)),
         ("fixed_block", dict(sigma=2.0, bt=3, pfactor=1.0, pshow=1, px=5, py=4)),
         ("bw16_degrid0", dict(sigma=2.0, bt=1, pfactor=0.5, pshow=1, bw=16, bh=16, ow=4, oh=4, degrid=0.0))]


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_pshow_matches_reference(gpu, name, kw):
    planes = synth.make_clip(192, 160, 5, noise_sigma=6, seed=97)
    got = engine.filter_clip(planes, **kw)
    want = reference.run(planes, threads=1, opt=1, **kw)
    for i, (g, w) in enumerate(zip(got, want)):
        d = np.abs(g.astype(np.int64) - w.astype(np.int64))
        assert (d <= 1).mean() >= 0.999 and d.max() <= 1, (name, i, d.max())
        # the background outside the block is flat: 2^(bits-1) for every plane of a YUV clip
        assert (g == 128).mean() > 0.5, (name, i)


@pytest.mark.gpu
def test_pshow_without_pfactor_filters_normally(gpu):
    """pshow needs pfactor != 0 (src/fft3d_engine.h:505); otherwise the frame is filtered."""
    planes = synth.make_clip(128, 96, 4, noise_sigma=5, seed=98)
    a = engine.filter_clip(planes, sigma=2.0, bt=3, pshow=1)
    b = engine.filter_clip(planes, sigma=2.0, bt=3)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
