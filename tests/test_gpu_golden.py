"""GPU path against the reference plugin's own outputs (golden fixtures) and
the known-answer tests, through the C ABI.

Bar: >= 99.9 % of output pixels within +-1 LSB of the reference.
"""
import numpy as np
import pytest

from neo_fft3d_b200 import engine, synth
from tests import golden_data

CASES = golden_data.load()
PIX_TOL_FRAC = 0.999


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_gpu_matches_reference_fixture(gpu, case):
    name, planes, bits, params, want = case
    got = engine.filter_clip(planes, bits=bits, **params)
    for i, (g, w) in enumerate(zip(got, want)):
        d = np.abs(g.astype(np.int64) - w.astype(np.int64))
        assert (d <= 1).mean() >= PIX_TOL_FRAC, (name, i, d.max(), (d <= 1).mean())
        assert d.max() <= 3, (name, i, d.max())


CLIP = synth.make_clip(128, 96, 6, noise_sigma=6, seed=31)


@pytest.mark.gpu
@pytest.mark.parametrize("bt", [1, 2, 3, 4, 5])
def test_gpu_sigma0_identity(gpu, bt):
    # (psd - 0) / psd = 1 and cos^2 + sin^2 = 1: output = input up to FFT rounding
    out = engine.filter_clip(CLIP, sigma=0.0, bt=bt)
    for o, i in zip(out, CLIP):
        d = np.abs(o.astype(int) - i.astype(int))
        assert d.max() <= 1 and (d == 0).mean() > 0.999


@pytest.mark.gpu
def test_gpu_kalman_sigma0_identity(gpu):
    out = engine.filter_clip(CLIP, sigma=0.0, bt=0)
    for o, i in zip(out, CLIP):
        assert np.abs(o.astype(int) - i.astype(int)).max() <= 1


@pytest.mark.gpu
def test_gpu_edge_frames_are_2d(gpu):
    out5 = engine.filter_clip(CLIP, sigma=3.0, bt=5)
    out1 = engine.filter_clip(CLIP, sigma=3.0, bt=1)
    for o5, o1 in zip(out5, out1):
        for n in (0, 1, CLIP[0].shape[0] - 2, CLIP[0].shape[0] - 1):
            assert np.abs(o5[n].astype(int) - o1[n].astype(int)).max() <= 1
