"""Known-answer tests derived from the reference's mathematics, on the oracle.

(a) sigma=0, sharpen=0, dehalo=0: every Wiener factor is (psd-0)/psd = 1 and
    the wintype-0 windows satisfy cos^2 + sin^2 = 1, so output == input
    exactly for 8/16-bit, for every bt >= 1 (src/code_impl/Apply.cpp:30-31,
    src/fft3d_engine.h:212-233).
(b) A constant plane with degrid=1: the grid correction equals the spectrum,
    so the filtered part is 0 and the output equals the input.
(c) Kalman with sigma=0: every bin is "motion", output == input.
(d) bt>1 edge frames equal a bt=1 run on those frames (src/fft3d_engine.h:579-582).
"""
import numpy as np
import pytest

from neo_fft3d_b200 import synth
from oracle import restate

CLIP = synth.make_clip(128, 96, 6, noise_sigma=6, seed=31)


@pytest.mark.parametrize("bt", [1, 2, 3, 4, 5])
def test_sigma0_identity(bt):
    out = restate.filter_clip(CLIP, sigma=0.0, bt=bt)
    for o, i in zip(out, CLIP):
        assert np.array_equal(o, i)


def test_constant_plane_identity():
    planes = [np.full_like(p, 100 + 20 * k) for k, p in enumerate(CLIP)]
    out = restate.filter_clip(planes, sigma=3.0, bt=3, degrid=1.0)
    for o, i in zip(out, planes):
        assert np.abs(o.astype(int) - i.astype(int)).max() <= 1


def test_kalman_sigma0_identity():
    out = restate.filter_clip(CLIP, sigma=0.0, bt=0)
    for o, i in zip(out, CLIP):
        assert np.array_equal(o, i)


def test_edge_frames_are_2d():
    out5 = restate.filter_clip(CLIP, sigma=3.0, bt=5)
    out1 = restate.filter_clip(CLIP, sigma=3.0, bt=1)
    for o5, o1 in zip(out5, out1):
        for n in (0, 1, CLIP[0].shape[0] - 2, CLIP[0].shape[0] - 1):
            assert np.array_equal(o5[n], o1[n])
        assert not np.array_equal(o5[2], o1[2])
