"""The engine's alternative kernel sequences (NEO_FFT3D_PATH = split | fused,
NEO_FFT3D_INV = bulk) against the default unfused path, which the parity and
golden tests pin to the oracle and the reference: every output pixel within
+-1 LSB and >= 99.9 % identical, for every filter mode."""
import os

import numpy as np
import pytest

from neo_fft3d_b200 import engine, synth

MODES = [dict(sigma=3.0, bt=5, sharpen=0.3), dict(sigma=2.0, bt=3, dehalo=0.5), dict(sigma=2.5, bt=2),
         dict(sigma=3.0, bt=4, degrid=0.0), dict(sigma=3.0, bt=0, kratio=2.0), dict(sigma=2.0, bt=1, l=6, t=4, r=2, b=8),
         dict(bt=-1, sharpen=0.5)]
VARIANTS = [("split", {"NEO_FFT3D_PATH": "split"}), ("fused", {"NEO_FFT3D_PATH": "fused"}),
            ("bulk", {"NEO_FFT3D_INV": "bulk"})]


def _run(monkeypatch, env, planes, bits, kw):
    for k in ("NEO_FFT3D_PATH", "NEO_FFT3D_INV"):
        monkeypatch.delenv(k, raising=False)
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    return engine.filter_clip(planes, bits=bits, **kw)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", VARIANTS, ids=[v[0] for v in VARIANTS])
@pytest.mark.parametrize("mode", MODES, ids=[str(i) for i in range(len(MODES))])
@pytest.mark.parametrize("bw", [32, 48])
def test_path_matches_default(gpu, monkeypatch, variant, mode, bw):
    planes = synth.make_clip(208, 152, 9, noise_sigma=5.0, seed=91)
    kw = dict(mode, bw=bw, bh=bw, ow=16, oh=16)
    ref = _run(monkeypatch, {}, planes, 8, kw)
    got = _run(monkeypatch, variant[1], planes, 8, kw)
    for r, g in zip(ref, got):
        d = np.abs(r.astype(int) - g.astype(int))
        assert d.max() <= 1
        assert np.mean(d == 0) >= 0.999


@pytest.mark.gpu
@pytest.mark.parametrize("variant", VARIANTS[1:], ids=[v[0] for v in VARIANTS[1:]])
def test_path_matches_default_10bit(gpu, monkeypatch, variant):
    planes = synth.make_clip(176, 128, 7, bits=10, noise_sigma=16.0, seed=92)
    kw = dict(sigma=3.0, bt=5, bw=32, bh=32, ow=16, oh=16, sharpen=0.2)
    ref = _run(monkeypatch, {}, planes, 10, kw)
    got = _run(monkeypatch, variant[1], planes, 10, kw)
    for r, g in zip(ref, got):
        d = np.abs(r.astype(int) - g.astype(int))
        assert d.max() <= 1 and np.mean(d == 0) >= 0.999
