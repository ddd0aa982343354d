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


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(sigma=3.0, bt=5, sharpen=0.3), dict(sigma=2.0, bt=1, l=4, r=6)],
                         ids=["wiener5", "wiener2d_crop"])
def test_host_calls_from_threads(gpu, kw):
    """fft3d_plane_filter called for different frames from several threads at
    once (copies of one call overlap the kernels of another) gives the same
    bytes as calling it frame by frame."""
    import threading
    from neo_fft3d_b200.params import make_params, plane_descs
    planes = synth.make_clip(200, 144, 24, noise_sigma=5.0, seed=93)
    F = planes[0].shape[0]
    p = make_params(bw=32, bh=32, ow=16, oh=16, **kw)
    descs = plane_descs([a.shape[1:] for a in planes], 8, F)
    ref = engine.filter_clip(planes, bits=8, bw=32, bh=32, ow=16, oh=16, **kw)
    for a, d, r in zip(planes, descs, ref):
        e = engine.PlaneEngine(p, d)
        out = np.zeros_like(a)
        counter, lock, errors = [0], threading.Lock(), []

        def work():
            while True:
                with lock:
                    n = counter[0]
                    counter[0] += 1
                if n >= F:
                    return
                try:
                    e.filter(n, [a[n + k] if 0 <= n + k < F else None for k in range(-2, 3)], out[n])
                except Exception as ex:  # reported below
                    errors.append(ex)

        th = [threading.Thread(target=work) for _ in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        e.close()
        assert not errors
        assert np.array_equal(out, r)
