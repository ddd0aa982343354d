"""Host-side pieces: the headless VapourSynth host, the synthetic clip
generator and the FFTW-API shim the reference runs on."""
import ctypes
import os

import numpy as np
import pytest

from neo_fft3d_b200 import synth
from oracle import reference

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_synth_is_deterministic():
    a = synth.make_clip(64, 48, 3, seed=5)
    b = synth.make_clip(64, 48, 3, seed=5)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert a[0].shape == (3, 48, 64) and a[1].shape == (3, 24, 32)
    assert a[0].min() >= 0 and a[0].dtype == np.uint8


def test_pack_roundtrip():
    a = synth.make_clip(64, 48, 2, bits=10, seed=6)
    b = synth.unpack(synth.pack(a), a)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


@pytest.mark.skipif(not reference.available(), reason="reference plugin not built")
def test_reference_registers_fft3d():
    c = reference.core()
    args = c.function_args("neo_fft3d", "FFT3D")
    assert args.startswith("clip:clip;sigma:float:opt;beta:float:opt;planes:int[]:opt;bw:int:opt;")
    assert "ncpu:int:opt;mt:int:opt;" in args


@pytest.mark.skipif(not reference.available(), reason="reference plugin not built")
@pytest.mark.parametrize("bh,bw", [(32, 32), (48, 48), (16, 32), (20, 20)])
def test_fftw_shim_matches_numpy(bh, bw):
    L = ctypes.CDLL(reference.SHIM_SO)
    L.fftwf_plan_many_dft_r2c.restype = ctypes.c_void_p
    L.fftwf_plan_many_dft_c2r.restype = ctypes.c_void_p
    nb, nh = 3, bw // 2 + 1
    op = (nh + 15) // 16 * 16
    x = np.random.RandomState(0).randn(nb, bh, bw).astype(np.float32)
    out = np.zeros((nb, bh, op, 2), np.float32)
    n = (ctypes.c_int * 2)(bh, bw)
    ie = (ctypes.c_int * 2)(bh, bw)
    oe = (ctypes.c_int * 2)(bh, op)
    p = L.fftwf_plan_many_dft_r2c(2, n, nb, None, ie, 1, bh * bw, None, oe, 1, op * bh, 0)
    L.fftwf_execute_dft_r2c(ctypes.c_void_p(p), x.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p))
    ref = np.fft.rfft2(x.astype(np.float64))
    got = out[:, :, :nh, 0] + 1j * out[:, :, :nh, 1]
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-6
    back = np.zeros_like(x)
    q = L.fftwf_plan_many_dft_c2r(2, n, nb, None, oe, 1, op * bh, None, ie, 1, bh * bw, 0)
    L.fftwf_execute_dft_c2r(ctypes.c_void_p(q), out.ctypes.data_as(ctypes.c_void_p), back.ctypes.data_as(ctypes.c_void_p))
    assert np.abs(back / (bh * bw) - x).max() < 1e-5
    L.fftwf_destroy_plan(ctypes.c_void_p(p))
    L.fftwf_destroy_plan(ctypes.c_void_p(q))


@pytest.mark.skipif(not reference.available(), reason="reference plugin not built")
def test_reference_reproduces_golden():
    from tests import golden_data
    for name, planes, bits, params, want in golden_data.load()[:3]:
        got = reference.run(planes, opt=1, bits=bits, **params)
        for g, w in zip(got, want):
            assert np.array_equal(g, w), name
