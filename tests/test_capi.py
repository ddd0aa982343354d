"""The C ABI library: loads, exports every symbol include/fft3d_b200.h
declares, and validates parameters with the reference's messages -- all
without a GPU (validation happens before any CUDA call)."""
import ctypes
import os
import re

import pytest

from neo_fft3d_b200 import engine
from neo_fft3d_b200.params import FFT3DParams, PlaneDesc, make_params

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "fft3d_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fft3d_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_functions():
    names = declared_functions()
    assert "fft3d_plane_create" in names and "fft3d_filter2d_static" in names


@pytest.mark.parametrize("name", declared_functions())
def test_library_exports(name):
    assert hasattr(engine.lib(), name), name


def _create(**kw):
    p = make_params(**kw)
    d = PlaneDesc(64, 48, 8, 0, 0, 0, 10)
    h = ctypes.c_void_p()
    rc = engine.lib().fft3d_plane_create(ctypes.byref(p), ctypes.byref(d), 0, ctypes.byref(h))
    return rc, engine.lib().fft3d_last_error().decode()


@pytest.mark.parametrize("kw,msg", [
    (dict(bw=32, ow=20), "ow must be less than bw / 2"),
    (dict(bh=32, oh=17), "oh must be less than bh / 2"),
    (dict(bt=6), "bt must be -1 (Sharpen), 0 (Kalman), 1..5 (Wiener)"),
    (dict(bt=-2), "bt must be -1 (Sharpen), 0 (Kalman), 1..5 (Wiener)"),
    (dict(beta=0.5), "beta must be not less 1.0"),
    (dict(l=40, r=30), "Width cannot be cropped to zero or below"),
    (dict(t=30, b=30), "Height cannot be cropped to zero or below"),
])
def test_reference_parameter_errors(kw, msg):
    rc, err = _create(**kw)
    assert rc == -1 and err == msg


def test_unsupported_block_size():
    rc, err = _create(bw=40, bh=40)
    assert rc == -3 and "block size" in err


def test_defaults_match_reference():
    p = FFT3DParams()
    engine.lib().fft3d_params_default(ctypes.byref(p))
    q = make_params()
    for name, _ in FFT3DParams._fields_:
        assert getattr(p, name) == pytest.approx(getattr(q, name)), name


def test_batch_argument_checks_without_gpu():
    L = engine.lib()
    rc = L.fft3d_batch_step(None, 1, None, None, None, None, None, None, None)
    assert rc == -1 and "invalid batch step" in L.fft3d_last_error().decode()
    h = ctypes.c_void_p()
    rc = L.fft3d_batch_create(0, ctypes.byref(h))
    # no CUDA device in the CPU suite: refused before any work
    assert rc in (0, -6)
    if rc == 0:
        L.fft3d_batch_destroy(h)


def test_frame_group_and_timing_argument_checks_without_gpu():
    """Frame-group calls and the batch timing counters refuse bad arguments
    before any CUDA call."""
    L = engine.lib()
    p = (ctypes.c_void_p * 20)()
    s = (ctypes.c_int * 20)()
    d = (ctypes.c_void_p * 16)()
    ds = (ctypes.c_int * 16)()
    for fn in (lambda c: L.fft3d_plane_filter_frames_device(None, 0, c, p, s, d, ds, None),
               lambda c: L.fft3d_plane_filter_frames(None, 0, c, p, s, d, ds)):
        for count in (0, 4, 17):
            assert fn(count) == -1
            assert "frame group" in L.fft3d_last_error().decode()
    out = (ctypes.c_double * 12)()
    assert L.fft3d_batch_timing(None, out) == -1
    assert L.fft3d_batch_set_timing(None, 1) == -1
