"""Failure paths of the C ABI, with every failure made on the host.

* FFT3D_E_FRAME: a frame the call needs and the device does not hold is not
  supplied (one-frame host and device calls, host frame groups, Kalman frame
  0, crop borders without the current frame);
* FFT3D_E_NOMEM: the plane's device allocations are capped
  (NEO_FFT3D_DEVICE_ALLOC_CAP) at creation and at frame-group growth;
* FFT3D_E_CUDA from the device error flag: the flag a kernel sets when a
  bounded wait runs out is raised by a test hook instead of a real timeout,
  and must be reported by the next host-buffer call (one frame and frame
  group) or by fft3d_plane_synchronize, then cleared.

After each failure the plane must still filter correctly.
"""
import ctypes

import numpy as np
import pytest

from neo_fft3d_b200 import engine, synth
from neo_fft3d_b200.engine import FFT3DError
from neo_fft3d_b200.params import make_params, plane_descs


def _luma(F=8, w=160, h=128, seed=31):
    return synth.make_clip(w, h, F, noise_sigma=5, seed=seed, planes=1)[0]


def _win(a, n):
    return [a[n + d] if 0 <= n + d < a.shape[0] else None for d in range(-2, 3)]


def _engine(a, **kw):
    p = make_params(**kw)
    d = plane_descs([a.shape[1:]], 8, a.shape[0])[0]
    return engine.PlaneEngine(p, d)


def _expect(rc_fn, status, text):
    with pytest.raises(FFT3DError) as ei:
        rc_fn()
    msg = str(ei.value)
    assert f"(status {status})" in msg and text in msg, msg


@pytest.mark.gpu
def test_missing_window_frame_host(gpu):
    a = _luma()
    e = _engine(a, sigma=2.0, bt=3)
    out = np.empty_like(a[0])
    w = _win(a, 4)
    w[1] = None  # frame 3 is needed (bt=3 window 3..5) and not cached
    _expect(lambda: e.filter(4, w, out), -5, "frame 3 is needed but was not supplied")
    ref = _engine(a, sigma=2.0, bt=3)
    want = np.empty_like(out)
    ref.filter(4, _win(a, 4), want)
    e.filter(4, _win(a, 4), out)  # still usable
    assert np.array_equal(out, want)


@pytest.mark.gpu
def test_missing_window_frame_device(gpu):
    import torch
    a = _luma()
    e = _engine(a, sigma=2.0, bt=5)
    dev = torch.from_numpy(a).cuda()
    out = torch.empty_like(dev[0])
    fb = a.shape[1] * a.shape[2]
    W = a.shape[2]
    ptrs = [dev.data_ptr() + (4 + d) * fb for d in range(-2, 3)]
    ptrs[4] = 0  # frame 6
    _expect(lambda: e.filter_device(4, ptrs, [W] * 5, out.data_ptr(), W), -5, "frame 6 is needed")


@pytest.mark.gpu
def test_missing_frame_in_host_group(gpu):
    a = _luma(F=12)
    e = _engine(a, sigma=2.0, bt=3)
    outs = [np.empty_like(a[0]) for _ in range(4)]
    srcs = [a[m] if 0 <= m < a.shape[0] else None for m in range(2, 10)]  # frames 2..9 for outputs 4..7
    srcs[5] = None  # frame 7
    _expect(lambda: e.filter_frames(4, srcs, outs), -5, "frame 7 is needed but was not supplied")
    srcs[5] = a[7]
    e.filter_frames(4, srcs, outs)
    ref = _engine(a, sigma=2.0, bt=3)
    for j in range(4):
        want = np.empty_like(a[0])
        ref.filter(4 + j, _win(a, 4 + j), want)
        assert np.array_equal(outs[j], want)


@pytest.mark.gpu
def test_missing_kalman_frame0_and_crop_frame(gpu):
    a = _luma()
    e = _engine(a, sigma=2.0, bt=0)
    out = np.empty_like(a[0])
    _expect(lambda: e.filter(0, [None] * 5, out), -5, "frame 0 was not supplied")
    e.filter(0, _win(a, 0), out)
    assert np.array_equal(out, a[0])  # Kalman frame 0 passes through
    c = _engine(a, sigma=2.0, bt=1, l=8, r=4, t=2, b=6)
    c.filter(3, _win(a, 3), out)  # frame 3's spectrum is now cached
    w = [None] * 5
    _expect(lambda: c.filter(3, w, out), -5, "current frame is needed for the crop borders")


@pytest.mark.gpu
def test_device_alloc_cap_at_creation(gpu, monkeypatch):
    a = _luma()
    monkeypatch.setenv("NEO_FFT3D_DEVICE_ALLOC_CAP", str(64 << 10))
    with pytest.raises(FFT3DError) as ei:
        _engine(a, sigma=2.0, bt=3)
    assert "(status -4)" in str(ei.value) and "out of device memory" in str(ei.value)


@pytest.mark.gpu
def test_device_alloc_cap_at_group_growth(gpu, monkeypatch):
    import torch
    a = _luma(F=12)
    probe = _engine(a, sigma=2.0, bt=3)
    base = probe.device_bytes()
    probe.close()
    assert base > 0
    monkeypatch.setenv("NEO_FFT3D_DEVICE_ALLOC_CAP", str(base + 1024))
    e = _engine(a, sigma=2.0, bt=3)
    assert e.device_bytes() == base
    dev = torch.from_numpy(a).cuda()
    outs = torch.empty_like(dev[:8])
    fb = a.shape[1] * a.shape[2]
    W = a.shape[2]
    ptrs = [dev.data_ptr() + m * fb if 0 <= m < 12 else 0 for m in range(-2, 10)]
    dsts = [outs.data_ptr() + j * fb for j in range(8)]
    _expect(lambda: e.filter_frames_device(0, ptrs, [W] * 12, dsts, [W] * 8), -4, "spectrum ring of a frame group")
    # one frame per call still fits the plane's own resources
    out = np.empty_like(a[0])
    e.filter(5, _win(a, 5), out)
    ref = _engine(a, sigma=2.0, bt=3)
    want = np.empty_like(out)
    ref.filter(5, _win(a, 5), want)
    assert np.array_equal(out, want)


@pytest.mark.gpu
@pytest.mark.parametrize("bits,text", [(1, "tensor-core MMA completion wait timed out"),
                                       (2, "bulk copy completion wait timed out")])
def test_device_error_flag_host_call(gpu, bits, text):
    a = _luma()
    e = _engine(a, sigma=2.0, bt=3)
    out = np.empty_like(a[0])
    e.filter(3, _win(a, 3), out)
    engine.lib().fft3d_plane_debug_set_error_flag(e.h, bits)
    _expect(lambda: e.filter(4, _win(a, 4), out), -2, text)
    e.filter(5, _win(a, 5), out)  # the flag was cleared: the next call succeeds
    ref = _engine(a, sigma=2.0, bt=3)
    want = np.empty_like(out)
    ref.filter(5, _win(a, 5), want)
    assert np.array_equal(out, want)


@pytest.mark.gpu
def test_device_error_flag_host_group(gpu):
    a = _luma(F=12)
    e = _engine(a, sigma=2.0, bt=3)
    outs = [np.empty_like(a[0]) for _ in range(4)]
    srcs = [a[m] if 0 <= m < 12 else None for m in range(-2, 6)]
    engine.lib().fft3d_plane_debug_set_error_flag(e.h, 1)
    _expect(lambda: e.filter_frames(0, srcs, outs), -2, "timed out")
    srcs = [a[m] if 0 <= m < 12 else None for m in range(2, 10)]
    e.filter_frames(4, srcs, outs)


@pytest.mark.gpu
def test_device_error_flag_synchronize(gpu):
    import torch
    a = _luma()
    e = _engine(a, sigma=2.0, bt=1)
    dev = torch.from_numpy(a).cuda()
    out = torch.empty_like(dev[0])
    W = a.shape[2]
    e.filter_device(2, [0, 0, dev[2].data_ptr(), 0, 0], [W] * 5, out.data_ptr(), W)
    e.synchronize()
    engine.lib().fft3d_plane_debug_set_error_flag(e.h, 2)
    e.filter_device(3, [0, 0, dev[3].data_ptr(), 0, 0], [W] * 5, out.data_ptr(), W)
    _expect(e.synchronize, -2, "bulk copy completion wait timed out")
    e.synchronize()  # cleared


def test_failure_hooks_refuse_null_handles():
    L = engine.lib()
    out = ctypes.c_uint64()
    assert L.fft3d_plane_device_bytes(None, ctypes.byref(out)) == -1
    assert L.fft3d_plane_synchronize(None) == -1
    assert L.fft3d_plane_debug_set_error_flag(None, 1) == -1
    assert "null" in L.fft3d_last_error().decode()
