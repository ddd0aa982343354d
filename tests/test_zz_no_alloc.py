"""The allocation-free entry point fft3d_filter2d_static, through the C ABI.

It serves callers that cannot allocate device memory while frames flow (their
device memory belongs to their own pool allocator, or they must not pay the
implicit synchronisation of cudaMalloc/cudaFree): its scratch is a fixed
32 MiB device array inside the library. This test checks that two calls in a
row, on different frames, give the output of the regular entry point
(fft3d_plane_filter_device) with the same parameters, within the +-1 LSB bar
the other GPU tests use, and that an oversized plane is refused.

Collected last (file name) so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from neo_fft3d_b200 import engine, synth
from neo_fft3d_b200.params import FFT3DParams, PlaneDesc, make_params, plane_descs

PIX_TOL_FRAC = 0.999


def _static_fn():
    L = engine.lib()
    f = L.fft3d_filter2d_static
    f.argtypes = [ctypes.POINTER(FFT3DParams), ctypes.POINTER(PlaneDesc), ctypes.c_void_p, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(sigma=3.0, bt=1, sharpen=0.4, dehalo=0.5),
                                dict(sigma=2.0, bt=-1, sharpen=0.7, bw=16, bh=16, ow=4, oh=4)],
                         ids=["wiener2d", "sharpen_only"])
def test_static_matches_regular_two_calls(gpu, kw):
    import torch

    fn = _static_fn()
    planes = synth.make_clip(320, 240, 2, noise_sigma=5, seed=21)
    p = make_params(**kw)
    descs = plane_descs([a.shape[1:] for a in planes], 8, 2)
    stream = torch.cuda.current_stream()
    for i, a in enumerate(planes):
        reg = engine.PlaneEngine(p, descs[i])
        for n in range(2):  # two calls in a row, different frames
            src = torch.from_numpy(np.ascontiguousarray(a[n])).cuda()
            want = torch.empty_like(src)
            got = torch.full_like(src, 7)
            W = src.shape[1]
            reg.filter_device(n, [0, 0, src.data_ptr(), 0, 0], [W] * 5, want.data_ptr(), W, stream.cuda_stream)
            rc = fn(ctypes.byref(p), ctypes.byref(descs[i]), src.data_ptr(), W, got.data_ptr(), W,
                    ctypes.c_void_p(stream.cuda_stream))
            assert rc == 0, engine.lib().fft3d_last_error().decode()
            torch.cuda.synchronize()
            d = (got.cpu().numpy().astype(np.int64) - want.cpu().numpy().astype(np.int64))
            assert (np.abs(d) <= 1).mean() >= PIX_TOL_FRAC, (kw, i, n, np.abs(d).max())
        reg.close()


@pytest.mark.gpu
def test_static_rejects_oversized_plane(gpu):
    import torch

    fn = _static_fn()
    p = make_params(sigma=3.0, bt=1, bw=32, bh=32, ow=16, oh=16)
    d = PlaneDesc(1920, 1080, 8, 0, 0, 0, 1)  # 1080p luma: ~70 MB of scratch, above the 32 MiB array
    src = torch.zeros((1080, 1920), dtype=torch.uint8, device="cuda")
    dst = torch.zeros_like(src)
    rc = fn(ctypes.byref(p), ctypes.byref(d), src.data_ptr(), 1920, dst.data_ptr(), 1920, None)
    assert rc == -3
    assert "scratch" in engine.lib().fft3d_last_error().decode()
