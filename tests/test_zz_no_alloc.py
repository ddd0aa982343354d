"""The allocation-free entry point fft3d_filter2d_static, through the C ABI.

It serves callers that cannot allocate device memory while frames flow (their
device memory belongs to their own pool allocator, or they must not pay the
implicit synchronisation of cudaMalloc/cudaFree): its scratch is a fixed
32 MiB device array inside the library. This test checks that two calls in a
row, on different frames, give exactly the output of the regular entry point
(fft3d_plane_filter_device) with the same parameters -- byte for byte, since
both run the same kernels on the same tables -- for 8-, 10- and 16-bit and
float samples and with crop borders, and that an oversized plane is refused.

Collected last (file name) so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from neo_fft3d_b200 import engine, synth
from neo_fft3d_b200.params import FFT3DParams, PlaneDesc, make_params, plane_descs


def _static_fn():
    L = engine.lib()
    f = L.fft3d_filter2d_static
    f.argtypes = [ctypes.POINTER(FFT3DParams), ctypes.POINTER(PlaneDesc), ctypes.c_void_p, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _clip(bits):
    if bits == 32:
        planes = synth.make_clip(320, 240, 2, noise_sigma=5, seed=23)
        return [(a.astype(np.float32) / 255.0) for a in planes]
    return synth.make_clip(320, 240, 2, bits=bits, noise_sigma=5 * (1 << (bits - 8)), seed=21 + bits)


CASES = [
    ("wiener2d_8bit", 8, dict(sigma=3.0, bt=1, sharpen=0.4, dehalo=0.5)),
    ("sharpen_only_8bit", 8, dict(sigma=2.0, bt=-1, sharpen=0.7, bw=16, bh=16, ow=4, oh=4)),
    ("wiener2d_10bit", 10, dict(sigma=3.0, bt=1, sharpen=0.3, bw=48, bh=48, ow=16, oh=16)),
    ("wiener2d_16bit_crop", 16, dict(sigma=2.5, bt=1, dehalo=0.4, l=6, t=4, r=10, b=2)),
    ("wiener2d_float", 32, dict(sigma=3.0, bt=1, sharpen=0.2, bw=24, bh=24, ow=8, oh=8)),
    ("sharpen_only_8bit_crop", 8, dict(sigma=2.0, bt=-1, sharpen=0.5, l=8, t=2, r=4, b=6)),
]


@pytest.mark.gpu
@pytest.mark.parametrize("bits,kw", [(c[1], c[2]) for c in CASES], ids=[c[0] for c in CASES])
def test_static_matches_regular_two_calls(gpu, bits, kw):
    import torch

    fn = _static_fn()
    planes = _clip(bits)
    p = make_params(**kw)
    descs = plane_descs([a.shape[1:] for a in planes], bits, 2)
    stream = torch.cuda.current_stream()
    for i, a in enumerate(planes):
        reg = engine.PlaneEngine(p, descs[i])
        for n in range(2):  # two calls in a row, different frames
            host = np.ascontiguousarray(a[n])
            src = torch.from_numpy(host.view(np.int16) if host.dtype == np.uint16 else host).cuda()
            want = torch.empty_like(src)
            got = torch.full_like(src, 7)
            pitch = host.strides[0]
            reg.filter_device(n, [0, 0, src.data_ptr(), 0, 0], [pitch] * 5, want.data_ptr(), pitch,
                              stream.cuda_stream)
            rc = fn(ctypes.byref(p), ctypes.byref(descs[i]), src.data_ptr(), pitch, got.data_ptr(), pitch,
                    ctypes.c_void_p(stream.cuda_stream))
            assert rc == 0, engine.lib().fft3d_last_error().decode()
            torch.cuda.synchronize()
            g, w = got.cpu().numpy(), want.cpu().numpy()
            assert np.array_equal(g.view(np.uint8), w.view(np.uint8)), (kw, i, n)
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
