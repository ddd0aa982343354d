"""The overlap-add fused into a frame group's filter/inverse launch
(NEO_FFT3D_FUSED_OLA=1; the default is a separate overlap-add launch): the
CTA that completes the last block an output tile reads does that tile's
overlap-add for the run's frames. Its output must equal the separate
overlap-add launch byte for byte, for both
pixel forms (4-pixel and single-pixel), every sample type, interlacing,
crop, rectangular blocks and every filter mode; and one frame per call
(always unfused) must give the same bytes too. Outputs start filled with a
value no filtered sample takes, so that a pixel left unwritten shows."""
import numpy as np
import pytest

from neo_fft3d_b200 import engine, synth
from neo_fft3d_b200.params import make_params, plane_descs

F = 19

CASES = [
    # 4-pixel form: block step, overlap and width multiples of 4
    ("u8_bt5_ow16", dict(width=224, height=128, bits=8, seed=91), dict(sigma=3.0, bt=5, ow=16, oh=16, sharpen=0.3)),
    # single-pixel form: overlap 10 (bw / 3)
    ("u8_bt5_default", dict(width=200, height=136, bits=8, seed=92), dict(sigma=3.0, bt=5)),
    ("u8_bt3_bw48", dict(width=152, height=96, bits=8, seed=103), dict(sigma=2.0, bt=3, bw=48, bh=48, ow=16, oh=16)),
    ("u16_bt3_bw16", dict(width=160, height=96, bits=16, seed=93), dict(sigma=200.0, bt=3, bw=16, bh=16, ow=8, oh=8)),
    ("u10_bt4_bw48", dict(width=176, height=144, bits=10, seed=94), dict(sigma=8.0, bt=4, bw=48, bh=48, ow=16, oh=16)),
    ("float_bt3", dict(width=160, height=96, bits=32, seed=95), dict(sigma=2.0, bt=3, bw=24, bh=24, ow=8, oh=8)),
    ("interlaced_bt3", dict(width=160, height=128, bits=8, seed=96), dict(sigma=2.0, bt=3, interlaced=1)),
    ("rect_16x24", dict(width=152, height=104, bits=8, seed=97), dict(sigma=2.0, bt=2, bw=16, bh=24, ow=4, oh=6)),
    ("crop_odd_width", dict(width=160, height=128, bits=8, seed=98), dict(sigma=2.0, bt=3, l=6, t=4, r=7, b=2)),
    ("kalman", dict(width=128, height=96, bits=8, seed=99), dict(sigma=3.0, bt=0)),
    ("wiener2d", dict(width=128, height=96, bits=8, seed=100), dict(sigma=3.0, bt=1, sharpen=0.2, dehalo=0.5)),
    ("sharpen_only", dict(width=128, height=96, bits=8, seed=101), dict(sigma=3.0, bt=-1, sharpen=0.4)),
]


def _planes(clip):
    bits = clip["bits"]
    if bits == 32:
        kw = dict(clip, bits=8)
        return [a.astype(np.float32) / 255.0 for a in synth.make_clip(frames=F, noise_sigma=5.0, **kw)]
    return synth.make_clip(frames=F, noise_sigma=5.0 * (1 << (bits - 8)), **clip)


def _to_dev(torch, a):
    if a.dtype == np.uint16:
        a = a.view(np.int16)
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _sentinel(torch, a):
    """An output buffer filled with a value no filtered sample takes."""
    return torch.full_like(a, -1.0 if a.dtype == torch.float32 else 1)


def _ptr(a, n):
    fb = a.shape[1] * a.shape[2] * a.element_size()
    return a.data_ptr() + n * fb if 0 <= n < a.shape[0] else 0


def _run(torch, planes, clip, filt, sizes):
    """Every plane in frame groups of the given sizes (cycled), device buffers;
    sizes None: one frame per call."""
    p = make_params(**filt)
    descs = plane_descs([a.shape[1:] for a in planes], clip["bits"], F)
    outs = []
    for a_np, d in zip(planes, descs):
        e = engine.PlaneEngine(p, d)
        a = _to_dev(torch, a_np)
        o = _sentinel(torch, a)
        st = a.shape[2] * a.element_size()
        if sizes is None:
            for n in range(F):
                e.filter_device(n, [_ptr(a, n + k) for k in range(-2, 3)], [st] * 5, _ptr(o, n), st, 0)
        else:
            n0, i = 0, 0
            while n0 < F:
                k = min(sizes[i % len(sizes)], F - n0)
                e.filter_frames_device(n0, [_ptr(a, n) for n in range(n0 - 2, n0 + k + 2)], [st] * (k + 4),
                                       [_ptr(o, n) for n in range(n0, n0 + k)], [st] * k, 0)
                n0 += k
                i += 1
        torch.cuda.synchronize()
        outs.append(o.cpu().numpy())
        e.close()
    return outs


@pytest.mark.gpu
@pytest.mark.parametrize("name,clip,filt", CASES, ids=[c[0] for c in CASES])
def test_fused_overlap_add_matches_separate(gpu, monkeypatch, name, clip, filt):
    import torch
    planes = _planes(clip)
    ref = _run(torch, planes, clip, filt, None)
    for sizes in ([8], [5, 3, 16], [4]):
        monkeypatch.delenv("NEO_FFT3D_FUSED_OLA", raising=False)
        sep = _run(torch, planes, clip, filt, sizes)
        monkeypatch.setenv("NEO_FFT3D_FUSED_OLA", "1")
        fused = _run(torch, planes, clip, filt, sizes)
        for i, (r, s, f) in enumerate(zip(ref, sep, fused)):
            assert np.array_equal(r, s), (name, sizes, i, "separate vs one frame per call")
            bad = np.argwhere(r != f)
            assert len(bad) == 0, (name, sizes, i, "fused vs one frame per call", len(bad), bad[:4].tolist())


@pytest.mark.gpu
def test_fused_overlap_add_launches_and_bytes(gpu, monkeypatch):
    """A fused frame group launches no overlap-add kernel; its filter/inverse
    launch counts the window spectra once and the output pixels (the
    time-domain blocks pass between CTAs of the launch); the separate form
    counts the time-domain blocks and launches the overlap-add."""
    import torch
    clip, filt = CASES[0][1], CASES[0][2]
    a_np = _planes(clip)[0]
    a = _to_dev(torch, a_np)
    H, W = a_np.shape[1:]
    desc = plane_descs([a_np.shape[1:]], 8, F)[0]
    for fused in (True, False):
        if fused:
            monkeypatch.setenv("NEO_FFT3D_FUSED_OLA", "1")
        else:
            monkeypatch.delenv("NEO_FFT3D_FUSED_OLA", raising=False)
        e = engine.PlaneEngine(make_params(**filt), desc)
        o = _sentinel(torch, a)
        e.filter_frames_device(2, [_ptr(a, n) for n in range(0, 10)], [W] * 10, [_ptr(o, n) for n in range(2, 8)],
                               [W] * 6, 0)
        e.timing()
        e.set_timing(True)
        e.filter_frames_device(8, [_ptr(a, n) for n in range(6, 16)], [W] * 10, [_ptr(o, n) for n in range(8, 14)],
                               [W] * 6, 0)
        torch.cuda.synchronize()
        t = e.timing()
        e.set_timing(False)
        S = e.nblocks * 32 * 17 * 8
        T = e.nblocks * 32 * 32 * 4
        assert t["filter_inverse"][0] == 1
        if fused:
            assert t["filter_inverse"][2] == pytest.approx(10 * S + 6 * W * H)
            assert t["overlap_add"][0] == 0
        else:
            assert t["filter_inverse"][2] == pytest.approx(10 * S + 6 * T)
            assert t["overlap_add"][0] == 1
        e.close()


@pytest.mark.gpu
def test_fused_overlap_add_many_calls(gpu, monkeypatch):
    """The arrival counters carry over from call to call (each launch counts
    in its own epoch): many short groups and a reset in between keep the
    output equal to one frame per call."""
    import torch
    clip, filt = CASES[0][1], CASES[0][2]
    planes = _planes(clip)[:1]
    ref = _run(torch, planes, clip, filt, None)[0]
    monkeypatch.setenv("NEO_FFT3D_FUSED_OLA", "1")
    a = _to_dev(torch, planes[0])
    W = a.shape[2]
    e = engine.PlaneEngine(make_params(**filt), plane_descs([planes[0].shape[1:]], 8, F)[0])
    for rep in range(3):
        o = _sentinel(torch, a)
        e.reset()
        for n0 in range(0, F, 2):
            k = min(2, F - n0)
            e.filter_frames_device(n0, [_ptr(a, n) for n in range(n0 - 2, n0 + k + 2)], [W] * (k + 4),
                                   [_ptr(o, n) for n in range(n0, n0 + k)], [W] * k, 0)
        torch.cuda.synchronize()
        assert np.array_equal(o.cpu().numpy(), ref), rep
    e.close()

