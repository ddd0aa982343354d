"""The overlap-add's 4-pixels-per-thread kernel (chosen when the block step,
overlap and width are multiples of 4 and the output rows are aligned) must
write exactly what the one-pixel-per-thread kernel writes (chosen for an
output one sample off alignment), for 8-bit, 10-bit and float samples,
interlaced planes and several block geometries."""
import numpy as np
import pytest

from neo_fft3d_b200 import engine, synth
from neo_fft3d_b200.params import make_params, plane_descs

F = 9

CASES = [
    ("8bit_bw32", dict(width=200, height=136, bits=8), dict(sigma=3.0, bt=3, sharpen=0.3)),
    ("10bit_bw48", dict(width=176, height=144, bits=10), dict(sigma=8.0, bt=5, bw=48, bh=48, ow=16, oh=16)),
    ("8bit_interlaced_crop", dict(width=160, height=128, bits=8),
     dict(sigma=2.0, bt=3, interlaced=1, l=4, r=8, t=2, b=2)),
    ("8bit_bw16_ow4", dict(width=128, height=96, bits=8), dict(sigma=2.0, bt=2, bw=16, bh=16, ow=4, oh=4)),
]


def _run(torch, e, a, offset):
    """Filter every frame into a buffer whose rows start `offset` samples in."""
    Fr, H, W = a.shape
    es = a.element_size()
    buf = torch.zeros((Fr, H, W + 4), dtype=a.dtype, device="cuda")
    st = a.shape[2] * es
    dst_stride = (W + 4) * es
    for n in range(Fr):
        ptrs = [a.data_ptr() + (n + d) * H * st if 0 <= n + d < Fr else 0 for d in range(-2, 3)]
        e.filter_device(n, ptrs, [st] * 5, buf.data_ptr() + n * H * dst_stride + offset * es, dst_stride, 0)
    torch.cuda.synchronize()
    return buf[:, :, offset:offset + W].cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("name,clip,filt", CASES, ids=[c[0] for c in CASES])
def test_four_pixel_overlap_add_matches_scalar(gpu, name, clip, filt):
    import torch
    planes = synth.make_clip(frames=F, noise_sigma=5.0 * (4 if clip["bits"] == 10 else 1), seed=81, **clip)
    descs = plane_descs([p.shape[1:] for p in planes], clip["bits"], F)
    for p, d in zip(planes, descs):
        a = torch.from_numpy(p.astype(np.int16) if p.dtype == np.uint16 else p).cuda()
        outs = []
        for offset in (0, 1):  # aligned rows: 4-pixel kernel; one sample in: one-pixel kernel
            e = engine.PlaneEngine(make_params(**filt), d)
            outs.append(_run(torch, e, a, offset))
            e.close()
        assert np.array_equal(outs[0], outs[1]), name


@pytest.mark.gpu
def test_four_pixel_overlap_add_float_samples(gpu):
    import torch
    planes = synth.make_clip(frames=F, noise_sigma=5.0, seed=82, width=160, height=96, bits=8)
    p = (planes[0].astype(np.float32) / 255.0)
    d = plane_descs([p.shape[1:]], 32, F)[0]
    a = torch.from_numpy(p).cuda()
    outs = []
    for offset in (0, 1):
        e = engine.PlaneEngine(make_params(sigma=3.0 / 255.0, bt=3), d)
        outs.append(_run(torch, e, a, offset))
        e.close()
    assert np.array_equal(outs[0], outs[1])
