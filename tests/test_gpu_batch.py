"""Batched multi-plane scheduler (fft3d_batch_*): a step of many planes of
mixed clips must give byte-identical output to filtering each plane on its own
(fft3d_plane_filter_device), through the tuning steps, the graph-captured
steps and the clip edges (btcur = 1, Kalman frame 0, crop borders)."""
import ctypes

import numpy as np
import pytest

from neo_fft3d_b200 import engine, synth
from neo_fft3d_b200.params import make_params, plane_descs

F = 26
CLIPS = [
    dict(clip=dict(width=200, height=136, bits=8, noise_sigma=4.0, seed=61), filt=dict(sigma=2.0, bt=5, bw=32, bh=32,
                                                                                       ow=16, oh=16, sharpen=0.3)),
    dict(clip=dict(width=176, height=144, bits=8, noise_sigma=6.0, seed=62), filt=dict(sigma=3.0, bt=3, bw=48, bh=48,
                                                                                       ow=16, oh=16)),
    dict(clip=dict(width=160, height=120, bits=10, noise_sigma=12.0, seed=63), filt=dict(sigma=3.0, bt=0, bw=32, bh=32,
                                                                                         ow=16, oh=16)),
    dict(clip=dict(width=144, height=112, bits=8, noise_sigma=5.0, seed=64), filt=dict(sigma=2.5, bt=1, bw=32, bh=32,
                                                                                       ow=16, oh=16, l=8, t=4, r=6,
                                                                                       b=2, dehalo=0.4)),
    dict(clip=dict(width=208, height=128, bits=8, noise_sigma=4.0, seed=65), filt=dict(sigma=2.0, bt=2, bw=32, bh=32,
                                                                                       ow=16, oh=16)),
]


def _setup(torch):
    clips = []
    for c in CLIPS:
        planes = synth.make_clip(frames=F, **c["clip"])
        bits = c["clip"]["bits"]
        p = make_params(**c["filt"])
        descs = plane_descs([a.shape[1:] for a in planes], bits, F)
        clips.append(dict(planes=[torch.from_numpy(a.astype(np.int16) if a.dtype == np.uint16 else a).cuda()
                                  for a in planes], params=p, descs=descs))
    return clips


def _window(a, n, F):
    fb = a.shape[1] * a.shape[2] * a.element_size()
    return [a.data_ptr() + (n + d) * fb if 0 <= n + d < F else 0 for d in range(-2, 3)], [a.shape[2] * a.element_size()] * 5


def _per_plane(torch, clips):
    outs = []
    for c in clips:
        for a, d in zip(c["planes"], c["descs"]):
            e = engine.PlaneEngine(c["params"], d)
            o = torch.empty_like(a)
            fb = a.shape[1] * a.shape[2] * a.element_size()
            for n in range(F):
                ptrs, st = _window(a, n, F)
                e.filter_device(n, ptrs, st, o.data_ptr() + n * fb, a.shape[2] * a.element_size(), 0)
            torch.cuda.synchronize()
            e.close()
            outs.append(o.cpu().numpy())
    return outs


def _batched(torch, clips, tuning):
    engs, outs, srcs = [], [], []
    for c in clips:
        for a, d in zip(c["planes"], c["descs"]):
            engs.append(engine.PlaneEngine(c["params"], d))
            outs.append(torch.empty_like(a))
            srcs.append(a)
    b = engine.Batch(tuning=tuning)
    stream = torch.cuda.current_stream().cuda_stream
    for n in range(F):
        items = []
        for e, a, o in zip(engs, srcs, outs):
            ptrs, st = _window(a, n, F)
            fb = a.shape[1] * a.shape[2] * a.element_size()
            items.append((e, n, ptrs, st, o.data_ptr() + n * fb, a.shape[2] * a.element_size()))
        b.step(items, stream)
    torch.cuda.synchronize()
    stats = b.stats()
    b.close()
    for e in engs:
        e.close()
    return [o.cpu().numpy() for o in outs], stats


@pytest.mark.gpu
@pytest.mark.parametrize("tuning", [False, True], ids=["default_schedule", "autotuned"])
def test_batch_matches_per_plane(gpu, tuning):
    import torch
    clips = _setup(torch)
    ref = _per_plane(torch, clips)
    got, stats = _batched(torch, clips, tuning)
    for i, (r, g) in enumerate(zip(ref, got)):
        assert np.array_equal(r, g), i
    assert stats["steps"] == F
    assert stats["kernels_last_step"] < 45  # 15 planes x 3 kernels unbatched
    if not tuning:
        assert stats["graph_launches"] > 0
    else:
        assert stats["tuning_steps"] > 0


@pytest.mark.gpu
def test_batch_rejects_bad_steps(gpu, monkeypatch):
    import torch
    a = torch.zeros((4, 64, 64), dtype=torch.uint8, device="cuda")
    p = make_params(sigma=2.0, bt=1, bw=32, bh=32, ow=16, oh=16)
    d = plane_descs([(64, 64)], 8, 4)[0]
    e = engine.PlaneEngine(p, d)
    b = engine.Batch()
    ptrs, st = _window(a, 0, 4)
    with pytest.raises(engine.FFT3DError, match="appears twice"):
        b.step([(e, 0, ptrs, st, a.data_ptr(), 64), (e, 0, ptrs, st, a.data_ptr(), 64)])
    monkeypatch.setenv("NEO_FFT3D_PATH", "tc")
    etc = engine.PlaneEngine(p, d)
    with pytest.raises(engine.FFT3DError, match="tensor-core|default"):
        b.step([(etc, 0, ptrs, st, a.data_ptr(), 64)])
    etc.close()
    e.close()
    b.close()


def _grouped(torch, clips, k, tuning):
    """Steps of k consecutive frames of every Wiener/sharpen plane (a frame
    group per plane); the last step takes what is left."""
    engs, outs, srcs = [], [], []
    for c in clips:
        if c["params"].bt == 0:
            continue
        for a, d in zip(c["planes"], c["descs"]):
            engs.append(engine.PlaneEngine(c["params"], d))
            outs.append(torch.empty_like(a))
            srcs.append(a)
    b = engine.Batch(tuning=tuning)
    stream = torch.cuda.current_stream().cuda_stream
    for n0 in range(0, F, k):
        items = []
        for e, a, o in zip(engs, srcs, outs):
            fb = a.shape[1] * a.shape[2] * a.element_size()
            for n in range(n0, min(n0 + k, F)):
                ptrs, st = _window(a, n, F)
                items.append((e, n, ptrs, st, o.data_ptr() + n * fb, a.shape[2] * a.element_size()))
        b.step(items, stream)
    torch.cuda.synchronize()
    stats = b.stats()
    b.close()
    for e in engs:
        e.close()
    return [o.cpu().numpy() for o in outs], stats


@pytest.mark.gpu
@pytest.mark.parametrize("k,tuning", [(4, False), (3, True), (8, False)], ids=["k4", "k3_autotuned", "k8"])
def test_frame_groups_match_per_plane(gpu, k, tuning):
    """Several consecutive frames of each plane in one step (frame groups,
    including the clip-edge frames with btcur = 1 and a short last group):
    byte-identical to one-frame-at-a-time filtering."""
    import torch
    clips = _setup(torch)
    ref = _per_plane(torch, [c for c in clips if c["params"].bt != 0])
    got, stats = _grouped(torch, clips, k, tuning)
    for i, (r, g) in enumerate(zip(ref, got)):
        assert np.array_equal(r, g), i
    assert stats["steps"] == (F + k - 1) // k


@pytest.mark.gpu
def test_frame_group_rules(gpu):
    import torch
    a = torch.zeros((6, 64, 64), dtype=torch.uint8, device="cuda")
    d = plane_descs([(64, 64)], 8, 6)[0]
    b = engine.Batch()
    ew = engine.PlaneEngine(make_params(sigma=2.0, bt=3, bw=32, bh=32, ow=16, oh=16), d)
    ek = engine.PlaneEngine(make_params(sigma=2.0, bt=0, bw=32, bh=32, ow=16, oh=16), d)

    def item(e, n):
        ptrs, st = _window(a, n, 6)
        return (e, n, ptrs, st, a.data_ptr(), 64)

    with pytest.raises(engine.FFT3DError, match="not consecutive"):
        b.step([item(ew, 1), item(ew, 3)])
    with pytest.raises(engine.FFT3DError, match="not consecutive"):
        b.step([item(ew, 2), item(ew, 1)])
    with pytest.raises(engine.FFT3DError, match="Kalman"):
        b.step([item(ek, 1), item(ek, 2)])
    ew.close()
    ek.close()
    b.close()


@pytest.mark.gpu
def test_batch_timing_counts_phases(gpu):
    """Per-phase timing: every timed step's launches are counted, with their
    algorithmic bytes (a frame group reads each window spectrum once)."""
    import torch
    clips = _setup(torch)[:1]
    c = clips[0]
    engs = [engine.PlaneEngine(c["params"], d) for d in c["descs"]]
    outs = [torch.empty_like(a) for a in c["planes"]]
    b = engine.Batch(tuning=False)
    b.set_timing(True)
    stream = torch.cuda.current_stream().cuda_stream
    k = 4
    for n0 in range(4, 12, k):
        items = []
        for e, a, o in zip(engs, c["planes"], outs):
            fb = a.shape[1] * a.shape[2] * a.element_size()
            for n in range(n0, n0 + k):
                ptrs, st = _window(a, n, F)
                items.append((e, n, ptrs, st, o.data_ptr() + n * fb, a.shape[2] * a.element_size()))
        b.step(items, stream)
    t = b.timing()
    assert t["forward"][0] >= 1 and t["filter_inverse"][0] == 2 and t["overlap_add"][0] == 2
    assert all(v[1] > 0 for k_, v in t.items() if v[0] > 0)
    # filter/inverse of the second step (frames 8..11, bt = 5): spectra of
    # frames 6..13 once per plane, and four time-domain buffers per plane
    S = sum(e.nblocks * 32 * 17 * 8 for e in engs)
    T = sum(e.nblocks * 32 * 32 * 4 for e in engs)
    assert t["filter_inverse"][2] == pytest.approx(2 * (8 * S + 4 * T))
    b.close()
    for e in engs:
        e.close()


@pytest.mark.gpu
def test_frame_groups_planes_larger_than_a_wave(gpu):
    """A 1080p plane's new spectra and time-domain blocks (about 70 MB) exceed
    the tuner's smallest wave budget (24 MiB), which its first step of every
    shape tries: all frames of a plane's group, whose filter/inverse runs as
    one run, must stay in one wave with the forward transforms it reads."""
    import torch
    Fb = 12
    planes = synth.make_clip(1920, 1080, Fb, noise_sigma=5.0, seed=66)
    p = make_params(sigma=2.5, bt=3, bw=32, bh=32, ow=16, oh=16, sharpen=0.2)
    descs = plane_descs([a.shape[1:] for a in planes], 8, Fb)
    dev = [torch.from_numpy(a).cuda() for a in planes]
    ref = []
    for a, d in zip(dev, descs):
        e = engine.PlaneEngine(p, d)
        o = torch.empty_like(a)
        fb = a.shape[1] * a.shape[2]
        for n in range(Fb):
            ptrs, st = _window(a, n, Fb)
            e.filter_device(n, ptrs, st, o.data_ptr() + n * fb, a.shape[2], 0)
        torch.cuda.synchronize()
        e.close()
        ref.append(o.cpu().numpy())
    engs = [engine.PlaneEngine(p, d) for d in descs]
    outs = [torch.empty_like(a) for a in dev]
    b = engine.Batch(tuning=True)
    stream = torch.cuda.current_stream().cuda_stream
    for n0 in range(0, Fb, 4):
        items = []
        for e, a, o in zip(engs, dev, outs):
            fb = a.shape[1] * a.shape[2]
            for n in range(n0, n0 + 4):
                ptrs, st = _window(a, n, Fb)
                items.append((e, n, ptrs, st, o.data_ptr() + n * fb, a.shape[2]))
        b.step(items, stream)
    torch.cuda.synchronize()
    b.close()
    for e in engs:
        e.close()
    for i, (r, o) in enumerate(zip(ref, outs)):
        assert np.array_equal(r, o.cpu().numpy()), i
