"""Frame groups (fft3d_plane_filter_frames_device): several consecutive
output frames of one plane in one call must give byte-identical output to
filtering the frames one at a time (fft3d_plane_filter_device), for every
Wiener 3D window length, block size, crop, pattern and sample type, across
the clip-edge frames (btcur = 1) and with groups of every size; planes that
are not grouped (Kalman, Wiener 2D, sharpen only, the tensor-core path) must
give their per-frame output too."""
import numpy as np
import pytest

from neo_fft3d_b200 import engine, synth
from neo_fft3d_b200.params import make_params, plane_descs

F = 23

CASES = [
    ("bt5_sharpen", dict(width=200, height=136, bits=8, seed=71), dict(sigma=3.0, bt=5, sharpen=0.3)),
    ("bt4_bw48", dict(width=176, height=144, bits=8, seed=72), dict(sigma=2.5, bt=4, bw=48, bh=48, ow=16, oh=16)),
    ("bt3_crop_dehalo", dict(width=160, height=128, bits=8, seed=73),
     dict(sigma=2.0, bt=3, l=6, t=4, r=8, b=2, dehalo=0.5)),
    ("bt2_degrid0", dict(width=144, height=112, bits=8, seed=74), dict(sigma=2.0, bt=2, degrid=0.0)),
    ("bt5_10bit", dict(width=160, height=120, bits=10, seed=75), dict(sigma=8.0, bt=5)),
    ("bt3_pattern", dict(width=160, height=128, bits=8, seed=76), dict(sigma=2.0, bt=3, pfactor=1.0, pframe=3)),
    ("kalman", dict(width=128, height=96, bits=8, seed=77), dict(sigma=3.0, bt=0)),
    ("bt1", dict(width=128, height=96, bits=8, seed=78), dict(sigma=3.0, bt=1, sharpen=0.2)),
    ("sharpen_only", dict(width=128, height=96, bits=8, seed=79), dict(sigma=3.0, bt=-1, sharpen=0.4)),
]


def _clip(torch, clip):
    planes = synth.make_clip(frames=F, noise_sigma=5.0 * (4 if clip["bits"] == 10 else 1), **clip)
    dev = [torch.from_numpy(a.astype(np.int16) if a.dtype == np.uint16 else a).cuda() for a in planes]
    return planes, dev


def _engines(planes, clip, filt):
    p = make_params(**filt)
    descs = plane_descs([a.shape[1:] for a in planes], clip["bits"], F)
    engs = [engine.PlaneEngine(p, d) for d in descs]
    if filt.get("pfactor"):
        for e, a in zip(engs, planes):
            e.set_pattern_frame(a[filt["pframe"]])
    return engs


def _ptr(a, n):
    fb = a.shape[1] * a.shape[2] * a.element_size()
    return a.data_ptr() + n * fb if 0 <= n < a.shape[0] else 0


def _per_frame(torch, planes, dev, clip, filt):
    engs = _engines(planes, clip, filt)
    outs = []
    for e, a in zip(engs, dev):
        o = torch.full_like(a, 1)  # a value no filtered sample takes: unwritten pixels show
        st = a.shape[2] * a.element_size()
        for n in range(F):
            e.filter_device(n, [_ptr(a, n + d) for d in range(-2, 3)], [st] * 5, _ptr(o, n), st, 0)
        outs.append(o)
        e.close()
    torch.cuda.synchronize()
    return [o.cpu().numpy() for o in outs]


def _grouped(torch, planes, dev, clip, filt, sizes):
    """Frames in groups of the given sizes (cycled) per plane."""
    engs = _engines(planes, clip, filt)
    outs = []
    for e, a in zip(engs, dev):
        o = torch.full_like(a, 1)  # a value no filtered sample takes: unwritten pixels show
        st = a.shape[2] * a.element_size()
        n0, i = 0, 0
        while n0 < F:
            k = min(sizes[i % len(sizes)], F - n0)
            e.filter_frames_device(n0, [_ptr(a, n) for n in range(n0 - 2, n0 + k + 2)], [st] * (k + 4),
                                   [_ptr(o, n) for n in range(n0, n0 + k)], [st] * k, 0)
            n0 += k
            i += 1
        outs.append(o)
        e.close()
    torch.cuda.synchronize()
    return [o.cpu().numpy() for o in outs]


@pytest.mark.gpu
@pytest.mark.parametrize("name,clip,filt", CASES, ids=[c[0] for c in CASES])
def test_frame_groups_match_per_frame(gpu, name, clip, filt):
    import torch
    planes, dev = _clip(torch, clip)
    ref = _per_frame(torch, planes, dev, clip, filt)
    for sizes in ([4], [16], [3, 1, 7, 2]):
        got = _grouped(torch, planes, dev, clip, filt, sizes)
        for i, (r, g) in enumerate(zip(ref, got)):
            assert np.array_equal(r, g), (name, sizes, i, int(np.abs(r.astype(int) - g).max()))


@pytest.mark.gpu
def test_frame_groups_tensor_core_path(gpu, monkeypatch):
    """The tensor-core path in frame groups (its forward transform per frame,
    the grouped filter/inverse and overlap-add) equals it one frame at a
    time."""
    import torch
    monkeypatch.setenv("NEO_FFT3D_PATH", "tc")
    clip, filt = CASES[0][1], CASES[0][2]
    planes, dev = _clip(torch, clip)
    ref = _per_frame(torch, planes, dev, clip, filt)
    for sizes in ([5], [8, 3]):
        got = _grouped(torch, planes, dev, clip, filt, sizes)
        for r, g in zip(ref, got):
            assert np.array_equal(r, g)


@pytest.mark.gpu
def test_frame_group_timing_counts_unique_spectra(gpu):
    """Per-kernel timing of a frame group: one forward launch for the new
    frames and one filter/inverse launch whose algorithmic bytes count each
    window spectrum once."""
    import torch
    clip, filt = CASES[0][1], CASES[0][2]
    planes, dev = _clip(torch, clip)
    e = _engines(planes[:1], clip, filt)[0]
    a = dev[0]
    o = torch.full_like(a, 1)  # a value no filtered sample takes: unwritten pixels show
    st = a.shape[2]
    e.filter_frames_device(4, [_ptr(a, n) for n in range(2, 12)], [st] * 10, [_ptr(o, n) for n in range(4, 10)],
                           [st] * 6, 0)  # warm: frames 4..9
    e.timing()
    e.set_timing(True)
    e.filter_frames_device(10, [_ptr(a, n) for n in range(8, 18)], [st] * 10, [_ptr(o, n) for n in range(10, 16)],
                           [st] * 6, 0)
    torch.cuda.synchronize()
    t = e.timing()
    e.set_timing(False)
    S = e.nblocks * 32 * 17 * 8
    T = e.nblocks * 32 * 32 * 4
    assert t["filter_inverse"][0] == 1
    assert t["filter_inverse"][2] == pytest.approx(10 * S + 6 * T)  # frames 8..17 once, six outputs
    # frames 12..17 are new: transformed by one launch
    assert t["forward"][0] == 1
    assert t["forward"][2] == pytest.approx(6 * (a.shape[1] * a.shape[2] + S))
    e.close()


@pytest.mark.gpu
def test_frame_group_argument_checks(gpu):
    import torch
    a = torch.zeros((4, 64, 64), dtype=torch.uint8, device="cuda")
    e = engine.PlaneEngine(make_params(sigma=2.0, bt=3), plane_descs([(64, 64)], 8, 4)[0])
    L = engine.lib()
    import ctypes
    p = (ctypes.c_void_p * 21)()
    s = (ctypes.c_int * 21)()
    d = (ctypes.c_void_p * 17)(*([a.data_ptr()] * 17))
    ds = (ctypes.c_int * 17)()
    assert L.fft3d_plane_filter_frames_device(e.h, 0, 17, p, s, d, ds, None) == -1
    assert "frame group" in L.fft3d_last_error().decode()
    assert L.fft3d_plane_filter_frames_device(e.h, 0, 0, p, s, d, ds, None) == -1
    e.close()


def _host_per_frame(planes, clip, filt):
    engs = _engines(planes, clip, filt)
    outs = []
    for e, a in zip(engs, planes):
        o = np.empty_like(a)
        for n in range(F):
            e.filter(n, [a[n + d] if 0 <= n + d < F else None for d in range(-2, 3)], o[n])
        outs.append(o)
        e.close()
    return outs


def _host_grouped(planes, clip, filt, sizes):
    engs = _engines(planes, clip, filt)
    outs = []
    for e, a in zip(engs, planes):
        o = np.empty_like(a)
        n0, i = 0, 0
        while n0 < F:
            k = min(sizes[i % len(sizes)], F - n0)
            e.filter_frames(n0, [a[n] if 0 <= n < F else None for n in range(n0 - 2, n0 + k + 2)],
                            [o[n] for n in range(n0, n0 + k)])
            n0 += k
            i += 1
        outs.append(o)
        e.close()
    return outs


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["bt5_sharpen", "bt5_10bit", "bt3_crop_dehalo", "kalman"])
def test_host_frame_groups_match_per_frame(gpu, name):
    """Host buffers: frame groups (uploads of only the missing frames,
    downloads of the group's outputs) equal the one-frame host path."""
    clip, filt = next((c[1], c[2]) for c in CASES if c[0] == name)
    planes = synth.make_clip(frames=F, noise_sigma=5.0 * (4 if clip["bits"] == 10 else 1), **clip)
    ref = _host_per_frame(planes, clip, filt)
    for sizes in ([8], [3, 5, 16]):
        got = _host_grouped(planes, clip, filt, sizes)
        for i, (r, g) in enumerate(zip(ref, got)):
            assert np.array_equal(r, g), (name, sizes, i)


@pytest.mark.gpu
@pytest.mark.parametrize("threads,group", [(4, 4), (7, 2)])
def test_host_frame_groups_from_threads(gpu, threads, group):
    """Several host threads taking groups of one plane from a shared counter
    (as the bench's end-to-end arm does): the outputs equal a serial run.
    Seven threads outnumber the plane's four group staging sets, so calls
    wait for a free set."""
    import threading
    clip, filt = CASES[0][1], CASES[0][2]
    planes = synth.make_clip(frames=F, noise_sigma=5.0, **clip)
    ref = _host_grouped(planes, clip, filt, [4])
    engs = _engines(planes, clip, filt)
    outs = [np.empty_like(a) for a in planes]
    for e, a, o in zip(engs, planes, outs):
        counter, lock = [0], threading.Lock()

        def work():
            while True:
                with lock:
                    n0 = counter[0]
                    counter[0] += group
                if n0 >= F:
                    return
                k = min(group, F - n0)
                e.filter_frames(n0, [a[n] if 0 <= n < F else None for n in range(n0 - 2, n0 + k + 2)],
                                [o[n] for n in range(n0, n0 + k)])

        th = [threading.Thread(target=work) for _ in range(threads)]
        for t in th:
            t.start()
        for t in th:
            t.join()
    for r, g in zip(ref, outs):
        assert np.array_equal(r, g)
    for e in engs:
        e.close()


@pytest.mark.gpu
@pytest.mark.parametrize("grouped", [False, True], ids=["one_frame_per_call", "frame_groups"])
def test_reset_waits_for_queued_work(gpu, grouped):
    """fft3d_plane_reset right after frames were queued on a caller's stream
    (no host synchronisation) must not clear the Kalman state under those
    frames' kernels: every pass over the clip gives the same output."""
    import torch
    clip = dict(width=640, height=480, bits=8, seed=91)
    planes, dev = _clip(torch, clip)
    a = dev[0]
    p = make_params(sigma=3.0, bt=0)
    e = engine.PlaneEngine(p, plane_descs([a.shape[1:]], 8, F)[0])
    s = torch.cuda.Stream()
    st = a.shape[2]
    outs = []
    for _ in range(3):
        o = torch.full_like(a, 1)  # a value no filtered sample takes: unwritten pixels show
        e.reset()
        if grouped:
            for n0 in range(0, F, 8):
                k = min(8, F - n0)
                e.filter_frames_device(n0, [_ptr(a, n) for n in range(n0 - 2, n0 + k + 2)], [st] * (k + 4),
                                       [_ptr(o, n) for n in range(n0, n0 + k)], [st] * k, s.cuda_stream)
        else:
            for n in range(F):
                e.filter_device(n, [0, 0, _ptr(a, n), 0, 0], [st] * 5, _ptr(o, n), st, s.cuda_stream)
        outs.append(o)
    torch.cuda.synchronize()
    for o in outs[1:]:
        assert torch.equal(outs[0], o)
    e.close()



@pytest.mark.gpu
@pytest.mark.parametrize("bw,runs", [(32, 1), (48, 2)])
def test_frame_group_runs_capped_by_block_size(gpu, bw, runs):
    """A group of 8 interior frames is one filter/inverse run for 32x32 blocks
    and two runs (5 + 3 frames) for 48x48 blocks, whose 8-frame tiles would
    leave only 2 CTAs per SM; the output still equals one frame per call."""
    import torch
    clip = dict(width=176, height=144, bits=8, seed=83)
    filt = dict(sigma=2.5, bt=3, bw=bw, bh=bw, ow=16, oh=16)
    planes, dev = _clip(torch, clip)
    ref = _per_frame(torch, planes[:1], dev[:1], clip, filt)[0]
    e = _engines(planes[:1], clip, filt)[0]
    a = dev[0]
    o = torch.full_like(a, 1)  # a value no filtered sample takes: unwritten pixels show
    st = a.shape[2]

    def group(n0, k):
        e.filter_frames_device(n0, [_ptr(a, n) for n in range(n0 - 2, n0 + k + 2)], [st] * (k + 4),
                               [_ptr(o, n) for n in range(n0, n0 + k)], [st] * k, 0)

    group(0, 6)
    e.timing()
    e.set_timing(True)
    group(6, 8)  # frames 6..13: interior (btcur = bt), one mode
    torch.cuda.synchronize()
    t = e.timing()
    e.set_timing(False)
    assert t["filter_inverse"][0] == runs
    group(14, F - 14)
    torch.cuda.synchronize()
    assert np.array_equal(o.cpu().numpy(), ref)
    e.close()
