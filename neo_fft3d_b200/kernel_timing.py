"""Per-kernel timing of the FFT3D filtering core on the 1080p bt=5 workload
(needs a GPU).

    python -m neo_fft3d_b200.kernel_timing [--frames 40] [--paths unfused:8,unfused:0]

A seeded synthetic 1080p YUV420P8 clip (synth.make_clip, noise sigma 6) is
filtered with bt=5, sigma=3, bw=bh=32, ow=oh=16, sharpen=0.3 through the C ABI
with device buffers. Each path is `form:frames_per_call`: form is the engine's
kernel sequence (NEO_FFT3D_PATH: unfused | fused | split | tc) and
frames_per_call 0 means one output frame per call (fft3d_plane_filter_device),
G > 0 frame groups of G (fft3d_plane_filter_frames_device). All planes are
queued on one stream.

Prints one JSON line per path:
  fps                     frames/s of the whole clip (all planes), 10 passes
  us_per_frame_by_kernel  per kernel kind, microseconds per output frame over
                          all planes, from events around every launch with
                          the launches queued behind a sleep so that the
                          events bracket the kernels alone
  luma_launch             per kernel kind on the luma plane: (launches,
                          microseconds per launch, algorithmic bytes per launch)
  maxdiff_vs_first        largest output difference to the first path (null
                          for the first)
"""
from __future__ import annotations

import argparse
import json
import os


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--frames", type=int, default=40)
    ap.add_argument("--paths", default="unfused:8,unfused:0")
    args = ap.parse_args()

    import torch

    from . import engine, synth
    from .params import make_params, plane_descs

    F = args.frames
    planes = synth.make_clip(1920, 1080, F, noise_sigma=6.0, seed=1001)
    p = make_params(sigma=3.0, bt=5, bw=32, bh=32, ow=16, oh=16, sharpen=0.3)
    descs = plane_descs([a.shape[1:] for a in planes], 8, F)
    dev = [torch.from_numpy(a).cuda() for a in planes]
    ref_out = None
    for spec in args.paths.split(","):
        form, group = spec.split(":")
        group = int(group)
        os.environ["NEO_FFT3D_PATH"] = form
        engs = [engine.PlaneEngine(p, d) for d in descs]
        outs = [torch.empty_like(d) for d in dev]
        strm = torch.cuda.Stream()
        s = strm.cuda_stream

        def frames(e, a, o, n0, count):
            W = a.shape[2]
            fb = a.shape[1] * W
            if group:
                ptrs = [a.data_ptr() + n * fb if 0 <= n < F else 0 for n in range(n0 - 2, n0 + count + 2)]
                e.filter_frames_device(n0, ptrs, [W] * (count + 4), [o.data_ptr() + n * fb for n in range(n0, n0 + count)],
                                       [W] * count, s)
                return
            for n in range(n0, n0 + count):
                ptrs = [a.data_ptr() + (n + d) * fb if 0 <= n + d < F else 0 for d in range(-2, 3)]
                e.filter_device(n, ptrs, [W] * 5, o.data_ptr() + n * fb, W, s)

        def run():
            for e, a, o in zip(engs, dev, outs):
                e.reset()
                step = group or F
                for n0 in range(0, F, step):
                    frames(e, a, o, n0, min(step, F - n0))

        for _ in range(3):
            run()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(strm)
        for _ in range(10):
            run()
        t1.record(strm)
        torch.cuda.synchronize()
        fps = 10 * F / (t0.elapsed_time(t1) / 1000.0)
        # per-kernel timing: each call queued behind a sleep, launches bracketed by events
        for e in engs:
            e.set_timing(True)
        with torch.cuda.stream(strm):
            for e, a, o in zip(engs, dev, outs):
                e.reset()
                step = max(group, 1)
                for n0 in range(0, F, step):
                    torch.cuda._sleep(1_000_000)
                    frames(e, a, o, n0, min(step, F - n0))
                torch.cuda.synchronize()
        tim = [e.timing() for e in engs]
        for e in engs:
            e.set_timing(False)
        per = {}
        for k in tim[0]:
            ms = sum(t[k][1] for t in tim)
            if ms > 0:
                per[k] = round(1000.0 * ms / F, 2)
        luma = {k: (int(v[0]), round(1000.0 * v[1] / v[0], 1), v[2] / v[0]) for k, v in tim[0].items() if v[0]}
        same = None
        if ref_out is None:
            ref_out = [o.clone() for o in outs]
        else:
            same = [int((o.to(torch.int16) - r.to(torch.int16)).abs().max().item()) for o, r in zip(outs, ref_out)]
        print(spec, json.dumps(dict(fps=round(fps), us_per_frame_by_kernel=per, luma_launch=luma,
                                    maxdiff_vs_first=same)), flush=True)
        for e in engs:
            e.close()


if __name__ == "__main__":
    main()
