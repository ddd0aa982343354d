"""Evaluate the learned noise PSD on the learned-PSD workload (needs a GPU).

    python -m neo_fft3d_b200.psd_eval [--frames 120] [--clips 3] [--seed 400]

1. Trains a model with the library defaults (2^21 generated blocks of 32x32,
   ow=oh=16, coloured noise sigma 2..10) and reports its device timing:
   block generation, training steps, tensor-core GEMM throughput.
2. Makes coloured-noise clips: the seeded 1920x1080 8-bit sinusoid field
   (luma), plus white Gaussian noise shaped by a random radially symmetric
   transfer function (4-knot monotone spline over normalised radius; knot span
   log-uniform in [0.1, 1], knots log-uniform in [span, 1], falling or rising)
   scaled to a total sigma uniform in [2, 10].
3. Filters each clip with Wiener 3D (bt=5, bw=bh=32, ow=oh=16) using the
   learned noise power (strength 3, per block and pooled over the frame) and
   with the plain scalar sigma (at the noise's true sigma and at the best
   sigma of a sweep), and reports PSNR against the clean frames over the
   frames with a full bt=5 window.
4. Times the device-resident filter with and without the model (the model's
   inference is ~14.8 GFLOP per 1080p luma frame).
Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import engine, psd, synth
from .params import make_params, plane_descs

FILT = dict(bt=5, bw=32, bh=32, ow=16, oh=16)


def noise_draw(rng):
    span = float(np.exp(np.log(0.1) * rng.uniform()))
    knots = np.exp(np.log(span) * rng.uniform(size=4))
    rising = rng.uniform() >= 0.5
    knots = np.sort(knots) if rising else np.sort(knots)[::-1]
    return [float(k) for k in knots], float(rng.uniform(2.0, 10.0))


def device_fps(noisy, model, pooled, reps=3):
    import torch
    F, H, W = noisy.shape
    p = make_params(sigma=3.0, **FILT)
    d = plane_descs([(H, W)], 8, F)[0]
    src = torch.from_numpy(noisy).cuda()
    dst = torch.empty_like(src)
    eng = engine.PlaneEngine(p, d)
    if model is not None:
        eng.set_psd(model, pooled)
    s = torch.cuda.current_stream()

    def run():
        eng.reset()
        for n in range(F):
            ptrs = [src.data_ptr() + (n + k) * H * W if 0 <= n + k < F else 0 for k in range(-2, 3)]
            eng.filter_device(n, ptrs, [W] * 5, dst.data_ptr() + n * H * W, W, s.cuda_stream)

    run()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(s)
    for _ in range(reps):
        run()
    t1.record(s)
    torch.cuda.synchronize()
    eng.close()
    return reps * F / (t0.elapsed_time(t1) / 1000.0)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--frames", type=int, default=120)
    ap.add_argument("--clips", type=int, default=3)
    ap.add_argument("--seed", type=int, default=400)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--train-only", action="store_true", help="report the training measurements only")
    ap.add_argument("--blocks", type=int, default=0, help="training blocks (0: library default)")
    args = ap.parse_args()

    m = psd.PsdModel(seed=1)
    t = time.perf_counter()
    curve, val = m.train(**({"blocks": args.blocks} if args.blocks else {}))
    wall = time.perf_counter() - t
    st = m.train_stats()
    train = dict(wall_s=wall, held_out_loss=val, first_loss=float(curve[0]), last_loss=float(curve[-1]), **st,
                 gemm_tflops=st["gemm_flops_per_step"] * st["steps"] / (st["train_ms"] / 1000.0) / 1e12,
                 blocks_per_s_generated=((args.blocks or psd.train_cfg().blocks) + 32768) / (st["generate_ms"] / 1000.0))
    if args.train_only:
        print(json.dumps(dict(train=train)), flush=True)
        m.close()
        return

    rng = np.random.default_rng(args.seed)
    clips = []
    core = slice(2, -2)
    for c in range(args.clips):
        knots, sigma = noise_draw(rng)
        noisy, clean = synth.make_coloured_clip(args.width, args.height, args.frames, knots, sigma,
                                                seed=args.seed + c)

        def score(**kw):
            out = engine.filter_clip([noisy], bits=8, **FILT, **kw)[0]
            return synth.psnr(out[core], clean[core])

        sweep = {round(float(s), 3): score(sigma=float(s)) for s in sigma * np.geomspace(0.25, 3.0, 8)}
        clips.append(dict(knots=knots, sigma=sigma, noisy=synth.psnr(noisy[core], clean[core]),
                          scalar_true_sigma=score(sigma=sigma), scalar_best=max(sweep.values()),
                          scalar_best_sigma=max(sweep, key=sweep.get),
                          learned=score(psd=m), learned_pooled=score(psd=m, psd_pooled=True)))
        if c == 0:
            fps_plain = device_fps(noisy, None, False)
            fps_learned = device_fps(noisy, m, False)
            fps_pooled = device_fps(noisy, m, True)
    mean = {k: float(np.mean([c[k] for c in clips])) for k in
            ("noisy", "scalar_true_sigma", "scalar_best", "learned", "learned_pooled")}
    line = dict(workload=f"learned_psd_{args.width}x{args.height}_bt5_bw32", frames=args.frames, train=train,
                psnr_db=dict(mean=mean, clips=clips),
                device_fps_luma=dict(scalar=fps_plain, learned=fps_learned, learned_pooled=fps_pooled,
                                     inference_ms_per_frame=1000.0 / fps_learned - 1000.0 / fps_plain))
    print(json.dumps(line), flush=True)
    m.close()


if __name__ == "__main__":
    main()
