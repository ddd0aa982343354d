"""Batched uneven-streams workload (needs a GPU).

    python -m neo_fft3d_b200.batch_eval [--frames 60] [--seed 3000] [--mix uneven|small]

mix "uneven" (default): 48 concurrent YUV420 streams of 60 frames: 16 at
640x480 8-bit, 16 at 1280x720 8-bit, 12 at 1920x1080 8-bit and 4 at
3840x2160 10-bit (uint16), per-stream seeds. mix "small": 48 streams at
640x480 8-bit. Per stream: noise sigma uniform on [2, 10] (8-bit units, x4
for 10-bit), bt uniform on {1..5}, bw = bh from {32, 48} with
ow = oh = bw / 2; filter sigma = the noise sigma. Clips are generated on the
device with the sinusoid-field formula of synth.make_clip.

All planes are filtered per time step: (a) one plane at a time
(fft3d_plane_filter_device, 3 launches per plane) on one stream, and (b) as
one batched step (fft3d_batch_step: one persistent launch per kernel variant,
phase and wave; autotuned; CUDA-graph replayed). With --group G (default 8)
the same comparison runs again in frame groups: (c) each plane's next G
output frames per call (fft3d_plane_filter_frames_device), plane after plane
on one stream, against (d) one batched step of G consecutive frames of every
plane (each plane's frames run as one run of its filter/inverse with one CTA
per block). Every pass is timed after a first untimed pass (which, for the
batch, tunes and captures); the outputs of each pair are compared byte for
byte. Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import engine, synth
from .params import make_params, plane_descs

MIXES = {
    "uneven": [(16, 640, 480, 8), (16, 1280, 720, 8), (12, 1920, 1080, 8), (4, 3840, 2160, 10)],
    "small": [(48, 640, 480, 8)],
}


def streams(kinds, seed: int):
    rng = np.random.default_rng(seed)
    out = []
    for count, w, h, bits in kinds:
        for _ in range(count):
            sigma = float(rng.uniform(2.0, 10.0))
            bt = int(rng.integers(1, 6))
            bw = int(rng.choice([32, 48]))
            out.append(dict(width=w, height=h, bits=bits, sigma=sigma, bt=bt, bw=bw, seed=int(rng.integers(1 << 30))))
    return out


def main():
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--frames", type=int, default=60)
    ap.add_argument("--seed", type=int, default=3000)
    ap.add_argument("--mix", default="uneven", choices=sorted(MIXES))
    ap.add_argument("--group", type=int, default=8, help="frames per plane per call/step of the grouped passes")
    ap.add_argument("--no-tune", action="store_true", help="default schedules (one wave), no autotuning")
    ap.add_argument("--phase-timing", action="store_true",
                    help="one more pass of each grouped form with per-kernel timing (per-plane) / per-phase timing (batch)")
    args = ap.parse_args()
    F = args.frames
    kinds = MIXES[args.mix]
    cfg = streams(kinds, args.seed)
    clips, engs, outs = [], [], []
    canonical = 0.0
    for s in cfg:
        noise = s["sigma"] * (4 if s["bits"] == 10 else 1)
        planes = synth.make_clip_device(s["width"], s["height"], F, bits=s["bits"], noise_sigma=noise, seed=s["seed"])
        p = make_params(sigma=s["sigma"], bt=s["bt"], bw=s["bw"], bh=s["bw"], ow=s["bw"] // 2, oh=s["bw"] // 2)
        descs = plane_descs([tuple(a.shape[1:]) for a in planes], s["bits"], F)
        for a, d in zip(planes, descs):
            e = engine.PlaneEngine(p, d)
            engs.append(e)
            clips.append(a)
            outs.append(torch.empty_like(a))
            # canonical cached-spectrum bytes per output frame: pixels in,
            # newest spectrum out, bt spectra in, pixels out
            S = e.nblocks * s["bw"] * (s["bw"] // 2 + 1) * 8
            P = a.shape[1] * a.shape[2] * a.element_size()
            canonical += 2 * P + S + max(s["bt"], 1) * S
    torch.cuda.synchronize()
    # every pass on one dedicated stream, which the timing events bracket
    # (stream 0 would mean each plane's own stream in the per-plane calls)
    stream = torch.cuda.Stream()

    def item(e, a, o, n):
        fb = a.shape[1] * a.shape[2] * a.element_size()
        ptrs = [a.data_ptr() + (n + k) * fb if 0 <= n + k < F else 0 for k in range(-2, 3)]
        return e, n, ptrs, [a.shape[2] * a.element_size()] * 5, o.data_ptr() + n * fb, a.shape[2] * a.element_size()

    def per_plane_pass():
        for n in range(F):
            for e, a, o in zip(engs, clips, outs):
                _, _, ptrs, st, dst, ds = item(e, a, o, n)
                e.filter_device(n, ptrs, st, dst, ds, stream.cuda_stream)

    batch = engine.Batch(tuning=not args.no_tune)

    def batched_pass():
        for n in range(F):
            batch.step([item(e, a, o, n) for e, a, o in zip(engs, clips, outs)], stream.cuda_stream)

    host_s = {}

    def timed(fn):
        for e in engs:
            e.reset()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        h = time.perf_counter()
        fn()
        host_s[fn.__name__] = time.perf_counter() - h  # the host's time to issue the pass
        t1.record(stream)
        torch.cuda.synchronize()
        return t0.elapsed_time(t1) / 1000.0

    G = args.group

    def group_items(e, a, o, n0, k):
        fb = a.shape[1] * a.shape[2] * a.element_size()
        st = a.shape[2] * a.element_size()
        return [item(e, a, o, n) for n in range(n0, n0 + k)], \
            ([a.data_ptr() + m * fb if 0 <= m < F else 0 for m in range(n0 - 2, n0 + k + 2)], [st] * (k + 4),
             [o.data_ptr() + n * fb for n in range(n0, n0 + k)], [st] * k)

    def per_plane_grouped_pass():
        for n0 in range(0, F, G):
            k = min(G, F - n0)
            for e, a, o in zip(engs, clips, outs):
                ptrs, sts, dsts, dsts_st = group_items(e, a, o, n0, k)[1]
                e.filter_frames_device(n0, ptrs, sts, dsts, dsts_st, stream.cuda_stream)

    gbatch = engine.Batch(tuning=not args.no_tune)

    def batched_grouped_pass():
        for n0 in range(0, F, G):
            k = min(G, F - n0)
            its = []
            for e, a, o in zip(engs, clips, outs):
                its += group_items(e, a, o, n0, k)[0]
            gbatch.step(its, stream.cuda_stream)

    timed(per_plane_pass)  # warm-up
    l0 = engine.kernel_launches()
    t_plane = timed(per_plane_pass)
    launches_plane = engine.kernel_launches() - l0
    ref = [o.clone() for o in outs]
    timed(batched_pass)  # tunes and captures
    l0 = engine.kernel_launches()
    t_batch = timed(batched_pass)
    launches_batch = engine.kernel_launches() - l0
    same = all(bool(torch.equal(r, o)) for r, o in zip(ref, outs))
    stats = batch.stats()
    grouped = None
    if G > 1:
        timed(per_plane_grouped_pass)
        l0 = engine.kernel_launches()
        t_pg = timed(per_plane_grouped_pass)
        launches_pg = engine.kernel_launches() - l0
        same_pg = all(bool(torch.equal(r, o)) for r, o in zip(ref, outs))
        # tuning and capture: every step shape of the pass (clip start, middle,
        # end) first takes its tuning steps
        for _ in range(10):
            before = gbatch.stats()["tuning_steps"]
            timed(batched_grouped_pass)
            if gbatch.stats()["tuning_steps"] == before:
                break
        l0 = engine.kernel_launches()
        t_bg = timed(batched_grouped_pass)
        launches_bg = engine.kernel_launches() - l0
        same_bg = all(bool(torch.equal(r, o)) for r, o in zip(ref, outs))
        phases = None
        if args.phase_timing:
            for e in engs:
                e.set_timing(True)
            timed(per_plane_grouped_pass)
            per = {}
            for e in engs:
                for k, (n, ms, _) in e.timing().items():
                    per[k] = per.get(k, 0.0) + ms
                e.set_timing(False)
            gbatch.set_timing(True)
            timed(batched_grouped_pass)
            bt_ = gbatch.timing()
            gbatch.set_timing(False)
            phases = dict(per_plane_ms_per_pass={k: v for k, v in per.items() if v > 0},
                          batched_ms_per_pass={k: v[1] for k, v in bt_.items()})
        grouped = dict(frames_per_call=G, phase_timing=phases,
                       stream_frames_per_s=dict(per_plane=len(cfg) * F / t_pg, batched=len(cfg) * F / t_bg),
                       speedup=t_pg / t_bg,
                       kernels_per_frame=dict(per_plane=launches_pg / F, batched=launches_bg / F),
                       outputs_identical_to_one_frame_per_call=dict(per_plane=same_pg, batched=same_bg),
                       batch_stats=gbatch.stats())
    peak = None
    peaks = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    if os.path.exists(peaks):
        with open(peaks) as f:
            peak = float(json.load(f)["hbm_gbs"])
    stream_frames = len(cfg) * F
    line = dict(workload=f"batched_{len(cfg)}_{args.mix}_streams", frames_per_stream=F, streams=len(cfg),
                planes=len(engs),
                stream_frames_per_s=dict(per_plane=stream_frames / t_plane, batched=stream_frames / t_batch),
                speedup=t_plane / t_batch,
                kernels_per_step=dict(per_plane=launches_plane / F, batched=launches_batch / F),
                canonical_bytes_per_step=canonical,
                hbm_gbs=dict(per_plane=canonical * F / t_plane / 1e9, batched=canonical * F / t_batch / 1e9),
                hbm_peak_gbs=peak, outputs_identical=same, batch_stats=stats,
                mix={f"{w}x{h}/{b}bit": c for c, w, h, b in kinds},
                bt_counts={str(k): sum(1 for s in cfg if s["bt"] == k) for k in range(1, 6)},
                bw_counts={str(k): sum(1 for s in cfg if s["bw"] == k) for k in (32, 48)})
    if peak:
        line["hbm_frac"] = {k: v / peak for k, v in line["hbm_gbs"].items()}
    line["host_issue_s_per_pass"] = dict(per_plane=host_s.get("per_plane_pass"), batched=host_s.get("batched_pass"))
    if grouped:
        grouped["hbm_gbs"] = {k: canonical * v / len(cfg) / 1e9 for k, v in grouped["stream_frames_per_s"].items()}
        grouped["host_issue_s_per_pass"] = dict(per_plane=host_s.get("per_plane_grouped_pass"),
                                                batched=host_s.get("batched_grouped_pass"))
        if peak:
            grouped["hbm_frac"] = {k: v / peak for k, v in grouped["hbm_gbs"].items()}
        line["frame_groups"] = grouped
    print(json.dumps(line), flush=True)
    gbatch.close()
    batch.close()
    for e in engs:
        e.close()


if __name__ == "__main__":
    main()
