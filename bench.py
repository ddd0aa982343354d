#!/usr/bin/env python
"""Benchmark of the FFT3D filtering core on B200.

Workload (the configuration the headline metric is quoted on): 120 frames of
seeded synthetic 8-bit YUV420 at 1920x1080 (sum-of-sinusoids field moving by
<= 2 px/frame, Gaussian noise sigma 6), filtered with bt=5, sigma=3,
bw=bh=32, ow=oh=16, sharpen=0.3 (all three planes, degrid=1 default).

One step = the whole 120-frame clip filtered end to end (all planes, every
output frame, edge frames with bt=1 as the reference does), inputs resident
in HBM. The clip (373 MB) and the spectrum ring (~350 MB) are larger than L2,
so no flush is needed between steps.

Both forms of the block transform run K timed steps each: the plain FP32
register FFT (as three kernels per plane-frame, fused into two, and in frame
groups of FRAME_GROUP consecutive frames per call, whose filter/inverse is one
launch) and the tensor-core split-precision BF16 DFT-GEMM (32x32 blocks); their
outputs are compared pixel by pixel (within +-1 LSB; the fused and grouped
forms byte for byte against the plain one).

Lines printed (rank 0, one JSON line):
  value      frames/s of the faster form, device-resident (whole job over N ranks)
  paths      frames/s of both forms, their ratio and output agreement
  e2e        frames/s through the C ABI with host buffers (pinned), copies in
  roofline   the dominant kernel's algorithmic bytes / its CUDA-event time
  cpu_baseline  the reference plugin (built from its sources, oracle/_ref) on
             a bounded sample of the same workload on this host's cores
  kalman_4k10_bw48  the Kalman workload (60 frames 4K 10-bit YUV420, scene cut
             at frame 30, bt=0, bw=bh=48, ow=oh=16): frames/s and its frame roofline
``--impl reference`` times only the reference's CPU implementation.
Multi-GPU (torchrun): independent replicas, one clip per rank, no collective
on the data path ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import faulthandler
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from neo_fft3d_b200 import synth  # noqa: E402

WORKLOAD = "1080p_bt5_bw32"
METRIC = "1080p bt=5 frames/s: TC split-precision vs plain FP32 kernel at \u00b11 LSB; %HBM roofline"
UNIT = "frames/s"
# the two forms of the block transform that the metric compares (NEO_FFT3D_PATH)
PATHS = {"plain_fp32": "unfused", "plain_fp32_fused": "fused", "plain_fp32_frames": "unfused",
         "tc_split_bf16": "tc", "tc_split_bf16_frames": "tc"}
PLAIN = ("plain_fp32", "plain_fp32_fused", "plain_fp32_frames")
TC = ("tc_split_bf16", "tc_split_bf16_frames")
GROUPED = ("plain_fp32_frames", "tc_split_bf16_frames")
# output frames per call of the grouped arm (fft3d_plane_filter_frames_device)
FRAME_GROUP = 8


def workload():
    w = synth.WORKLOADS[WORKLOAD]
    return w["clip"], w["filt"]


def canonical_frame_bytes(width, height, nblocks_total, bh, nh, bt):
    """Cached-spectrum byte model per output frame: P_in + S + bt*S + P_out
    (P = pixel bytes of all planes, S = unpadded FP32 complex half-spectra of
    all blocks of all planes)."""
    P = width * height * 3 // 2
    S = nblocks_total * bh * nh * 8
    return P + S + bt * S + P


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic():
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        rows = [r.split(",") for r in out.strip().splitlines() if r.strip()]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# The reference plugin grows its per-thread scratch and its spectrum cache the
# first time more threads call it at once than before (src/fft3d_engine.h:
# 460-483): cache::resize appends to the cache's LRU list under
# thread_check_mutex while other threads reorder that list under cache_mutex
# (src/cache.hpp:34-71, src/fft3d_engine.h:647-667), and the scratch vectors
# it appends to are indexed after the lock is released (:481-483). That race
# can corrupt the heap while the thread count ramps up, so the reference is
# timed in a child process of its own: one filter node per process (as one
# script renders a clip), the ramp-up inside an untimed first render, and a
# fresh child if one dies by a signal.
REF_FIRST, REF_LAST = 10, 110  # frames rendered by the reference arm (the clip has 120)


def reference_child(args):
    """Child-process body of the reference measurement: one reference filter
    node over the 1080p bt=5 clip, an untimed ramp-up render of `threads`
    frames, then args.warmup untimed and args.steps timed renders of `frames`
    frames each (consecutive frame ranges, wrapping within the clip). Prints
    one JSON line with the per-step seconds."""
    from oracle import reference
    clip_kw, filt = workload()
    planes = synth.make_clip(**clip_kw)
    threads = args.ref_threads or os.cpu_count() or 1
    c = reference.core()
    clip = c.clip(planes)
    node = c.invoke("neo_fft3d", "FFT3D", clip, opt=0, ncpu=1, **filt)
    span = REF_LAST - REF_FIRST
    t = time.perf_counter()
    node.render(first=REF_FIRST, count=threads, threads=threads)
    per_frame = (time.perf_counter() - t) / threads
    frames = args.ref_frames or int(max(1, min(span, args.ref_budget / max(1, args.steps + args.warmup) / per_frame)))
    frames = min(frames, span)
    start = REF_FIRST + threads
    secs = []
    for i in range(args.warmup + args.steps):
        if start + frames > REF_LAST:
            start = REF_FIRST
        t = time.perf_counter()
        node.render(first=start, count=frames, threads=threads)
        if i >= args.warmup:
            secs.append(time.perf_counter() - t)
        start += frames
    print(json.dumps({"frames": frames, "threads": threads, "secs": secs, "ramp_up_s_per_frame": per_frame}),
          flush=True)


def run_reference_isolated(steps, warmup, frames=0, budget=150.0, threads=0, attempts=3):
    """reference_child in a fresh process (retried when a child dies by a
    signal); returns its result dict plus the number of attempts."""
    cmd = [sys.executable, os.path.abspath(__file__), "--impl", "reference", "--ref-child",
           "--steps", str(steps), "--warmup", str(warmup), "--ref-frames", str(frames),
           "--ref-budget", str(budget), "--ref-threads", str(threads)]
    env = dict(os.environ)
    env.pop("RANK", None)
    env.pop("WORLD_SIZE", None)
    err = ""
    for k in range(attempts):
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, env=env)
        lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
        if r.returncode == 0 and lines:
            out = json.loads(lines[-1])
            out["attempts"] = k + 1
            return out
        err = f"child rc {r.returncode}: {r.stderr.strip()[-300:]}"
        if r.returncode >= 0:
            break  # an error, not a crash: no retry
    raise RuntimeError(err)


def reference_arm(args, rank):
    if rank != 0:
        return None
    r = run_reference_isolated(args.steps, args.warmup)
    frames, threads, secs = r["frames"], r["threads"], r["secs"]
    total = sum(secs)
    fps = len(secs) * frames / total
    line = {
        "impl": "reference", "metric": METRIC, "value": fps, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total / len(secs),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "frames_per_step": frames, "opt": 0, "ncpu": 1, "host_threads": threads,
                   "child_attempts": r["attempts"]},
        "cpu_baseline": {"value": fps, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{frames} output frames (of 120) of the 1080p bt=5 clip per step, one filter "
                                   f"node, {threads} host threads (frame-parallel), opt=0, FFT = project FFTW-API shim"},
        "e2e": {"value": fps, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


def kalman_4k(args, torch, dist, engine, make_params, plane_descs, local, world, steps=3):
    """The Kalman workload: 60 frames of 3840x2160 10-bit YUV420 (noise sigma 12
    in 10-bit codes, scene cut at frame 30), bt=0, sigma=3, kratio=2,
    bw=bh=48, ow=oh=16; one step = the whole clip from frame 0 (state reset),
    planes on their own streams. Frame roofline: the minimal-state byte model
    2 P + 32 B per bin (pixels in and out; the spectrum's re/im and the
    Kalman state's last value and two covariances, read and written)."""
    F = 60
    planes = synth.make_clip_device(3840, 2160, F, bits=10, noise_sigma=12.0, seed=1002, scene_cut=30)
    p = make_params(sigma=3.0, bt=0, kratio=2.0, bw=48, bh=48, ow=16, oh=16)
    descs = plane_descs([tuple(a.shape[1:]) for a in planes], 10, F)
    engs = [engine.PlaneEngine(p, d, local) for d in descs]
    outs = [torch.empty_like(a) for a in planes]
    streams = [torch.cuda.Stream() for _ in engs]
    master = torch.cuda.current_stream()

    def step(group=0):
        ev = torch.cuda.Event()
        ev.record(master)
        for e, a, o, s in zip(engs, planes, outs, streams):
            s.wait_event(ev)
            e.reset()
            fb = a.shape[1] * a.shape[2] * 2
            st = a.shape[2] * 2
            if group:
                # frame groups: one forward and one overlap-add launch per group,
                # the Kalman filter/inverse per frame in order
                for n0 in range(0, F, group):
                    k = min(group, F - n0)
                    ptrs = [a.data_ptr() + n * fb if 0 <= n < F else 0 for n in range(n0 - 2, n0 + k + 2)]
                    e.filter_frames_device(n0, ptrs, [st] * (k + 4), [o.data_ptr() + n * fb for n in range(n0, n0 + k)],
                                           [st] * k, s.cuda_stream)
                continue
            for n in range(F):
                ptrs = [0, 0, a.data_ptr() + n * fb, 0, 0]
                e.filter_device(n, ptrs, [st] * 5, o.data_ptr() + n * fb, st, s.cuda_stream)
        for s in streams:
            master.wait_stream(s)

    def timed(group):
        step(group)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(master)
        for _ in range(steps):
            step(group)
        t1.record(master)
        torch.cuda.synchronize()
        ms = t0.elapsed_time(t1)
        if world > 1:
            tt = torch.tensor([ms], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ms = float(tt.item())
        return ms

    ms_frame = timed(0)
    ref = [o.clone() for o in outs]
    ms_group = timed(FRAME_GROUP)
    identical = all(bool(torch.equal(r, o)) for r, o in zip(ref, outs))
    fps_frame = world * F * steps / (ms_frame / 1000.0)
    fps_group = world * F * steps / (ms_group / 1000.0)
    ms = min(ms_frame, ms_group)
    fps = max(fps_frame, fps_group)
    P = sum(a[0].numel() * 2 for a in planes)
    bins = sum(e.nblocks * 48 * 25 for e in engs)
    fb = 2 * P + 32 * bins
    peak, kind = load_peaks()
    for e in engs:
        e.close()
    return {"value": fps, "unit": UNIT, "frames_per_step": F, "steps": steps, "ms_per_step": ms / steps,
            "config": {"width": 3840, "height": 2160, "format": "YUV420P10", "bt": 0, "sigma": 3.0, "kratio": 2.0,
                       "bw": 48, "bh": 48, "ow": 16, "oh": 16, "scene_cut": 30, "noise_sigma": 12},
            "frame_roofline": {"bytes_per_frame": fb, "achieved_gbs": fb * fps / world / 1e9,
                               "frac": fb * fps / world / 1e9 / peak, "peak_kind": kind},
            "paths": {"one_frame_per_call": fps_frame, f"frame_groups_of_{FRAME_GROUP}": fps_group,
                      "outputs_identical": identical}}


def main():
    faulthandler.enable()  # a native fault leaves its Python stack on stderr
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-kalman", action="store_true")
    # child process of the reference measurement (run_reference_isolated)
    ap.add_argument("--ref-child", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--ref-frames", type=int, default=0, help=argparse.SUPPRESS)
    ap.add_argument("--ref-budget", type=float, default=150.0, help=argparse.SUPPRESS)
    ap.add_argument("--ref-threads", type=int, default=0, help=argparse.SUPPRESS)
    ap.add_argument("--arms", default=",".join(PATHS),
                    help="comma-separated subset of the timed arms (profiling runs); the comparisons need all")
    args = ap.parse_args()
    if args.impl == "reference" and args.ref_child:
        reference_child(args)  # warm-up count as given (the ramp-up render is untimed anyway)
        return
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        # the reference is a CPU implementation: rank 0 runs it, others exit
        line = reference_arm(args, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    from neo_fft3d_b200 import engine
    from neo_fft3d_b200.params import make_params, plane_descs

    clip_kw, filt = workload()
    F = clip_kw["frames"]
    planes = synth.make_clip(**clip_kw)
    p = make_params(**filt)
    descs = plane_descs([a.shape[1:] for a in planes], 8, F)
    dev = [torch.from_numpy(a).cuda() for a in planes]
    master = torch.cuda.current_stream()

    def make_arm(path, group=0):
        os.environ["NEO_FFT3D_PATH"] = path
        engs = [engine.PlaneEngine(p, d, local) for d in descs]
        outs = [torch.empty_like(d) for d in dev]
        streams = [torch.cuda.Stream() for _ in engs]

        def frames(i, lo, hi, s):
            """Output frames [lo, hi) of plane i on stream s."""
            e, a, o = engs[i], dev[i], outs[i]
            W = a.shape[2]
            fb = a.shape[1] * W
            base = a.data_ptr()
            obase = o.data_ptr()
            if group:
                for n0 in range(lo, hi, group):
                    k = min(group, hi - n0)
                    ptrs = [base + n * fb if 0 <= n < F else 0 for n in range(n0 - 2, n0 + k + 2)]
                    e.filter_frames_device(n0, ptrs, [W] * (k + 4), [obase + n * fb for n in range(n0, n0 + k)],
                                           [W] * k, s.cuda_stream)
                return
            for n in range(lo, hi):
                ptrs = [base + (n + d) * fb if 0 <= n + d < F else 0 for d in range(-2, 3)]
                e.filter_device(n, ptrs, [W] * 5, obase + n * fb, W, s.cuda_stream)

        def step(serial=False):
            ev = torch.cuda.Event()
            ev.record(master)
            for i in range(len(engs)):
                s = master if serial else streams[i]
                s.wait_event(ev)
                frames(i, 0, F, s)
            for s in streams:
                master.wait_stream(s)

        return {"engs": engs, "outs": outs, "step": step, "frames": frames, "group": group}

    def time_arm(arm):
        for _ in range(args.warmup):
            arm["step"]()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        l0 = engine.kernel_launches()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0.record(master)
        for _ in range(args.steps):
            arm["step"]()
        t1.record(master)
        torch.cuda.synchronize()
        arm["launches"] = engine.kernel_launches() - l0
        ms = t0.elapsed_time(t1)
        if world > 1:
            tt = torch.tensor([ms], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ms = float(tt.item())
            dist.barrier()
        arm["ms"] = ms
        arm["value"] = world * F * args.steps / (ms / 1000.0)

    chosen = [a for a in args.arms.split(",") if a]
    for a in chosen:
        if a not in PATHS:
            raise SystemExit(f"unknown arm {a}; arms: {', '.join(PATHS)}")
    arms = {name: make_arm(path, FRAME_GROUP if name in GROUPED else 0)
            for name, path in PATHS.items() if name in chosen}
    os.environ["NEO_FFT3D_PATH"] = PATHS["plain_fp32"]
    clocks = ClockSampler(local)
    clocks.start()
    for arm in arms.values():
        time_arm(arm)
    clk = clocks.stop()
    head_name = max(arms, key=lambda k: arms[k]["value"])
    head = arms[head_name]
    engs = head["engs"]
    step = head["step"]
    value = head["value"]
    ms_per_step = head["ms"] / args.steps
    launches = head["launches"]
    paths = {name: {"value": arm["value"], "ms_per_step": arm["ms"] / args.steps, "launches": arm["launches"],
                    "NEO_FFT3D_PATH": PATHS[name]} for name, arm in arms.items()}
    if len(arms) == len(PATHS):
        # the two forms' outputs (the last step wrote every frame of every plane)
        diff_max, within, total_px = 0, 0, 0
        for a, b in zip(arms["plain_fp32"]["outs"], arms["tc_split_bf16"]["outs"]):
            d = (a.to(torch.int16) - b.to(torch.int16)).abs()
            diff_max = max(diff_max, int(d.max().item()))
            within += int((d <= 1).sum().item())
            total_px += d.numel()
        best_plain = max(arms[k]["value"] for k in PLAIN)
        paths["tc_over_plain"] = max(arms[k]["value"] for k in TC) / best_plain
        # the same schedule (frame groups of FRAME_GROUP) for both transforms
        paths["tc_frames_over_plain_frames"] = arms["tc_split_bf16_frames"]["value"] / arms["plain_fp32_frames"]["value"]
        paths["tc_frames_vs_tc_output_identical"] = all(
            bool(torch.equal(a, b)) for a, b in zip(arms["tc_split_bf16"]["outs"], arms["tc_split_bf16_frames"]["outs"]))
        # the fused sequence against the unfused one (same FP32 arithmetic)
        fd_max, fd_within = 0, 0
        for a, b in zip(arms["plain_fp32"]["outs"], arms["plain_fp32_fused"]["outs"]):
            d = (a.to(torch.int16) - b.to(torch.int16)).abs()
            fd_max = max(fd_max, int(d.max().item()))
            fd_within += int((d <= 1).sum().item())
        paths["fused_vs_unfused_output"] = {"within_1lsb": fd_within / total_px, "max_abs_diff": fd_max}
        # frame groups run the unfused kernels' arithmetic: byte-identical
        paths["frames_vs_unfused_output"] = {
            "identical": all(bool(torch.equal(a, b)) for a, b in zip(arms["plain_fp32"]["outs"],
                                                                       arms["plain_fp32_frames"]["outs"])),
            "frames_per_call": FRAME_GROUP}
        paths["tc_vs_plain_output"] = {"within_1lsb": within / total_px, "max_abs_diff": diff_max,
                                       "pixels": total_px}

    # per-kernel roofline from an instrumented pass (events around each
    # launch; planes serialised on one stream so that no other kernel shares
    # the GPU during a timed launch). The dominant kernel is taken on the luma
    # plane, whose launches are the largest.
    # Each chunk of frames is queued while the GPU waits in a sleep kernel, so
    # that the events around a launch bracket the kernel alone and not the
    # host's time to issue it.
    for e in engs:
        e.set_timing(True)
    chunk = max(head["group"], 1) * max(1, 8 // max(head["group"], 1))
    for _ in range(2):
        for i in range(len(engs)):
            for lo in range(0, F, chunk):
                torch.cuda._sleep(2_000_000)
                head["frames"](i, lo, min(lo + chunk, F), master)
            torch.cuda.synchronize()
    per_plane = [e.timing() for e in engs]
    for e in engs:
        e.set_timing(False)
    total_ms = {k: sum(pp[k][1] for pp in per_plane) for k in per_plane[0]}
    dom = max(total_ms, key=total_ms.get)
    n_l, ms_l, b_l = per_plane[0][dom]
    peak, peak_kind = load_peaks()
    achieved = (b_l / n_l) / (ms_l / n_l / 1000.0) / 1e9
    traffic = load_traffic().get(f"{dom}_frames{head['group']}" if head["group"] else dom)
    if isinstance(traffic, dict):
        # captured on one launch; scaled to the average launch by algorithmic bytes
        traffic = traffic["traffic"] * (b_l / n_l) / traffic["algorithmic"]
    share_den = sum(total_ms.values())
    roofline = {"bound": "hbm", "kernel": dom, "plane": "luma", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "traffic": traffic, "algorithmic_bytes_per_launch": b_l / n_l,
                "avg_launch_us": 1000.0 * ms_l / n_l,
                "kernel_share": {k: v / share_den for k, v in total_ms.items() if v > 0}}
    nblocks_total = sum(e.nblocks for e in engs)
    fb_bytes = canonical_frame_bytes(clip_kw["width"], clip_kw["height"], nblocks_total, p.bh, p.bw // 2 + 1, p.bt)
    frame_roofline = {"model": "cached spectra, one output frame at a time: P_in + S + bt*S + P_out",
                      "bytes_per_frame": fb_bytes, "achieved_gbs": fb_bytes * value / world / 1e9,
                      "frac": fb_bytes * value / world / 1e9 / peak}
    if head["group"]:
        # a frame group of G frames reads the G + bt - 1 window spectra once
        G = head["group"]
        S_all = nblocks_total * p.bh * (p.bw // 2 + 1) * 8
        gb = fb_bytes - p.bt * S_all + (G + p.bt - 1) / G * S_all
        frame_roofline["head_path_model"] = {
            "model": f"frame groups of {G}: P_in + S + (G + bt - 1)/G * S + P_out",
            "bytes_per_frame": gb, "achieved_gbs": gb * value / world / 1e9, "frac": gb * value / world / 1e9 / peak}

    # end to end through the C ABI with pinned host buffers (one host thread per plane)
    host_in = [torch.from_numpy(a).pin_memory() for a in planes]
    host_out = [torch.empty_like(h).pin_memory() for h in host_in]
    nps_in = [h.numpy() for h in host_in]
    nps_out = [h.numpy() for h in host_out]

    # each plane is served by E2E_THREADS host threads taking output frames
    # from a shared counter, as a frame-parallel VapourSynth filter is called;
    # the engine queues each call and overlaps its copies with other calls' kernels
    E2E_THREADS = 4

    G = head["group"]

    def e2e_plane(i, counter, lock):
        e, a, o = engs[i], nps_in[i], nps_out[i]
        while True:
            with lock:
                n = counter[0]
                counter[0] += max(G, 1)
            if n >= F:
                return
            if G:
                k = min(G, F - n)
                e.filter_frames(n, [a[m] if 0 <= m < F else None for m in range(n - 2, n + k + 2)],
                                [o[m] for m in range(n, n + k)])
                continue
            win = [a[n + d] if 0 <= n + d < F else None for d in range(-2, 3)]
            e.filter(n, win, o[n])

    def e2e_step():
        th = []
        for i, e in enumerate(engs):
            e.reset()
            counter, lock = [0], threading.Lock()
            th += [threading.Thread(target=e2e_plane, args=(i, counter, lock)) for _ in range(E2E_THREADS)]
        for t in th:
            t.start()
        for t in th:
            t.join()

    e2e = None
    if args.e2e_steps > 0:
        e2e_step()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step()
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t
        if world > 1:
            tt = torch.tensor([e2e_s], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            e2e_s = float(tt.item())
        frame_bytes = sum(a[0].nbytes for a in planes)
        e2e = {"value": world * F * args.e2e_steps / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": F * frame_bytes, "d2h_bytes_per_step": F * frame_bytes,
               "path": (f"fft3d_plane_filter_frames (host API, groups of {G} frames)" if G else
                        "fft3d_plane_filter (host API)") +
                       f", {E2E_THREADS} host threads per plane (frame-parallel), pinned buffers"}

    kalman = None if args.no_kalman else kalman_4k(args, torch, dist, engine, make_params, plane_descs, local, world)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # in a child process (see reference_child): the reference cannot take
        # this process and its GPU record down with it
        try:
            threads = os.cpu_count() or 1
            r = run_reference_isolated(steps=1, warmup=0, frames=2 * threads, threads=threads)
            sample, secs = r["frames"], sum(r["secs"])
            cpu = {"value": sample / secs, "unit": UNIT, "cores": r["threads"], "kind": "reference",
                   "sample": f"{sample} output frames of the same clip after a ramp-up render of {threads}, "
                             f"one filter node, {r['threads']} host threads, opt=0, ncpu=1, "
                             f"FFT = project FFTW-API shim (child attempts: {r['attempts']})"}
        except Exception as ex:  # the reference build is optional on a box
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"unavailable: {ex}"}

    if world > 1:
        dist.barrier()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "frames_per_step": F, "width": 1920, "height": 1080,
                       "format": "YUV420P8", "bt": 5, "sigma": 3.0, "bw": 32, "bh": 32, "ow": 16, "oh": 16,
                       "sharpen": 0.3, "path": head_name, "frames_per_call": head["group"] or 1,
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (373 MB clip + ~350 MB spectrum ring per rank), no flush"},
            "roofline": roofline, "frame_roofline": frame_roofline, "cpu_baseline": cpu, "e2e": e2e,
            "clocks": clk, "gpu_launches": launches, "paths": paths, "kalman_4k10_bw48": kalman,
        }
        print(json.dumps(line), flush=True)
    for arm in arms.values():
        for e in arm["engs"]:
            e.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
