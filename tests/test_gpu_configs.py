"""Parity on the benchmark configurations, at their full frame sizes.

The GPU path (through the C ABI) against the oracle: its float mode (the
reference's C path, opt=1, reproduced bit for bit given the same FFT) and its
FP64 mode (the truth the errors are stated against). For each configuration
and each form of the block transform:

* output pixels within +-1 LSB of the float oracle (bar: >= 99.9 %) and the
  largest difference;
* the same against the FP64 oracle (and, for scale, the float oracle itself
  against FP64);
* the per-block relative spectrum error max |X - X64| / max |X64| of the
  GPU's forward transform against the FP64 oracle's (bar: <= 1e-4).

Configurations (seeded synthetic clips of the benchmark shapes):
  0  640x480 8-bit YUV420, bt=3, sigma=2, bw=bh=48, ow=oh=16, frames 0..7 of 30
  1  1920x1080 8-bit YUV420, bt=5, sigma=3, bw=bh=32, ow=oh=16, sharpen=0.3:
     frames 0,1,2,3,7,8,9 of a 10-frame clip (both clip edges, where bt
     drops to 1, and the interior), plain FP32 and tensor-core split BF16
  2  3840x2160 10-bit YUV420, Kalman bt=0, sigma=3, kratio=2, bw=bh=48,
     ow=oh=16, scene cut at frame 30: frames 0..33 (the Kalman state runs
     from frame 0), statistics over frames 27..33 across the cut

With NEO_FFT3D_PARITY_REPORT=<file>, every measured figure is appended to that
file as one JSON line per configuration and form.
"""
import json
import os
import threading

import numpy as np
import pytest

from neo_fft3d_b200 import engine, synth
from neo_fft3d_b200.params import make_params, plane_descs
from oracle import restate

PIX_TOL_FRAC = 0.999  # fraction of output pixels within +-1 LSB of the float oracle
SPEC_TOL = 1e-4       # max per-block relative spectrum error against FP64

CONFIGS = {
    "cfg0_640x480_bt3_bw48": dict(
        clip=dict(width=640, height=480, frames=30, bits=8, noise_sigma=4.0, seed=1000),
        filt=dict(sigma=2.0, bt=3, bw=48, bh=48, ow=16, oh=16), frames=list(range(8)), stats=None, spec_frame=4),
    "cfg1_1080p_bt5_bw32": dict(
        clip=dict(width=1920, height=1080, frames=10, bits=8, noise_sigma=6.0, seed=1001),
        filt=dict(sigma=3.0, bt=5, bw=32, bh=32, ow=16, oh=16, sharpen=0.3), frames=[0, 1, 2, 3, 7, 8, 9],
        stats=None, spec_frame=5),
    "cfg2_4k10_kalman_bw48": dict(
        clip=dict(width=3840, height=2160, frames=34, bits=10, noise_sigma=12.0, seed=1002, scene_cut=30),
        filt=dict(sigma=3.0, bt=0, kratio=2.0, bw=48, bh=48, ow=16, oh=16), frames=list(range(34)),
        stats=list(range(27, 34)), spec_frame=31),
}
FORMS = [("cfg0_640x480_bt3_bw48", "plain_fp32"), ("cfg1_1080p_bt5_bw32", "plain_fp32"),
         ("cfg1_1080p_bt5_bw32", "tc_split_bf16"), ("cfg2_4k10_kalman_bw48", "plain_fp32")]

_clips = {}
_oracle = {}


def _clip(name):
    if name not in _clips:
        _clips[name] = synth.make_clip(**CONFIGS[name]["clip"])
    return _clips[name]


def _run_oracle_plane(planes, i, cfg, dbl):
    p = make_params(**cfg["filt"])
    d = plane_descs([a.shape[1:] for a in planes], cfg["clip"]["bits"], planes[0].shape[0])[i]
    eng = restate.OraclePlane(p, d, dbl)
    a = planes[i]
    o = np.empty((len(cfg["frames"]),) + a.shape[1:], a.dtype)
    for j, n in enumerate(cfg["frames"]):
        eng.filter(n, restate.window_of(a, n), o[j])
    return o


def _oracle_planes(name, dbl):
    """Oracle outputs of the configuration's frames: float and FP64 modes of
    every plane at once, one thread each (the restatement releases the GIL
    inside its C++ calls)."""
    if (name, dbl) not in _oracle:
        cfg = CONFIGS[name]
        planes = _clip(name)
        outs = {}

        def run(i, mode):
            outs[(i, mode)] = _run_oracle_plane(planes, i, cfg, mode)

        th = [threading.Thread(target=run, args=(i, mode)) for i in range(len(planes)) for mode in (False, True)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        for mode in (False, True):
            _oracle[(name, mode)] = [outs[(i, mode)] for i in range(len(planes))]
    return _oracle[(name, dbl)]


def _gpu_planes(name, form):
    """GPU outputs of the configuration's frames (host-buffer C ABI, one
    engine per plane, frames in order) and each plane's spectrum of
    spec_frame as the GPU's forward transform computed it."""
    cfg = CONFIGS[name]
    planes = _clip(name)
    p = make_params(**cfg["filt"])
    descs = plane_descs([a.shape[1:] for a in planes], cfg["clip"]["bits"], planes[0].shape[0])
    old = os.environ.get("NEO_FFT3D_PATH")
    os.environ["NEO_FFT3D_PATH"] = "tc" if form == "tc_split_bf16" else "unfused"
    try:
        outs, specs = [], []
        for i, a in enumerate(planes):
            eng = engine.PlaneEngine(p, descs[i])
            o = np.empty((len(cfg["frames"]),) + a.shape[1:], a.dtype)
            for j, n in enumerate(cfg["frames"]):
                eng.filter(n, [a[n + d] if 0 <= n + d < a.shape[0] else None for d in range(-2, 3)], o[j])
            # the spectrum of spec_frame: filtered alone (bt=1 window) by a fresh engine
            e1 = engine.PlaneEngine(make_params(**dict(cfg["filt"], bt=1)), descs[i])
            tmp = np.empty_like(a[0])
            e1.filter(cfg["spec_frame"], [None, None, a[cfg["spec_frame"]], None, None], tmp)
            specs.append(e1.spectrum(cfg["spec_frame"]))
            e1.close()
            eng.close()
            outs.append(o)
    finally:
        if old is None:
            os.environ.pop("NEO_FFT3D_PATH", None)
        else:
            os.environ["NEO_FFT3D_PATH"] = old
    return outs, specs


def _px_stats(got, want, sel):
    d = np.abs(got[sel].astype(np.int64) - want[sel].astype(np.int64))
    return float((d <= 1).mean()), int(d.max())


def _spec_err(name, planes, i, got):
    cfg = CONFIGS[name]
    p = make_params(**dict(cfg["filt"], bt=1))
    d = plane_descs([a.shape[1:] for a in planes], cfg["clip"]["bits"], planes[0].shape[0])[i]
    ref = restate.OraclePlane(p, d, dbl=True).spectrum(planes[i][cfg["spec_frame"]])
    num = np.abs(got - ref).reshape(got.shape[0], -1).max(1)
    den = np.abs(ref).reshape(ref.shape[0], -1).max(1)
    return float((num / den).max())


@pytest.mark.gpu
@pytest.mark.parametrize("name,form", FORMS, ids=[f"{n}-{f}" for n, f in FORMS])
def test_config_parity(gpu, name, form):
    cfg = CONFIGS[name]
    planes = _clip(name)
    want = _oracle_planes(name, False)
    want64 = _oracle_planes(name, True)
    got, specs = _gpu_planes(name, form)
    frames = cfg["frames"]
    sel = [frames.index(n) for n in cfg["stats"]] if cfg["stats"] else list(range(len(frames)))
    report = {"config": name, "form": form, "frames": [frames[j] for j in sel], "planes": []}
    for i in range(len(planes)):
        frac, mx = _px_stats(got[i], want[i], sel)
        frac64, mx64 = _px_stats(got[i], want64[i], sel)
        ref_frac64, ref_mx64 = _px_stats(want[i], want64[i], sel)
        err = _spec_err(name, planes, i, specs[i])
        report["planes"].append(dict(plane=i, within_1lsb=frac, max_abs_diff=mx, within_1lsb_vs_fp64=frac64,
                                     max_abs_diff_vs_fp64=mx64, reference_c_within_1lsb_vs_fp64=ref_frac64,
                                     reference_c_max_abs_diff_vs_fp64=ref_mx64, max_rel_spectrum_err_vs_fp64=err))
    path = os.environ.get("NEO_FFT3D_PARITY_REPORT")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(report) + "\n")
    for pl in report["planes"]:
        assert pl["within_1lsb"] >= PIX_TOL_FRAC, (name, form, pl)
        assert pl["max_rel_spectrum_err_vs_fp64"] <= SPEC_TOL, (name, form, pl)
