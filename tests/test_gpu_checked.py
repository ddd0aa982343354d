"""The bounds-checked build of the library (lib/libfft3d_b200_checked.so, `make
-C neo_fft3d_b200 checked`): every guarded global access of the default
path's kernels (forward gather and spectrum stores, filter/inverse and
frame-group loads and time-domain stores, overlap-add reads and writes) is
checked against its buffer, and a failed check skips the access and sets a
device error bit that the call reports.

A child process runs small clips through the checked library -- every filter
mode, several block sizes, crop, interlacing, 10-bit and float samples, one
frame per call and frame groups -- and must finish without a reported check;
its outputs must equal the regular library's byte for byte.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from neo_fft3d_b200 import engine, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECKED = os.path.join(ROOT, "neo_fft3d_b200", "lib", "libfft3d_b200_checked.so")

CASES = [
    ("wiener5_sharpen", 8, dict(sigma=3.0, bt=5, bw=32, bh=32, ow=16, oh=16, sharpen=0.3)),
    ("wiener3_bw48", 8, dict(sigma=2.0, bt=3, bw=48, bh=48, ow=16, oh=16)),
    ("wiener2_dehalo", 8, dict(sigma=3.0, bt=2, dehalo=1.0)),
    ("wiener4_rect", 8, dict(sigma=2.0, bt=4, bw=16, bh=24, ow=4, oh=6, sharpen=0.5)),
    ("wiener2d", 8, dict(sigma=2.0, bt=1, bw=24, bh=24, ow=8, oh=8)),
    ("kalman", 10, dict(sigma=3.0, bt=0, bw=48, bh=48, ow=16, oh=16)),
    ("sharpen_only", 8, dict(sigma=3.0, bt=-1, sharpen=0.5, bw=8, bh=8, ow=2, oh=2)),
    ("crop", 8, dict(sigma=2.0, bt=3, l=8, t=6, r=10, b=4)),
    ("interlaced", 8, dict(sigma=2.0, bt=3, interlaced=1)),
    ("float", 32, dict(sigma=2.0, bt=3, bw=12, bh=12, ow=4, oh=4)),
]


def _clip(bits):
    if bits == 32:
        return [a.astype(np.float32) / 255.0 for a in synth.make_clip(152, 96, 9, noise_sigma=5, seed=81)]
    return synth.make_clip(152, 96, 9, bits=bits, noise_sigma=5 << (bits - 8), seed=80 + bits)


def _run_all():
    """Every case one frame per call, and the Wiener/Kalman cases also in frame
    groups of 4 (host-buffer C ABI); returns {name: [planes]}."""
    out = {}
    for name, bits, kw in CASES:
        planes = _clip(bits)
        out[name] = engine.filter_clip(planes, bits=bits, **kw)
        if kw.get("bt", 3) >= 0 and not kw.get("l"):
            from neo_fft3d_b200.params import make_params, plane_descs
            F = planes[0].shape[0]
            p = make_params(**kw)
            descs = plane_descs([a.shape[1:] for a in planes], bits, F)
            grp = []
            for a, d in zip(planes, descs):
                e = engine.PlaneEngine(p, d)
                o = np.empty_like(a)
                for n0 in range(0, F, 4):
                    k = min(4, F - n0)
                    e.filter_frames(n0, [a[m] if 0 <= m < F else None for m in range(n0 - 2, n0 + k + 2)],
                                    [o[m] for m in range(n0, n0 + k)])
                e.close()
                grp.append(o)
            out[name + "_groups"] = grp
    return out


def _child(path):
    res = _run_all()
    np.savez(path, **{f"{k}__{i}": a for k, planes in res.items() for i, a in enumerate(planes)})


@pytest.mark.gpu
def test_checked_build_reports_nothing_and_matches(gpu, tmp_path):
    if not os.path.exists(CHECKED):
        pytest.skip("checked library not built (make -C neo_fft3d_b200 checked)")
    out = tmp_path / "checked.npz"
    env = dict(os.environ, NEO_FFT3D_LIB=CHECKED, PYTHONPATH=ROOT)
    r = subprocess.run([sys.executable, "-c", f"import tests.test_gpu_checked as t; t._child({str(out)!r})"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    got = np.load(out)
    want = _run_all()
    for k, planes in want.items():
        for i, a in enumerate(planes):
            assert np.array_equal(got[f"{k}__{i}"], a), (k, i)
