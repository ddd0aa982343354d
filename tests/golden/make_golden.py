"""Generate the golden fixtures of tests/golden from the REFERENCE plugin.

The reference (neo_fft3d) ships no tests, golden vectors or fixtures, so its
own outputs pin parity: this script renders small seeded synthetic clips
through the unmodified reference plugin (built from its sources by
``make -C oracle ref``, run through the headless VapourSynth host with the C
path, opt=1, behind the project's FFTW-API shim) and stores inputs, parameters
and outputs in ``golden.npz``.

Run from the repository root (needs the reference sources to have been built
into oracle/_ref):
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from neo_fft3d_b200 import synth  # noqa: E402

# Sizes are chosen so that no plane hits the reference's undefined mirror
# padding: its bottom mirror (src/buffer.cpp:65-71) reads cover rows that are
# only written afterwards when 2*H + (bh-oh) - 1 < cover height, i.e. for
# planes not much taller than one block step (it then reads stale memory and
# is not reproducible run to run).
CLIP8 = dict(width=128, height=96, frames=6, bits=8, noise_sigma=5.0, seed=501)
CLIP10 = dict(width=128, height=96, frames=5, bits=10, noise_sigma=12.0, seed=502)

CASES = [
    ("wiener3_default", "clip8", dict(sigma=2.0, bt=3)),
    ("wiener5_sharpen", "clip8", dict(sigma=3.0, bt=5, bw=32, bh=32, ow=16, oh=16, sharpen=0.3)),
    ("wiener2d", "clip8", dict(sigma=2.0, bt=1)),
    ("wiener2_dehalo", "clip8", dict(sigma=3.0, bt=2, dehalo=1.0)),
    ("wiener4_sharpen_dehalo", "clip8", dict(sigma=3.0, bt=4, sharpen=0.5, dehalo=0.7)),
    ("kalman", "clip8", dict(sigma=3.0, bt=0)),
    ("sharpen_only", "clip8", dict(sigma=3.0, bt=-1, sharpen=0.5)),
    ("wiener3_bw48", "clip8", dict(sigma=2.0, bt=3, bw=48, bh=48, ow=16, oh=16)),
    ("sigma_pattern", "clip8", dict(sigma=2.0, bt=3, sigma2=3.0, sigma3=4.0, sigma4=5.0)),
    ("degrid0", "clip8", dict(sigma=2.0, bt=1, degrid=0.0)),
    ("wintype1", "clip8", dict(sigma=2.0, bt=3, wintype=1)),
    ("wintype2_beta", "clip8", dict(sigma=2.0, bt=3, wintype=2, beta=1.5)),
    ("rect16x24", "clip8", dict(sigma=2.0, bt=3, bw=16, bh=24, ow=4, oh=6)),
    ("crop", "clip8", dict(sigma=2.0, bt=3, l=8, t=6, r=10, b=4)),
    ("interlaced", "clip8", dict(sigma=2.0, bt=3, interlaced=1)),
    ("kalman10_bw48", "clip10", dict(sigma=3.0, bt=0, kratio=2.0, bw=48, bh=48, ow=16, oh=16)),
    ("wiener3_10bit", "clip10", dict(sigma=3.0, bt=3)),
]


def main():
    from oracle import reference
    clips = {"clip8": synth.make_clip(**CLIP8), "clip10": synth.make_clip(**CLIP10)}
    arrays = {}
    for name, planes in clips.items():
        for i, p in enumerate(planes):
            arrays[f"{name}_in{i}"] = p
    meta = {"clips": {"clip8": CLIP8, "clip10": CLIP10}, "cases": []}
    for name, clip, kw in CASES:
        bits = CLIP8["bits"] if clip == "clip8" else CLIP10["bits"]
        out = reference.run(clips[clip], opt=1, bits=bits, **kw)
        for i, p in enumerate(out):  # stored as output - input (small values, compresses well)
            arrays[f"{name}_diff{i}"] = (p.astype(np.int32) - clips[clip][i].astype(np.int32)).astype(np.int16)
        meta["cases"].append({"name": name, "clip": clip, "bits": bits, "params": kw})
        print(name, [int(np.abs(o.astype(int) - c.astype(int)).mean() * 100) / 100 for o, c in zip(out, clips[clip])])
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **arrays)


if __name__ == "__main__":
    main()
