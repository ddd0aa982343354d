"""Seeded synthetic YUV clips with the shapes of the benchmark workloads.

No public dataset is involved: every workload is a seeded smooth field (a sum of
64 random 2D sinusoids, periods 8-200 px, random orientation and phase) that
moves by a seeded sub-pixel translation of at most 2 px per frame, evaluated
analytically (no resampling), scaled to the legal range of the format, plus
i.i.d. Gaussian noise, then rounded and clipped. The same seed gives the same
bytes on every machine (numpy PCG64).

A clip is returned as a list of planes, each an array [frames, height, width]
of uint8 (8-bit) or uint16 (9..16-bit), plus ``clean`` planes without noise.
"""
from __future__ import annotations

import numpy as np

N_SINES = 64


def _field_params(rng: np.random.Generator):
    period = rng.uniform(8.0, 200.0, N_SINES)
    theta = rng.uniform(0.0, np.pi, N_SINES)
    phase = rng.uniform(0.0, 2 * np.pi, N_SINES)
    amp = rng.uniform(0.5, 1.0, N_SINES)
    fx = np.cos(theta) / period
    fy = np.sin(theta) / period
    return fx, fy, phase, amp


def _eval_field(params, width, height, dx, dy, scale):
    """sum_k amp_k sin(2 pi (fx_k (x-dx) + fy_k (y-dy)) + phase_k), evaluated as
    two rank-64 products: sin(a+b) = sin a cos b + cos a sin b."""
    fx, fy, phase, amp = params
    x = (np.arange(width, dtype=np.float64) * scale - dx)[:, None]
    y = (np.arange(height, dtype=np.float64) * scale - dy)[:, None]
    ax = 2 * np.pi * x * fx[None, :]
    by = 2 * np.pi * y * fy[None, :] + phase[None, :]
    sx, cx = np.sin(ax), np.cos(ax)
    sy, cy = np.sin(by) * amp, np.cos(by) * amp
    return sy @ cx.T + cy @ sx.T  # [height, width]


def make_clip(width: int, height: int, frames: int, *, bits: int = 8, noise_sigma: float = 4.0,
              seed: int = 0, ssw: int = 1, ssh: int = 1, scene_cut: int | None = None,
              planes: int = 3, with_clean: bool = False):
    """Seeded synthetic clip. ``noise_sigma`` is in units of the format's code
    values (e.g. 12 for 12 codes of a 10-bit clip). Luma is scaled to 16..235
    (8-bit; 64..940 for 10-bit), chroma to 16..240 (64..960), i.e. the same
    ranges shifted by bits-8."""
    dtype = np.uint8 if bits <= 8 else np.uint16
    shift = bits - 8
    maxv = (1 << bits) - 1
    rng_motion = np.random.default_rng([seed, 1])
    steps = rng_motion.uniform(-2.0, 2.0, size=(frames, 2))
    steps[0] = 0.0
    path = np.cumsum(steps, axis=0)
    out, clean_out = [], []
    for p in range(planes):
        w = width >> ssw if p else width
        h = height >> ssh if p else height
        scale = float(1 << ssw) if p else 1.0
        lo, hi = (16 << shift, (235 if p == 0 else 240) << shift)
        arr = np.empty((frames, h, w), dtype)
        carr = np.empty((frames, h, w), dtype) if with_clean else None
        noise_rng = np.random.default_rng([seed, 100 + p])
        seg_seed = seed
        params = _field_params(np.random.default_rng([seg_seed, 10 + p]))
        f0 = _eval_field(params, w, h, 0.0, 0.0, scale)
        fmin, fmax = f0.min(), f0.max()
        for t in range(frames):
            if scene_cut is not None and t == scene_cut:
                seg_seed = seed + 7919
                params = _field_params(np.random.default_rng([seg_seed, 10 + p]))
                f0 = _eval_field(params, w, h, 0.0, 0.0, scale)
                fmin, fmax = f0.min(), f0.max()
            dx, dy = path[t]
            f = _eval_field(params, w, h, dx, dy, scale)
            v = lo + (f - fmin) * ((hi - lo) / (fmax - fmin))
            if with_clean:
                carr[t] = np.clip(np.rint(v), 0, maxv).astype(dtype)
            if noise_sigma > 0:
                v = v + noise_rng.standard_normal((h, w), dtype=np.float32) * np.float32(noise_sigma)
            arr[t] = np.clip(np.rint(v), 0, maxv).astype(dtype)
        out.append(arr)
        if with_clean:
            clean_out.append(carr)
    return (out, clean_out) if with_clean else out


def make_clip_device(width: int, height: int, frames: int, *, bits: int = 8, noise_sigma: float = 4.0, seed: int = 0,
                     ssw: int = 1, ssh: int = 1, scene_cut: int | None = None, planes: int = 3):
    """make_clip's clip evaluated on the GPU (torch, FP64 field, device RNG for
    the noise): the same field, motion and scaling, for workloads too large to
    generate on the host quickly. Returns a list of CUDA tensors [F, H, W],
    uint8 for 8-bit and int16 (same bit patterns as uint16) for 9..15-bit."""
    import math

    import torch
    shift = bits - 8
    maxv = (1 << bits) - 1
    rng_motion = np.random.default_rng([seed, 1])
    steps = rng_motion.uniform(-2.0, 2.0, size=(frames, 2))
    steps[0] = 0.0
    path = np.cumsum(steps, axis=0)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    dtype = torch.uint8 if bits <= 8 else torch.int16
    out = []
    for p in range(planes):
        w = width >> ssw if p else width
        h = height >> ssh if p else height
        scale = float(1 << ssw) if p else 1.0
        lo, hi = 16 << shift, (235 if p == 0 else 240) << shift

        def params(s):
            return [torch.tensor(v, device="cuda", dtype=torch.float64)
                    for v in _field_params(np.random.default_rng([s, 10 + p]))]

        def field(prm, dx, dy):
            fx, fy, phase, amp = prm
            x = torch.arange(w, device="cuda", dtype=torch.float64) * scale - dx
            y = torch.arange(h, device="cuda", dtype=torch.float64) * scale - dy
            ax = 2 * math.pi * x[:, None] * fx[None, :]
            by = 2 * math.pi * y[:, None] * fy[None, :] + phase[None, :]
            return (torch.sin(by) * amp) @ torch.cos(ax).T + (torch.cos(by) * amp) @ torch.sin(ax).T

        prm = params(seed)
        f0 = field(prm, 0.0, 0.0)
        fmin, fmax = f0.min(), f0.max()
        arr = torch.empty((frames, h, w), dtype=dtype, device="cuda")
        for t in range(frames):
            if scene_cut is not None and t == scene_cut:
                prm = params(seed + 7919)
                f0 = field(prm, 0.0, 0.0)
                fmin, fmax = f0.min(), f0.max()
            v = lo + (field(prm, float(path[t][0]), float(path[t][1])) - fmin) * ((hi - lo) / (fmax - fmin))
            if noise_sigma > 0:
                v = v + torch.randn((h, w), generator=gen, device="cuda", dtype=torch.float64) * noise_sigma
            arr[t] = torch.clamp(torch.round(v), 0, maxv).to(dtype)
        out.append(arr)
    return out


def pack(planes) -> np.ndarray:
    """Pack a clip (list of [F,H,W] planes) into one contiguous byte buffer:
    frame after frame, planes in order, rows without padding."""
    frames = planes[0].shape[0]
    per = [p.reshape(frames, -1).view(np.uint8) for p in planes]
    return np.ascontiguousarray(np.concatenate(per, axis=1)).reshape(-1)


def unpack(buf: np.ndarray, like) -> list:
    """Inverse of :func:`pack` for planes shaped like ``like`` (list of arrays or shapes)."""
    shapes = [(p.shape, p.dtype) if hasattr(p, "shape") else p for p in like]
    frames = shapes[0][0][0]
    row = buf.reshape(frames, -1)
    out, off = [], 0
    for shape, dtype in shapes:
        nb = int(np.prod(shape[1:])) * np.dtype(dtype).itemsize
        out.append(np.ascontiguousarray(row[:, off:off + nb]).view(dtype).reshape(shape))
        off += nb
    return out


# The benchmark workloads, by name.
WORKLOADS = {
    # 30 frames 640x480 8-bit YUV420, sigma_noise 4; filter sigma=2, bt=3, bw=bh=48, ow=oh=16
    "small_640x480_bt3_bw48": dict(clip=dict(width=640, height=480, frames=30, bits=8, noise_sigma=4.0, seed=1000),
                                   filt=dict(sigma=2.0, bt=3, bw=48, bh=48, ow=16, oh=16, sharpen=0.0)),
    # 120 frames 1080p 8-bit YUV420, sigma_noise 6; filter sigma=3, bt=5, bw=bh=32, ow=oh=16, sharpen=0.3
    "1080p_bt5_bw32": dict(clip=dict(width=1920, height=1080, frames=120, bits=8, noise_sigma=6.0, seed=1001),
                           filt=dict(sigma=3.0, bt=5, bw=32, bh=32, ow=16, oh=16, sharpen=0.3)),
    # 60 frames 4K 10-bit YUV420 in uint16, scene cut at 30, sigma_noise 12; Kalman bt=0
    "4k10_kalman_bw48": dict(clip=dict(width=3840, height=2160, frames=60, bits=10, noise_sigma=12.0, seed=1002,
                                       scene_cut=30),
                             filt=dict(sigma=3.0, bt=0, kratio=2.0, bw=48, bh=48, ow=16, oh=16)),
}


# ---------------------------------------------------------------- coloured noise
# Noise of the learned-PSD workload: white Gaussian noise shaped by a 16x16 FIR
# whose frequency response samples a radially symmetric transfer function, a
# monotone cubic (Fritsch-Carlson) spline through 4 knot amplitudes at
# normalised radius 0, 1/3, 2/3, 1 (radius 1 = 0.5 cycles per pixel), scaled
# to a total standard deviation sigma. The same process family trains the
# model (on the GPU, per block) and makes the evaluation clips (here, per frame).

FIR_TAPS = 16


def _spline(v, r):
    v = np.asarray(v, np.float64)
    dl = (v[1:] - v[:-1]) * 3.0
    m = np.array([dl[0], 0.0, 0.0, dl[2]])
    for k in (1, 2):
        m[k] = 0.0 if dl[k - 1] * dl[k] <= 0 else 0.5 * (dl[k - 1] + dl[k])
    for k in range(3):
        if dl[k] == 0:
            m[k] = m[k + 1] = 0.0
        else:
            a, b = m[k] / dl[k], m[k + 1] / dl[k]
            if a * a + b * b > 9.0:
                tau = 3.0 / np.sqrt(a * a + b * b)
                m[k], m[k + 1] = tau * a * dl[k], tau * b * dl[k]
    i = np.minimum(2, (r * 3.0).astype(int))
    t = (r - i / 3.0) * 3.0
    return ((2 * t ** 3 - 3 * t ** 2 + 1) * v[i] + (t ** 3 - 2 * t ** 2 + t) / 3.0 * m[i]
            + (-2 * t ** 3 + 3 * t ** 2) * v[i + 1] + (t ** 3 - t ** 2) / 3.0 * m[i + 1])


def noise_fir(knots) -> np.ndarray:
    """Centred 16x16 FIR (tap [a][b] at lag (a-8, b-8)) of the transfer
    function with the given 4 monotone knot amplitudes."""
    n = FIR_TAPS
    f = np.array([(i if i <= n // 2 else i - n) / n for i in range(n)])
    r = np.minimum(1.0, 2.0 * np.sqrt(f[:, None] ** 2 + f[None, :] ** 2))
    h = np.real(np.fft.ifft2(_spline(knots, r)))
    return np.roll(h, (n // 2, n // 2), axis=(0, 1))


def coloured_noise(frames: int, height: int, width: int, knots, sigma: float, seed: int = 0) -> np.ndarray:
    """[frames, height, width] float64 coloured noise of total std sigma."""
    from scipy.signal import correlate
    h = noise_fir(knots)
    gain = sigma / np.sqrt(np.sum(h * h))
    rng = np.random.default_rng([seed, 300])
    out = np.empty((frames, height, width))
    for t in range(frames):
        w = rng.standard_normal((height + FIR_TAPS - 1, width + FIR_TAPS - 1))
        out[t] = gain * correlate(w, h, mode="valid", method="fft")
    return out


def make_coloured_clip(width: int, height: int, frames: int, knots, sigma: float, seed: int = 0):
    """Luma-only 8-bit clip of the sinusoid field (as make_clip) plus coloured
    noise; returns (noisy, clean) uint8 arrays [frames, height, width]."""
    v = _field_values(width, height, frames, seed)
    noisy = np.clip(np.rint(v + coloured_noise(frames, height, width, knots, sigma, seed)), 0, 255).astype(np.uint8)
    return noisy, np.clip(np.rint(v), 0, 255).astype(np.uint8)


def _field_values(width: int, height: int, frames: int, seed: int) -> np.ndarray:
    """Unrounded luma values of make_clip's field (no noise)."""
    rng_motion = np.random.default_rng([seed, 1])
    steps = rng_motion.uniform(-2.0, 2.0, size=(frames, 2))
    steps[0] = 0.0
    path = np.cumsum(steps, axis=0)
    params = _field_params(np.random.default_rng([seed, 10]))
    f0 = _eval_field(params, width, height, 0.0, 0.0, 1.0)
    fmin, fmax = f0.min(), f0.max()
    out = np.empty((frames, height, width))
    for t in range(frames):
        f = _eval_field(params, width, height, path[t][0], path[t][1], 1.0)
        out[t] = 16 + (f - fmin) * ((235 - 16) / (fmax - fmin))
    return out


def psnr(a: np.ndarray, b: np.ndarray, peak: float = 255.0) -> float:
    d = a.astype(np.float64) - b.astype(np.float64)
    return float(10 * np.log10(peak * peak / np.mean(d * d)))
