"""FP64 CPU restatement of the learned noise-PSD model: its block generator and
its 3-layer MLP with forward and backward passes.

TEST INFRASTRUCTURE ONLY: this module is the checker of the device code in
neo_fft3d_b200/csrc/fft3d_psd.cu (generator, features, targets) and
neo_fft3d_b200/csrc/mlp_kernels.cu (GEMM, GELU, loss, gradients). Only tests/
may import it. The model has no counterpart in the reference; what it plugs
into is the reference's noise pattern slot (pattern2d, and pattern3d =
bt x pattern2d, src/helper.cpp:171-178, src/fft3d_engine.h:625-630), whose
units (|X|^2 of the windowed, unnormalised block FFT) the targets use.

Everything here follows the device code's definitions:
  * counter-based random numbers: the SplitMix64 finaliser over
    (seed, stream, index); 24-bit uniforms; Box-Muller normals;
  * clean frames: 64 sinusoids per frame, scaled to 16..235 by the frame's
    min / max;
  * per block: total sigma, 4 knot amplitudes (log-uniform in [span, 1], the
    span log-uniform in [knot_min, 1]), falling or rising, frame and position;
    a monotone (Fritsch-Carlson) cubic spline over normalised radius,
    sampled on a 16x16 frequency grid and inverted to a centred 16x16 FIR; noise = gain * (FIR correlated with white noise), gain
    = sigma / sqrt(sum FIR^2);
  * features: (log(|X|^2 + 1) - 8) * 0.4 of the windowed 8-bit block, DC and
    padding 0, rounded to BF16;
  * targets: log(sum_d R(d) A(d) cos(k.d) + sum(window^2) / 12) - 7.
The MLP mirrors the device's BF16 rounding points when ``mirror`` is set.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

BS, NH = 32, 17
BINS = BS * NH
IN, HID, OUT = 576, 512, 640
FIR = 16
PATCH = BS + FIR - 1
LAGS = 2 * FIR - 1
NSINES = 64
FEAT_MEAN, FEAT_SCALE, LOG_OFFSET = 8.0, 0.4, 7.0
RNG_BLOCK, RNG_WHITE, RNG_FIELD, RNG_INIT = 1, 2, 3, 4

O_W1 = 0
O_B1 = O_W1 + HID * IN
O_W2 = O_B1 + HID
O_B2 = O_W2 + HID * HID
O_W3 = O_B2 + HID
O_B3 = O_W3 + OUT * HID
NPARAM = O_B3 + OUT

_U = np.uint64


def mix64(z):
    z = np.asarray(z, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = z + _U(0x9E3779B97F4A7C15)
        z = (z ^ (z >> _U(30))) * _U(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> _U(27))) * _U(0x94D049BB133111EB)
    return z ^ (z >> _U(31))


def rnd(seed, stream, index):
    with np.errstate(over="ignore"):
        key = mix64(np.asarray(seed, dtype=np.uint64) ^ (np.asarray(stream, dtype=np.uint64) * _U(0xD1B54A32D192ED03)))
    return mix64(key ^ np.asarray(index, dtype=np.uint64))


def unif(z):
    return (np.asarray(z, dtype=np.uint64) >> _U(40)).astype(np.float64) / 16777216.0


def unif_int(z, n):
    return ((np.asarray(z, dtype=np.uint64) >> _U(40)) * _U(n)) >> _U(24)


def gauss(z):
    z = np.asarray(z, dtype=np.uint64)
    u1 = ((z >> _U(40)).astype(np.float64) + 1.0) / 16777216.0
    u2 = ((z >> _U(16)) & _U(0xFFFFFF)).astype(np.float64) / 16777216.0
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


def bf16(x):
    """Round to BF16 (nearest, ties to even) and return as float64."""
    f = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


# ---------------------------------------------------------------- windows

def analysis_window(wintype: int, b: int, o: int) -> np.ndarray:
    """Analysis window of src/fft3d_engine.h:204-283 (computed in float like the reference)."""
    w = np.ones(b, np.float32)
    pi = np.float32(np.pi)
    for i in range(o):
        cl = np.float32(np.cos(np.float32(pi * np.float32(i - o + 0.5) / np.float32(o * 2))))
        cr = np.float32(np.cos(np.float32(pi * np.float32(i + 0.5) / np.float32(o * 2))))
        if wintype == 0:
            l, r = cl, cr
        elif wintype == 1:
            l, r = np.float32(np.sqrt(float(cl))), np.float32(np.sqrt(float(cr)))
        else:
            l = r = np.float32(1.0)
        w[i] = l
        w[b - o + i] = r
    return w.astype(np.float64)


# ---------------------------------------------------------------- clean frames

def field_params(seed: int, frame: int):
    k = np.arange(NSINES, dtype=np.uint64)
    base = (_U(frame) * _U(NSINES) + k) * _U(4)
    period = 8.0 + 192.0 * unif(rnd(seed, RNG_FIELD, base))
    theta = np.pi * unif(rnd(seed, RNG_FIELD, base + _U(1)))
    phase = unif(rnd(seed, RNG_FIELD, base + _U(2)))
    amp = 0.5 + 0.5 * unif(rnd(seed, RNG_FIELD, base + _U(3)))
    # the device evaluates float32 copies of these
    fx = (np.cos(theta) / period).astype(np.float32).astype(np.float64)
    fy = (np.sin(theta) / period).astype(np.float32).astype(np.float64)
    return fx, fy, phase.astype(np.float32).astype(np.float64), amp.astype(np.float32).astype(np.float64)


def clean_frame(seed: int, frame: int, width: int, height: int) -> np.ndarray:
    fx, fy, ph, amp = field_params(seed, frame)
    x = np.arange(width, dtype=np.float64)
    y = np.arange(height, dtype=np.float64)
    v = np.zeros((height, width))
    for k in range(NSINES):
        v += amp[k] * np.sin(2 * np.pi * (fx[k] * x[None, :] + fy[k] * y[:, None] + ph[k]))
    return 16.0 + (v - v.min()) * (219.0 / (v.max() - v.min()))


# ---------------------------------------------------------------- noise process

def block_params(seed: int, gb: int, frames: int, width: int, height: int, sigma_min=2.0, sigma_max=10.0,
                 knot_min=0.1):
    base = _U(gb) * _U(16)
    u = [float(unif(rnd(seed, RNG_BLOCK, base + _U(k)))) for k in range(10)]
    sigma = sigma_min + (sigma_max - sigma_min) * u[0]
    lk = np.log(knot_min) * u[9]  # span of the knots: log-uniform in [knot_min, 1]
    v = [float(np.exp(lk * u[1 + k])) for k in range(4)]
    rising = 1 if u[5] >= 0.5 else 0
    v = sorted(v) if rising else sorted(v, reverse=True)
    frame = int(unif_int(rnd(seed, RNG_BLOCK, base + _U(6)), frames))
    x0 = int(unif_int(rnd(seed, RNG_BLOCK, base + _U(7)), width - BS + 1))
    y0 = int(unif_int(rnd(seed, RNG_BLOCK, base + _U(8)), height - BS + 1))
    return dict(sigma=sigma, knots=np.array(v), rising=rising, frame=frame, x0=x0, y0=y0)


def spline_tangents(v):
    """Fritsch-Carlson tangents of the monotone cubic through (i/3, v[i])."""
    v = np.asarray(v, np.float64)
    dl = (v[1:] - v[:-1]) * 3.0
    m = np.zeros(4)
    m[0], m[3] = dl[0], dl[2]
    for k in (1, 2):
        m[k] = 0.0 if dl[k - 1] * dl[k] <= 0 else 0.5 * (dl[k - 1] + dl[k])
    for k in range(3):
        if dl[k] == 0:
            m[k] = m[k + 1] = 0.0
        else:
            a, b = m[k] / dl[k], m[k + 1] / dl[k]
            s2 = a * a + b * b
            if s2 > 9.0:
                tau = 3.0 / np.sqrt(s2)
                m[k], m[k + 1] = tau * a * dl[k], tau * b * dl[k]
    return m


def spline(v, r):
    v = np.asarray(v, np.float64)
    m = spline_tangents(v)
    r = np.asarray(r, np.float64)
    i = np.minimum(2, (r * 3.0).astype(int))
    t = (r - i / 3.0) * 3.0
    d = 1.0 / 3.0
    return ((2 * t ** 3 - 3 * t ** 2 + 1) * v[i] + (t ** 3 - 2 * t ** 2 + t) * d * m[i]
            + (-2 * t ** 3 + 3 * t ** 2) * v[i + 1] + (t ** 3 - t ** 2) * d * m[i + 1])


def transfer_samples(knots) -> np.ndarray:
    f = np.array([(i if i <= FIR // 2 else i - FIR) / FIR for i in range(FIR)])
    r = np.minimum(1.0, 2.0 * np.sqrt(f[:, None] ** 2 + f[None, :] ** 2))
    return spline(knots, r)


def fir(knots) -> np.ndarray:
    """Centred 16x16 FIR: h[a][b] is lag (a-8, b-8) of the inverse DFT of the samples."""
    h = np.real(np.fft.ifft2(transfer_samples(knots)))
    return np.roll(h, (FIR // 2, FIR // 2), axis=(0, 1))


def white_patch(seed: int, gb: int) -> np.ndarray:
    p = np.arange(PATCH * PATCH, dtype=np.uint64)
    return gauss(rnd(seed, RNG_WHITE, _U(gb) * _U(4096) + p)).reshape(PATCH, PATCH)


def shaped_noise(h: np.ndarray, w: np.ndarray) -> np.ndarray:
    """n[y][x] = sum_ab h[a][b] w[y+a][x+b] (valid correlation)."""
    out = np.zeros((w.shape[0] - FIR + 1, w.shape[1] - FIR + 1))
    for a in range(FIR):
        for b in range(FIR):
            out += h[a, b] * w[a:a + out.shape[0], b:b + out.shape[1]]
    return out


def noise_power(h: np.ndarray, gain: float, wx: np.ndarray, wy: np.ndarray) -> np.ndarray:
    """E|N_k|^2 of the windowed block (32 x 17 bins): sum_d R(d) A(d) cos(k.d)."""
    R = np.zeros((LAGS, LAGS))
    for dy in range(-(FIR - 1), FIR):
        for dx in range(-(FIR - 1), FIR):
            a0, a1 = max(0, -dy), min(FIR, FIR - dy)
            b0, b1 = max(0, -dx), min(FIR, FIR - dx)
            R[dy + FIR - 1, dx + FIR - 1] = np.sum(h[a0:a1, b0:b1] * h[a0 + dy:a1 + dy, b0 + dx:b1 + dx])
    R *= gain * gain
    lags = np.arange(-(FIR - 1), FIR)
    ax = np.array([np.sum(wx[max(0, -d):BS - max(0, d)] * wx[max(0, d):BS - max(0, -d)]) for d in lags])
    ay = np.array([np.sum(wy[max(0, -d):BS - max(0, d)] * wy[max(0, d):BS - max(0, -d)]) for d in lags])
    ky = np.arange(BS)[:, None, None, None]
    kx = np.arange(NH)[None, :, None, None]
    dy = lags[None, None, :, None]
    dx = lags[None, None, None, :]
    ph = np.cos(2 * np.pi * (ky * dy + kx * dx) / BS)
    RA = R * ay[:, None] * ax[None, :]
    return np.einsum("yxab,ab->yx", ph, RA)


def features(noisy: np.ndarray, wx: np.ndarray, wy: np.ndarray) -> np.ndarray:
    """Model input (576 values, BF16-rounded) of one 32x32 8-bit block."""
    X = np.fft.rfft2(noisy.astype(np.float64) * wy[:, None] * wx[None, :])
    f = np.zeros(IN)
    f[:BINS] = (np.log(np.abs(X.reshape(-1)) ** 2 + 1.0) - FEAT_MEAN) * FEAT_SCALE
    f[0] = 0.0
    return bf16(f)


def target(h: np.ndarray, gain: float, wx: np.ndarray, wy: np.ndarray) -> np.ndarray:
    q = np.sum(wx ** 2) * np.sum(wy ** 2) / 12.0
    return (np.log(noise_power(h, gain, wx, wy) + q) - LOG_OFFSET).reshape(-1)


def generate_block(seed: int, gb: int, frames: int, width: int, height: int, wx, wy, clean_block=None,
                   sigma_min=2.0, sigma_max=10.0, knot_min=0.1, clean_frames=None):
    """One training block as the device makes it. ``clean_block`` (32x32,
    unrounded) overrides the oracle's own clean frame evaluation."""
    p = block_params(seed, gb, frames, width, height, sigma_min, sigma_max, knot_min)
    h = fir(p["knots"])
    sumh2 = float(np.sum(h * h))
    gain = p["sigma"] / np.sqrt(sumh2)
    n = gain * shaped_noise(h, white_patch(seed, gb))
    if clean_block is None:
        fr = clean_frames[p["frame"]] if clean_frames is not None else clean_frame(seed, p["frame"], width, height)
        clean_block = fr[p["y0"]:p["y0"] + BS, p["x0"]:p["x0"] + BS]
    noisy = np.clip(np.rint(clean_block + n), 0, 255)
    return dict(params=p, h=h, gain=gain, sumh2=sumh2, clean=clean_block, noisy=noisy,
                features=features(noisy, wx, wy), target=target(h, gain, wx, wy))


# ---------------------------------------------------------------- MLP

def split(params: np.ndarray):
    p = np.asarray(params, np.float64)
    return (p[O_W1:O_B1].reshape(HID, IN), p[O_B1:O_W2], p[O_W2:O_B2].reshape(HID, HID), p[O_B2:O_W3],
            p[O_W3:O_B3].reshape(OUT, HID), p[O_B3:NPARAM])


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2 * np.pi)


def forward(params, X, mirror=True):
    W1, b1, W2, b2, W3, b3 = split(params)
    rnd_ = bf16 if mirror else (lambda a: np.asarray(a, np.float64))
    Xb = rnd_(X)
    W1b, W2b, W3b = rnd_(W1), rnd_(W2), rnd_(W3)
    Z1 = Xb @ W1b.T + b1
    H1 = rnd_(gelu(Z1))
    Z2 = H1 @ W2b.T + b2
    H2 = rnd_(gelu(Z2))
    Y = H2 @ W3b.T + b3
    return dict(Xb=Xb, W1b=W1b, W2b=W2b, W3b=W3b, Z1=Z1, H1=H1, Z2=Z2, H2=H2, Y=Y)


def loss_and_grads(params, X, T, mirror=True):
    """Mean squared error over the 544 outputs and its gradient (parameter layout)."""
    f = forward(params, X, mirror)
    rnd_ = bf16 if mirror else (lambda a: np.asarray(a, np.float64))
    R = X.shape[0]
    diff = f["Y"][:, :BINS] - T
    loss = float(np.mean(diff * diff))
    dY = np.zeros((R, OUT))
    dY[:, :BINS] = 2.0 * diff / (R * BINS)
    dYb = rnd_(dY)
    gW3 = dYb.T @ f["H2"]
    gb3 = dY.sum(0)
    dZ2 = (dYb @ f["W3b"]) * gelu_grad(f["Z2"])
    dZ2b = rnd_(dZ2)
    gW2 = dZ2b.T @ f["H1"]
    gb2 = dZ2.sum(0)
    dZ1 = (dZ2b @ f["W2b"]) * gelu_grad(f["Z1"])
    dZ1b = rnd_(dZ1)
    gW1 = dZ1b.T @ f["Xb"]
    gb1 = dZ1.sum(0)
    g = np.concatenate([gW1.reshape(-1), gb1, gW2.reshape(-1), gb2, gW3.reshape(-1), gb3])
    return loss, g


def init_params(seed: int) -> np.ndarray:
    """Initial weights as the device makes them: N(0, 1/fan_in), zero biases
    and zero weights on the padding input columns."""
    p = np.zeros(NPARAM)
    idx = np.arange(NPARAM, dtype=np.uint64)
    z = rnd(seed, RNG_INIT, idx)
    u1 = ((z >> _U(40)).astype(np.float64) + 1.0) / 16777216.0
    u2 = ((z >> _U(16)) & _U(0xFFFFFF)).astype(np.float64) / 16777216.0
    nrm = np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)
    W1 = (nrm[O_W1:O_B1] / np.sqrt(BINS)).reshape(HID, IN)
    W1[:, BINS:] = 0.0
    p[O_W1:O_B1] = W1.reshape(-1)
    p[O_W2:O_B2] = nrm[O_W2:O_B2] / np.sqrt(HID)
    p[O_W3:O_B3] = nrm[O_W3:O_B3] / np.sqrt(HID)
    return p.astype(np.float32).astype(np.float64)
