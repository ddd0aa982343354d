"""CPU checks of the learned noise-PSD oracle (oracle/psd.py) itself, before it
judges the GPU: its backward pass against finite differences of its own FP64
loss, its exact noise-power formula against a Monte-Carlo estimate, the
monotone spline and the FIR design, and BF16 rounding."""
import numpy as np
import pytest

from neo_fft3d_b200 import synth
from oracle import psd


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, 1.0 + 2 ** -9, 3.14159, -2.5e-3, 0.0])
    got = psd.bf16(x)
    # 1 + 2^-9 is a tie between 1 and 1 + 2^-7 ... ties to even -> 1.0
    assert got[0] == 1.0 and got[1] == 1.0 and got[3] == 1.0
    assert got[2] == 1.0078125
    assert abs(got[4] - 3.140625) < 1e-12
    assert got[6] == 0.0


def test_mlp_backward_matches_finite_differences():
    rng = np.random.default_rng(5)
    p = psd.init_params(2)
    p[psd.O_B1:psd.O_W2] = rng.normal(0, 0.1, psd.HID)
    p[psd.O_B2:psd.O_W3] = rng.normal(0, 0.1, psd.HID)
    p[psd.O_B3:] = rng.normal(0, 0.1, psd.OUT)
    X = np.zeros((4, psd.IN))
    X[:, :psd.BINS] = rng.normal(0, 1, (4, psd.BINS))
    T = rng.normal(0, 1, (4, psd.BINS))
    loss, g = psd.loss_and_grads(p, X, T, mirror=False)
    eps = 1e-6
    idx = []
    for lo, hi in [(psd.O_W1, psd.O_B1), (psd.O_B1, psd.O_W2), (psd.O_W2, psd.O_B2), (psd.O_B2, psd.O_W3),
                   (psd.O_W3, psd.O_W3 + psd.BINS * psd.HID), (psd.O_B3, psd.O_B3 + psd.BINS)]:
        idx += list(rng.integers(lo, hi, 4))
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        lp = psd.loss_and_grads(pp, X, T, mirror=False)[0]
        lm = psd.loss_and_grads(pm, X, T, mirror=False)[0]
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * max(1e-3, abs(g[i])) + 1e-10, (i, fd, g[i])


def test_padding_outputs_get_no_gradient():
    rng = np.random.default_rng(1)
    p = psd.init_params(3)
    X = np.zeros((2, psd.IN))
    X[:, 1:psd.BINS] = rng.normal(0, 1, (2, psd.BINS - 1))
    _, g = psd.loss_and_grads(p, X, rng.normal(0, 1, (2, psd.BINS)), mirror=True)
    W1g = g[psd.O_W1:psd.O_B1].reshape(psd.HID, psd.IN)
    W3g = g[psd.O_W3:psd.O_B3].reshape(psd.OUT, psd.HID)
    assert np.all(W1g[:, psd.BINS:] == 0) and np.all(W3g[psd.BINS:] == 0)
    assert np.all(g[psd.O_B3 + psd.BINS:] == 0)


@pytest.mark.parametrize("knots", [[1.0, 0.5, 0.2, 0.1], [0.1, 0.4, 0.4, 1.0], [0.3, 0.3, 0.3, 0.3]])
def test_spline_monotone_and_interpolating(knots):
    r = np.linspace(0, 1, 301)
    h = psd.spline(knots, r)
    d = np.diff(h)
    assert np.all(d <= 1e-12) or np.all(d >= -1e-12)
    np.testing.assert_allclose(psd.spline(knots, np.array([0, 1 / 3, 2 / 3, 1.0])), knots, atol=1e-12)


def test_fir_reproduces_transfer_samples():
    knots = [1.0, 0.6, 0.25, 0.1]
    h = psd.fir(knots)
    H = np.real(np.fft.fft2(np.roll(h, (-8, -8), axis=(0, 1))))
    np.testing.assert_allclose(H, psd.transfer_samples(knots), atol=1e-12)
    np.testing.assert_allclose(synth.noise_fir(knots), h, atol=1e-12)


def test_noise_power_matches_monte_carlo():
    """E|N_k|^2 of windowed shaped noise: analytic sum_d R(d) A(d) cos(k.d)
    against the mean over 4000 independent noise blocks."""
    knots = [1.0, 0.5, 0.2, 0.1]
    h = psd.fir(knots)
    gain = 5.0 / np.sqrt(np.sum(h * h))
    wx = wy = psd.analysis_window(0, 32, 16)
    P = psd.noise_power(h, gain, wx, wy)
    rng = np.random.default_rng(9)
    acc = np.zeros((32, 17))
    n = 4000
    from scipy.signal import correlate
    for _ in range(n // 500):
        w = rng.standard_normal((500, psd.PATCH, psd.PATCH))
        blk = gain * correlate(w, h[None], mode="valid", method="fft")
        X = np.fft.rfft2(blk * wy[None, :, None] * wx[None, None, :])
        acc += np.sum(np.abs(X) ** 2, axis=0)
    mc = acc / n
    rel = np.abs(mc / P - 1)
    # |N_k|^2 is exponential-like: the mean of 4000 has a relative std of ~1.6 %
    # (~2.2 % at the real-valued DC / Nyquist bins)
    assert np.mean(rel) < 0.03 and np.max(rel) < 0.12, (np.mean(rel), np.max(rel))


def test_noise_sigma_scaling():
    knots = [0.1, 0.3, 0.6, 1.0]
    h = psd.fir(knots)
    gain = 7.0 / np.sqrt(np.sum(h * h))
    w = np.random.default_rng(4).standard_normal((600, 600))
    n = gain * psd.shaped_noise(h, w)
    assert abs(np.std(n) - 7.0) < 0.1


def test_generator_random_streams_are_stable():
    # SplitMix64 known answers (the finaliser of seed 0 at index 0, and one keyed draw)
    assert int(psd.mix64(np.uint64(0))) == 0xE220A8397B1DCDAF
    a = psd.rnd(4, 1, np.arange(4, dtype=np.uint64))
    b = psd.rnd(4, 1, np.arange(4, dtype=np.uint64))
    assert np.array_equal(a, b) and len(set(int(x) for x in a)) == 4
