"""Learned noise PSD on the GPU, checked against the FP64 oracle (oracle/psd.py)
through the C ABI:

* the device block generator (clean frames, noise process, noisy pixels,
  features, exact noise-power targets);
* the tensor-core MLP forward pass and its gradients (all six parameter
  tensors) against an FP64 autograd that rounds to BF16 where the device does;
* training lowers the held-out loss;
* the trained model (2^21 generated blocks), feeding the Wiener 3D (bt=5)
  gain in place of sigma, against the scalar-sigma filter's PSNR on
  coloured-noise clips: at the noise's true sigma and at the best sigma of a
  sweep; 10-bit samples, Kalman and Wiener 2D; geometry checks.
"""
import numpy as np
import pytest

from neo_fft3d_b200 import engine, psd, synth
from oracle import psd as opsd

GEN = dict(width=256, height=192, clean_frames=2, seed=11)


@pytest.fixture(scope="module")
def model(gpu):
    m = psd.PsdModel(seed=3)
    yield m
    m.close()


@pytest.mark.gpu
def test_generator_vs_oracle(model):
    first, count = 1000, 64
    out = model.generate(first, count, **GEN)
    wx = wy = opsd.analysis_window(0, 32, 16)
    frames = [opsd.clean_frame(GEN["seed"], f, GEN["width"], GEN["height"]) for f in range(GEN["clean_frames"])]
    same = 0
    for i in range(count):
        info = out["info"][i]
        ref = opsd.generate_block(GEN["seed"], first + i, GEN["clean_frames"], GEN["width"], GEN["height"], wx, wy,
                                  clean_block=out["clean"][i].astype(np.float64))
        p = ref["params"]
        assert abs(info[0] - p["sigma"]) <= 1e-5 * p["sigma"]
        np.testing.assert_allclose(info[1:5], p["knots"], rtol=1e-5)
        assert (int(info[5]), int(info[7]), int(info[8]), int(info[9])) == (p["rising"], p["frame"], p["x0"], p["y0"])
        assert abs(info[10] - ref["sumh2"]) <= 1e-4 * ref["sumh2"]
        assert abs(info[6] - ref["gain"]) <= 1e-4 * ref["gain"]
        # clean pixels: the same sinusoid field (FP32 on the device)
        cref = frames[p["frame"]][p["y0"]:p["y0"] + 32, p["x0"]:p["x0"] + 32]
        assert np.max(np.abs(out["clean"][i] - cref)) < 0.05
        # noisy pixels from the same white noise and FIR (FP32 vs FP64 sums can
        # move a value across a rounding boundary: then by one code)
        d = out["noisy"][i].astype(int) - ref["noisy"].astype(int)
        assert np.max(np.abs(d)) <= 1
        same += int(np.sum(d == 0))
        # features of the device's own noisy block, to BF16 rounding
        fref = opsd.features(out["noisy"][i], wx, wy)
        assert np.max(np.abs(out["features"][i] - fref)) <= 0.01 * np.max(np.abs(fref)) + 1e-6
        # exact noise power of the windowed block (log domain)
        assert np.max(np.abs(out["target"][i] - ref["target"])) < 2e-3
    assert same >= 0.999 * count * 1024, same


def _params(seed):
    rng = np.random.default_rng(seed)
    p = opsd.init_params(seed)
    p[opsd.O_B1:opsd.O_W2] = rng.normal(0, 0.1, opsd.HID)
    p[opsd.O_B2:opsd.O_W3] = rng.normal(0, 0.1, opsd.HID)
    p[opsd.O_B3:] = rng.normal(0, 0.1, opsd.OUT)
    return p.astype(np.float32)


TENSORS = [("W1", opsd.O_W1, opsd.O_B1), ("b1", opsd.O_B1, opsd.O_W2), ("W2", opsd.O_W2, opsd.O_B2),
           ("b2", opsd.O_B2, opsd.O_W3), ("W3", opsd.O_W3, opsd.O_B3), ("b3", opsd.O_B3, opsd.NPARAM)]


@pytest.mark.gpu
def test_init_params_match_oracle(gpu):
    m = psd.PsdModel(seed=7)
    np.testing.assert_allclose(m.params(), opsd.init_params(7), rtol=0, atol=1e-7)
    m.close()


@pytest.mark.gpu
def test_forward_and_gradients_vs_fp64(model):
    blk = model.generate(0, 256, **GEN)
    X, T = blk["features"], blk["target"]
    p = _params(21)
    model.set_params(p)
    np.testing.assert_array_equal(model.params(), p)
    # forward
    Y = model.forward(X)
    f = opsd.forward(p.astype(np.float64), X.astype(np.float64), mirror=True)
    ref = f["Y"][:, :opsd.BINS]
    assert np.linalg.norm(Y - ref) <= 1e-3 * np.linalg.norm(ref)
    # gradients: FP64 autograd with the device's BF16 rounding points
    loss, g = model.gradients(X, T)
    loss_o, g_o = opsd.loss_and_grads(p.astype(np.float64), X.astype(np.float64), T.astype(np.float64), mirror=True)
    assert abs(loss - loss_o) <= 1e-4 * loss_o
    for name, lo, hi in TENSORS:
        a, b = g[lo:hi].astype(np.float64), g_o[lo:hi]
        err = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert err < 5e-3, (name, err)
    # and against pure FP64 (no BF16 anywhere): the BF16 model's gradients
    # point the same way
    _, g64 = opsd.loss_and_grads(p.astype(np.float64), X.astype(np.float64), T.astype(np.float64), mirror=False)
    for name, lo, hi in TENSORS:
        a, b = g[lo:hi].astype(np.float64), g64[lo:hi]
        assert np.dot(a, b) / (np.linalg.norm(a) * np.linalg.norm(b)) > 0.99, name


@pytest.mark.gpu
def test_training_lowers_loss(gpu):
    m = psd.PsdModel(seed=5)
    curve, val = m.train(blocks=131072, batch=2048, epochs=2, width=640, height=480, clean_frames=4, curve_len=8)
    assert np.all(np.isfinite(curve)) and np.isfinite(val)
    assert curve[-1] < 0.5 * curve[0], curve
    assert val < 1.5 * curve[-1] + 0.02, (val, curve)
    m.close()


# coloured-noise clips: falling (low-pass), rising (high-pass), near white
CASES = [("lowpass", [1.0, 0.45, 0.2, 0.1], 6.0), ("highpass", [0.12, 0.3, 0.7, 1.0], 5.0),
         ("flat", [1.0, 0.9, 0.85, 0.8], 4.0)]
STRENGTH = 3.0


@pytest.fixture(scope="module")
def trained(gpu):
    m = psd.PsdModel(seed=1)
    curve, val = m.train()  # library defaults: 2^21 blocks, 3 epochs
    assert val < 0.05, val
    yield m, curve, val
    m.close()


def _filter(noisy, bits=8, **kw):
    return engine.filter_clip([noisy], bits=bits, bt=5, bw=32, bh=32, ow=16, oh=16, **kw)[0]


@pytest.mark.gpu
@pytest.mark.parametrize("name,knots,sigma", CASES, ids=[c[0] for c in CASES])
def test_learned_psd_vs_scalar_sigma(trained, name, knots, sigma):
    """PSNR against the clean frames, Wiener 3D bt=5: the learned noise power
    (strength 3, no knowledge of the noise) against the scalar-sigma filter at
    the noise's true sigma and at the best sigma of a sweep (hindsight)."""
    m, curve, val = trained
    noisy, clean = synth.make_coloured_clip(640, 480, 12, knots, sigma, seed=77)
    core = slice(2, -2)  # frames with the full bt = 5 window
    sweep = {float(s): synth.psnr(_filter(noisy, sigma=float(s))[core], clean[core])
             for s in sigma * np.geomspace(0.25, 3.0, 12)}
    best = max(sweep.values())
    at_true = synth.psnr(_filter(noisy, sigma=sigma)[core], clean[core])
    learned = synth.psnr(_filter(noisy, psd=m, psd_strength=STRENGTH)[core], clean[core])
    pooled = synth.psnr(_filter(noisy, psd=m, psd_pooled=True, psd_strength=STRENGTH)[core], clean[core])
    base = synth.psnr(noisy[core], clean[core])
    print(f"\n{name}: noisy {base:.2f} dB | scalar at true sigma {at_true:.2f}, best scalar {best:.2f} | "
          f"learned per-block {learned:.2f}, pooled {pooled:.2f} | held-out loss {val:.4f}")
    assert min(learned, pooled) > base + 5.0
    # never far below the hindsight-tuned scalar filter, clearly above it on
    # high-pass noise (which a single sigma cannot fit)
    assert pooled > best - 1.0 and learned > best - 1.0
    if name == "highpass":
        assert pooled > best + 2.0
    # against the scalar filter at the noise's own sigma
    assert pooled > at_true - 0.75
    if name != "flat":
        assert pooled > at_true + 1.0


@pytest.mark.gpu
def test_learned_psd_high_bit_depth(trained):
    """10-bit samples: the model sees power / 16 and its prediction is scaled
    back, so the 10-bit result is the 8-bit one at 4x finer output rounding."""
    m, _, _ = trained
    noisy, clean = synth.make_coloured_clip(320, 256, 8, [0.12, 0.3, 0.7, 1.0], 5.0, seed=78)
    out8 = _filter(noisy, psd=m).astype(np.float64)
    out10 = _filter(noisy.astype(np.uint16) * 4, bits=10, psd=m).astype(np.float64) / 4
    d = np.abs(out10 - out8)
    assert d.max() <= 0.75 and d.mean() < 0.3, (d.max(), d.mean())
    core = slice(2, -2)
    assert synth.psnr(out10[core], clean[core]) >= synth.psnr(out8[core], clean[core]) - 0.05


@pytest.mark.gpu
def test_learned_psd_kalman_and_edges(trained):
    """Kalman (bt=0) and Wiener 2D (bt=1) take the learned noise power too."""
    m, _, _ = trained
    noisy, clean = synth.make_coloured_clip(320, 256, 8, [1.0, 0.45, 0.2, 0.1], 6.0, seed=79)
    base = synth.psnr(noisy[1:], clean[1:])
    for bt in (0, 1):
        out = engine.filter_clip([noisy], bits=8, bt=bt, bw=32, bh=32, ow=16, oh=16, psd=m)[0]
        assert synth.psnr(out[1:], clean[1:]) > base + 1.0, bt


@pytest.mark.gpu
def test_set_psd_rejects_other_geometry(trained):
    m, _, _ = trained
    p = engine.make_params(sigma=2.0, bt=3, bw=48, bh=48, ow=16, oh=16)
    eng = engine.PlaneEngine(p, engine.plane_descs([(120, 160)], 8, 4)[0])
    with pytest.raises(engine.FFT3DError, match="bw = bh = 32"):
        eng.set_psd(m)
    eng.close()
    p = engine.make_params(sigma=2.0, bt=3, bw=32, bh=32, ow=8, oh=8)
    eng = engine.PlaneEngine(p, engine.plane_descs([(120, 160)], 8, 4)[0])
    with pytest.raises(engine.FFT3DError, match="ow/oh/wintype"):
        eng.set_psd(m)
    eng.close()
