"""The oracle (CPU restatement) against the reference's own outputs.

The golden fixtures are the unmodified reference plugin's outputs (C path,
opt=1) on seeded clips. The float restatement must reproduce them BIT FOR BIT
(it keeps the reference's operand order and uses the same FFT); the FP64
restatement must agree within +-1 LSB on >= 99.9 % of pixels.
"""
import numpy as np
import pytest

from oracle import restate
from tests import golden_data

CASES = golden_data.load()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_float_restatement_is_bit_exact(case):
    name, planes, bits, params, want = case
    got = restate.filter_clip(planes, bits=bits, **params)
    for i, (g, w) in enumerate(zip(got, want)):
        assert np.array_equal(g, w), (name, i, int(np.abs(g.astype(int) - w.astype(int)).max()))


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_fp64_restatement_close(case):
    name, planes, bits, params, want = case
    got = restate.filter_clip(planes, bits=bits, dbl=True, **params)
    for i, (g, w) in enumerate(zip(got, want)):
        d = np.abs(g.astype(np.int64) - w.astype(np.int64))
        assert (d <= 1).mean() >= 0.999, (name, i, d.max(), (d <= 1).mean())
