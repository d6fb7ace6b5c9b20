"""The FP64 restatement of the learned hash (oracle/learned_hash.py) on its
own: its analytic gradient against finite differences of its loss, and the
BF16 rounding against torch's."""
import numpy as np
import pytest

from oracle import learned_hash as lh
from matching_sift_b200 import datagen


def _rows(B, seed):
    base = datagen.make_base(4 * B, seed=seed)
    q = datagen.make_queries(B, base, seed=seed)
    return np.concatenate([q, base[:B], base[2 * B:3 * B]])


@pytest.mark.parametrize("k", [3, 16])
def test_gradient_matches_finite_differences(k):
    B = 8
    x = _rows(B, 3)
    p = lh.init_params(k, seed=1).astype(np.float64)
    loss, g = lh.loss_grad(p, x, B, k, 0.7, 0.5, round_bf16=False)
    rng = np.random.default_rng(0)
    # coordinates of every parameter block (W2 / b2 rows < k only)
    idx = np.concatenate([rng.choice(lh.HID * lh.IN, 20, replace=False),
                          lh.HID * lh.IN + rng.choice(lh.HID, 10, replace=False),
                          lh.HID * lh.IN + lh.HID + rng.choice(k * lh.HID, 20, replace=False),
                          lh.HID * lh.IN + lh.HID + lh.OUT_ROWS * lh.HID + np.arange(k)])
    eps = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (lh.loss_grad(pp, x, B, k, 0.7, 0.5, round_bf16=False)[0][0] -
              lh.loss_grad(pm, x, B, k, 0.7, 0.5, round_bf16=False)[0][0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])
    # padded W2 rows and b2 entries get no gradient
    off = lh.HID * lh.IN + lh.HID
    assert not g[off + k * lh.HID: off + lh.OUT_ROWS * lh.HID].any()
    assert not g[off + lh.OUT_ROWS * lh.HID + k:].any()


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    x = np.random.default_rng(0).normal(0, 3, 10000).astype(np.float32)
    x[:4] = [0.0, -0.0, 1.00390625, 1.01171875]  # exact ties round to even
    want = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    np.testing.assert_array_equal(lh.bf16_round(x), want)
