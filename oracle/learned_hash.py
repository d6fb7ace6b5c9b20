"""FP64 restatement of the learned hash (test infrastructure only).

The learned hash has no counterpart in the reference (its hash family is the
random hyperplanes of src/lsh_h.cu:88-100); this module restates the model,
the training loss and its gradients as the product documents them
(include/sift2nn.h, sift_mlp_train), in float64 numpy, so that the CUDA
kernels can be checked:

  a1 = W1 (x / 64) + b1,  h = bf16(relu(a1)),  z = W2 h + b2,  t = tanh(z)
  code bit j = (z_j > 0)
  loss = mean_i (1 - s(q_i, p_i)) + neg * mean_i s(q_i, n_i)^2 + balance * sum_j m_j^2
  s(a, b) = mean_j t_aj t_bj,  m_j = mean over the 3B rows of t_j

Weights enter the forward pass rounded to BF16; gradients pass straight
through the roundings (of the weights and of h). Parameters are one flat
float array: W1 [256][128], b1 [256], W2 [32][256] (rows >= k zero), b2 [32].
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT_ROWS = 128, 256, 32
N_PARAMS = HID * IN + HID + OUT_ROWS * HID + OUT_ROWS


def bf16_round(x) -> np.ndarray:
    """Round to the nearest bfloat16 (ties to even), returned as float32."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(params):
    p = np.asarray(params, dtype=np.float64)
    o = 0
    w1 = p[o:o + HID * IN].reshape(HID, IN)
    o += HID * IN
    b1 = p[o:o + HID]
    o += HID
    w2 = p[o:o + OUT_ROWS * HID].reshape(OUT_ROWS, HID)
    o += OUT_ROWS * HID
    b2 = p[o:o + OUT_ROWS]
    return w1, b1, w2, b2


def pack(w1, b1, w2, b2) -> np.ndarray:
    return np.concatenate([np.ravel(w1), np.ravel(b1), np.ravel(w2), np.ravel(b2)]).astype(np.float32)


def init_params(k: int, seed: int = 0) -> np.ndarray:
    """Random parameters at the training's initial scales (test inputs)."""
    rng = np.random.default_rng(seed)
    w1 = rng.normal(0, 0.125, (HID, IN))
    b1 = rng.normal(0, 0.3, HID)
    w2 = np.zeros((OUT_ROWS, HID))
    w2[:k] = rng.normal(0, 0.0884, (k, HID))
    b2 = np.zeros(OUT_ROWS)
    b2[:k] = rng.normal(0, 0.1, k)
    return pack(w1, b1, w2, b2)


def forward(params, x, k: int, round_bf16: bool = True):
    """(h, z) for uint8 rows x [n][128]: float64 arithmetic on BF16-rounded
    weights, h rounded to BF16 (round_bf16=False: the unrounded model, whose
    gradient a finite-difference check can test)."""
    w1, b1, w2, b2 = unpack(params)
    rnd = (lambda a: bf16_round(a).astype(np.float64)) if round_bf16 else (lambda a: np.asarray(a, np.float64))
    w1b = rnd(w1)
    w2b = rnd(w2[:k])
    a1 = (np.asarray(x, np.float64) / 64.0) @ w1b.T + b1
    h = rnd(np.maximum(a1, 0.0))
    z = h @ w2b.T + b2[:k]
    return h, z


def codes(params, x, k: int) -> np.ndarray:
    _, z = forward(params, x, k)
    return ((z > 0).astype(np.uint64) << np.arange(k, dtype=np.uint64)).sum(1).astype(np.uint32)


def loss_grad(params, x, B: int, k: int, neg: float, balance: float, round_bf16: bool = True):
    """(loss[4], flat gradient) for rows x = [queries | neighbours | random] (3B rows)."""
    w1, b1, w2, b2 = unpack(params)
    w2b = bf16_round(w2[:k]).astype(np.float64) if round_bf16 else w2[:k]
    xs = np.asarray(x, np.float64) / 64.0
    h, z = forward(params, x, k, round_bf16)
    t = np.tanh(z)
    R = 3 * B
    tq, tp, tn = t[:B], t[B:2 * B], t[2 * B:]
    sqp = (tq * tp).sum(1) / k
    sqn = (tq * tn).sum(1) / k
    m = t.mean(0)
    pos, negl, bal = (1 - sqp).mean(), (sqn ** 2).mean(), (m ** 2).sum()
    loss = np.array([pos + neg * negl + balance * bal, pos, negl, bal])
    dt = np.zeros_like(t)
    dt[:B] += -tp / (k * B) + (neg * 2 * sqn / (k * B))[:, None] * tn
    dt[B:2 * B] += -tq / (k * B)
    dt[2 * B:] += (neg * 2 * sqn / (k * B))[:, None] * tq
    dt += balance * 2 * m / R
    dz = dt * (1 - t ** 2)
    gw2 = np.zeros((OUT_ROWS, HID))
    gb2 = np.zeros(OUT_ROWS)
    gw2[:k] = dz.T @ h
    gb2[:k] = dz.sum(0)
    da1 = (dz @ w2b) * (h > 0)
    gw1 = da1.T @ xs
    gb1 = da1.sum(0)
    return loss, np.concatenate([gw1.ravel(), gb1, gw2.ravel(), gb2])
