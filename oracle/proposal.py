"""Test infrastructure (oracle): numpy restatement of the proposal network of
diff-triangle-tracer_b200/csrc/proposal.cu (no counterpart in the reference,
which traces every ray to the far plane). Used only by tests to check the
tensor-core kernels.

Network: the ray origin o is moved along the ray to the closest approach of
its line to the centre c (o' = o + s d, s = -(o - c).d / d.d); 80 inputs
((o' - c) * origin_scale and the direction, sin / cos of 2^k pi x for
k = 0..5 over those 6 coordinates, a constant 1, a zero) ->
64 -> 64 -> 64 (ReLU, each followed by a constant-1 input) -> 16 outputs (the
first two used). Weights W1 [64][80], W2 [64][80], W3 [64][80], W4 [16][80]
flattened in that order; a layer's bias is the weight column fed by the
constant 1.

`bf16=True` rounds exactly where the kernels do: the encoded inputs, the
weights, every hidden activation and every backpropagated pre-activation
gradient go to BF16 (round to nearest even); sums are FP64 here (FP32 in the
kernels).
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT_ROWS = 80, 64, 16
ROWS = (HID, HID, HID, OUT_ROWS)
OFF = (0, HID * IN, 2 * HID * IN, 3 * HID * IN)
PARAMS = 3 * HID * IN + OUT_ROWS * IN


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) & 0xFFFF0000).astype(np.uint32).view(np.float32).reshape(np.shape(x))


def layers(params):
    p = np.asarray(params, np.float64).reshape(-1)
    return [p[OFF[l]:OFF[l] + ROWS[l] * IN].reshape(ROWS[l], IN) for l in range(4)]


def closest_offset(rays, center=(0.0, 0.0, 0.0)):
    """s of each ray and its centred closest-approach origin o + s d - c."""
    rays = np.asarray(rays, np.float64)
    o = rays[:, :3] - np.asarray(center, np.float64)
    d = rays[:, 3:6]
    s = -np.sum(o * d, 1) / np.sum(d * d, 1)
    return s, o + s[:, None] * d


def encode(rays, origin_scale, center=(0.0, 0.0, 0.0)):
    """rays [n, 6] -> inputs [n, 80] (float64)."""
    rays = np.asarray(rays, np.float64)
    _, o = closest_offset(rays, center)
    v = np.concatenate([o * origin_scale, rays[:, 3:6]], 1).astype(np.float32).astype(np.float64)
    f = [v]
    for k in range(6):
        a = v * float(1 << k)
        f.append(np.sin(np.pi * a))
        f.append(np.cos(np.pi * a))
    n = rays.shape[0]
    f.append(np.ones((n, 1)))
    f.append(np.zeros((n, 1)))
    return np.concatenate(f, 1)


def _r(x, on):
    return bf16(x.astype(np.float32)).astype(np.float64) if on else x


def _ext(h):
    n = h.shape[0]
    return np.concatenate([h, np.ones((n, 1)), np.zeros((n, IN - HID - 1))], 1)


def forward(params, rays, origin_scale, center=(0.0, 0.0, 0.0), bf16_ops=True):
    """Returns (raw outputs [n, 16], activations [act0..act3])."""
    W = [_r(w, bf16_ops) for w in layers(params)]
    act = [_r(encode(rays, origin_scale, center), bf16_ops)]
    for l in range(3):
        z = act[l] @ W[l].T
        act.append(_ext(_r(np.maximum(z, 0.0), bf16_ops)))
    y = act[3] @ W[3].T
    return y, act


def predict(params, rays, origin_scale, t_shift, t_scale, center=(0.0, 0.0, 0.0), bf16_ops=True):
    """(t_near, t_far) [n, 2] in t along the ray from its origin."""
    y, _ = forward(params, rays, origin_scale, center, bf16_ops)
    s, _ = closest_offset(rays, center)
    return y[:, :2] * t_scale + t_shift + s[:, None]


def loss_and_grad(params, rays, targets, origin_scale, t_shift, t_scale, near_weight, far_weight,
                  center=(0.0, 0.0, 0.0), bf16_ops=True):
    """Mean asymmetric loss and its gradient with respect to the flattened
    parameters (the kernels' training step before Adam). A t_near above its
    target weighs near_weight, a t_far below its target far_weight; a ray
    whose t_near target is negative (no hit) has no t_near term."""
    W = [_r(w, bf16_ops) for w in layers(params)]
    y, act = forward(params, rays, origin_scale, center, bf16_ops)
    n = rays.shape[0]
    raw = np.asarray(targets, np.float32).astype(np.float64)
    s, _ = closest_offset(rays, center)
    tg = (raw - s[:, None] - t_shift) / t_scale
    e0, e1 = y[:, 0] - tg[:, 0], y[:, 1] - tg[:, 1]
    w0 = np.where(raw[:, 0] >= 0, np.where(e0 > 0, near_weight, 1.0), 0.0)
    w1 = np.where(e1 < 0, far_weight, 1.0)
    loss = float(np.sum(w0 * e0 ** 2 + w1 * e1 ** 2) / n)
    dz = np.zeros((n, OUT_ROWS))
    dz[:, 0], dz[:, 1] = 2 * w0 * e0, 2 * w1 * e1
    dz = _r(dz, bf16_ops)
    grads = [None] * 4
    for l in range(3, -1, -1):
        grads[l] = dz.T @ act[l]
        if l > 0:
            da = dz @ W[l][:, :HID]
            dz = _r(da * (act[l][:, :HID] > 0), bf16_ops)
    g = np.concatenate([x.reshape(-1) for x in grads]) / n
    return loss, g


def adam(params, m, v, g, step, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    m = beta1 * m + (1 - beta1) * g
    v = beta2 * v + (1 - beta2) * g * g
    c1 = 1.0 / (1.0 - beta1 ** step)
    c2 = 1.0 / (1.0 - beta2 ** step)
    return params - lr * (m * c1) / (np.sqrt(v * c2) + eps), m, v
