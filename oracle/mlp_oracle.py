"""CPU oracle of the warm-start network (test infrastructure, not product code).

The network has no counterpart in the reference: it is the learned warm start
of the PBF constraint solve whose plain iteration is particles.c:588-746
(ComputeLambda / UpdateDPs).  This file restates, in numpy, what the CUDA
kernels in sphpc_b200/csrc/mlp.cu compute, so that tests can check them:

  x0 = bf16((f - mean) * inv_std)                          16 features
  z1 = x0 . bf16(W1)^T + bf16(b1),  h1 = bf16(relu(z1))    64
  z2 = h1 . bf16(W2)^T + bf16(b2),  h2 = bf16(relu(z2))    64
  z3 = h2 . bf16(W3)^T + bf16(b3),  h3 = relu(z3)          64 (FP32)
  u  = w4 . h3 + b4,           lambda0 = out_scale * u

relu(z) = max(z, 0), with derivative 1 for z > 0 and 0 otherwise.
With bf16=False every rounding is skipped and the arithmetic is float64:
that variant is the one the finite-difference gradient check runs on.

Training loss over a batch of B rows with targets t:
  L = 1/(2B) * sum_p (u_p - t_p / out_scale)^2
and the update is AdamW (Loshchilov & Hutter 2019) with decoupled weight decay
on the weight matrices only (W1, W2, W3, w4), not on the biases.
"""
from __future__ import annotations

import numpy as np

N_IN = 16
N_HID = 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + N_HID * N_IN
OFF_W2 = OFF_B1 + N_HID
OFF_B2 = OFF_W2 + N_HID * N_HID
OFF_W3 = OFF_B2 + N_HID
OFF_B3 = OFF_W3 + N_HID * N_HID
OFF_W4 = OFF_B3 + N_HID
OFF_B4 = OFF_W4 + N_HID
N_PARAMS = OFF_B4 + 1  # 9473
N_NORM = 2 * N_IN + 1


def bf16(a):
    """Round float32 values to the nearest bfloat16 (ties to even), kept as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def relu(z):
    return np.maximum(z, 0.0)


def relu_grad(z):
    return (z > 0.0).astype(np.float64)


def unpack(params):
    p = np.asarray(params)
    return {
        "W1": p[OFF_W1:OFF_B1].reshape(N_HID, N_IN),
        "b1": p[OFF_B1:OFF_W2],
        "W2": p[OFF_W2:OFF_B2].reshape(N_HID, N_HID),
        "b2": p[OFF_B2:OFF_W3],
        "W3": p[OFF_W3:OFF_B3].reshape(N_HID, N_HID),
        "b3": p[OFF_B3:OFF_W4],
        "w4": p[OFF_W4:OFF_B4],
        "b4": p[OFF_B4],
    }


def init_params(seed=0):
    """Uniform +-1/sqrt(fan_in) weights and zero biases (float32)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    for off, fan_out, fan_in in ((OFF_W1, N_HID, N_IN), (OFF_W2, N_HID, N_HID),
                                 (OFF_W3, N_HID, N_HID), (OFF_W4, 1, N_HID)):
        lim = 1.0 / np.sqrt(fan_in)
        p[off:off + fan_out * fan_in] = rng.uniform(-lim, lim, fan_out * fan_in)
    return p


def forward(params, norm, feat, bf16_emulation=True):
    """Returns (lambda0, cache); cache holds what backward needs."""
    q = unpack(params)
    norm = np.asarray(norm, np.float32)
    mean, istd, scale = norm[:N_IN], norm[N_IN:2 * N_IN], norm[2 * N_IN]
    if bf16_emulation:
        f = np.asarray(feat, np.float32)
        x0 = bf16((f - mean) * istd).astype(np.float64)
        W = [bf16(q["W1"]).astype(np.float64), bf16(q["W2"]).astype(np.float64),
             bf16(q["W3"]).astype(np.float64)]
        rnd = lambda a: bf16(a.astype(np.float32)).astype(np.float64)
    else:
        f = np.asarray(feat, np.float64)
        x0 = (f - mean.astype(np.float64)) * istd.astype(np.float64)
        W = [q["W1"].astype(np.float64), q["W2"].astype(np.float64), q["W3"].astype(np.float64)]
        rnd = lambda a: a
    b = [q["b1"].astype(np.float64), q["b2"].astype(np.float64), q["b3"].astype(np.float64)]
    if bf16_emulation:
        # the kernels carry each hidden bias through the MMA as a BF16 weight
        # against a constant-one input column
        b = [bf16(v.astype(np.float32)).astype(np.float64) for v in b]
    hs = [x0]
    zs = []
    h = x0
    for l in range(3):
        z = h @ W[l].T + b[l]
        zs.append(z)
        a = relu(z)
        h = rnd(a) if l < 2 else a
        hs.append(h)
    u = h @ q["w4"].astype(np.float64) + float(q["b4"])
    cache = {"hs": hs, "zs": zs, "W": W, "w4": q["w4"].astype(np.float64), "u": u,
             "scale": float(scale), "rnd": rnd}
    return u * float(scale), cache


def loss_and_grad(params, norm, feat, target, bf16_emulation=True):
    """L and dL/dparams (float64 vector of N_PARAMS) for one batch."""
    _, c = forward(params, norm, feat, bf16_emulation)
    B = len(target)
    r = c["u"] - np.asarray(target, np.float64) / c["scale"]
    loss = 0.5 * np.mean(r * r)
    g = np.zeros(N_PARAMS, np.float64)
    gu = r / B
    hs, zs, W, rnd = c["hs"], c["zs"], c["W"], c["rnd"]
    # the kernels form the last layer's weight gradient on the tensor cores from
    # bf16(gu) and bf16(h3)
    g[OFF_W4:OFF_B4] = rnd(gu) @ rnd(hs[3])
    g[OFF_B4] = rnd(gu).sum()
    # dz of the last hidden layer; with bf16 emulation the kernels keep dz in bf16
    dz = rnd(np.outer(gu, c["w4"]) * relu_grad(zs[2]))
    offs = ((OFF_W1, OFF_B1), (OFF_W2, OFF_B2), (OFF_W3, OFF_B3))
    for l in (2, 1, 0):
        ow, ob = offs[l]
        g[ow:ob] = (dz.T @ hs[l]).ravel()
        g[ob:ob + N_HID] = dz.sum(axis=0)
        if l > 0:
            dz = rnd((dz @ W[l]) * relu_grad(zs[l - 1]))
    return loss, g


WEIGHT_DECAY_MASK = np.zeros(N_PARAMS, bool)
WEIGHT_DECAY_MASK[OFF_W1:OFF_B1] = True
WEIGHT_DECAY_MASK[OFF_W2:OFF_B2] = True
WEIGHT_DECAY_MASK[OFF_W3:OFF_B3] = True
WEIGHT_DECAY_MASK[OFF_W4:OFF_B4] = True


def adamw_step(params, grad, m, v, step, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, wd=1e-4):
    """One AdamW update (step counts from 1); returns new (params, m, v) as float32."""
    p = np.asarray(params, np.float64)
    g = np.asarray(grad, np.float64)
    m = beta1 * np.asarray(m, np.float64) + (1 - beta1) * g
    v = beta2 * np.asarray(v, np.float64) + (1 - beta2) * g * g
    mh = m / (1 - beta1 ** step)
    vh = v / (1 - beta2 ** step)
    p = p - lr * (mh / (np.sqrt(vh) + eps) + wd * np.where(WEIGHT_DECAY_MASK, p, 0.0))
    return p.astype(np.float32), m.astype(np.float32), v.astype(np.float32)
