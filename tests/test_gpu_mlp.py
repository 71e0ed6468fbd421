"""Tensor-core (tcgen05) kernels of the warm-start network against the numpy
oracle of the same network (bf16 operands and activations, FP32 accumulate)."""
import ctypes as C

import numpy as np
import pytest

from oracle import mlp_oracle as mo
from sphpc_b200 import _lib

pytestmark = pytest.mark.gpu


def _fptr(t):
    return C.c_void_p(t.data_ptr())


def _case(n, seed):
    rng = np.random.default_rng(seed)
    sd = rng.uniform(0.2, 4.0, mo.N_IN)
    mu = rng.normal(size=mo.N_IN) * 3
    feat = (rng.normal(size=(n, mo.N_IN)) * sd + mu).astype(np.float32)
    norm = np.concatenate([mu, 1.0 / sd, [0.37]]).astype(np.float32)
    params = mo.init_params(seed)
    params[mo.OFF_B1:mo.OFF_W2] = rng.normal(size=64) * 0.3
    params[mo.OFF_B2:mo.OFF_W3] = rng.normal(size=64) * 0.3
    params[mo.OFF_B3:mo.OFF_W4] = rng.normal(size=64) * 0.3
    params[mo.OFF_B4] = 0.05
    return feat, norm, params.astype(np.float32)


@pytest.mark.parametrize("n,seed", [(1, 0), (1000, 1), (592 * 128 + 77, 2)])
def test_forward_matches_oracle(n, seed):
    import torch
    feat, norm, params = _case(n, seed)
    d_feat = torch.from_numpy(feat).cuda()
    d_out = torch.full((n,), float("nan"), device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.call("sphpc_mlp_forward", _fptr(d_feat), n,
              params.ctypes.data_as(C.POINTER(C.c_float)),
              norm.ctypes.data_as(C.POINTER(C.c_float)), _fptr(d_out), stream)
    torch.cuda.synchronize()
    got = d_out.cpu().numpy().astype(np.float64)
    ref, _ = mo.forward(params, norm, feat, bf16_emulation=True)
    exact, _ = mo.forward(params, norm, feat, bf16_emulation=False)
    assert np.all(np.isfinite(got))
    scale = max(np.abs(ref).max(), 1e-3)
    # bf16 activations: the tensor cores' FP32 accumulation order can move a hidden
    # value across a bf16 rounding boundary (one 2^-8 step, or a ReLU gate near 0);
    # the output then moves by well under 1% of its range
    err = np.abs(got - ref)
    assert err.max() <= 1e-2 * scale, err.max() / scale
    assert np.median(err) <= 1e-3 * scale
    # and the bf16 network stays within a few percent of the float64 one
    assert np.abs(got - exact).max() <= 5e-2 * max(np.abs(exact).max(), 1e-3)


def _grad_case(n, seed):
    feat, norm, params = _case(n, seed)
    rng = np.random.default_rng(seed + 100)
    target = (np.tanh(feat[:, 0] * 0.3) * 0.5 + 0.1 * feat[:, 1] * norm[mo.N_IN + 1]
              + 0.05 * rng.normal(size=n)).astype(np.float32)
    return feat, norm, params, target


@pytest.mark.parametrize("n,seed", [(1000, 5), (148 * 128 * 2 + 300, 6)])
def test_gradient_matches_oracle(n, seed):
    """Backward pass and weight gradients on the tensor cores (MN-major
    operand reads) against the oracle's gradient of the same bf16 network."""
    import torch
    feat, norm, params, target = _grad_case(n, seed)
    d_feat = torch.from_numpy(feat).cuda()
    d_tgt = torch.from_numpy(target).cuda()
    grad = np.zeros(mo.N_PARAMS, np.float32)
    loss = C.c_float(0.0)
    F = C.POINTER(C.c_float)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.call("sphpc_mlp_grad", _fptr(d_feat), _fptr(d_tgt), n, params.ctypes.data_as(F),
              norm.ctypes.data_as(F), grad.ctypes.data_as(F), C.byref(loss), stream)
    want_loss, want = mo.loss_and_grad(params, norm, feat, target, bf16_emulation=True)
    assert abs(loss.value - want_loss) <= 2e-3 * want_loss
    blocks = {"W1": (mo.OFF_W1, mo.OFF_B1), "b1": (mo.OFF_B1, mo.OFF_W2),
              "W2": (mo.OFF_W2, mo.OFF_B2), "b2": (mo.OFF_B2, mo.OFF_W3),
              "W3": (mo.OFF_W3, mo.OFF_B3), "b3": (mo.OFF_B3, mo.OFF_W4),
              "w4": (mo.OFF_W4, mo.OFF_B4), "b4": (mo.OFF_B4, mo.N_PARAMS)}
    rel = {}
    for k, (a, b) in blocks.items():
        g, w = grad[a:b].astype(np.float64), want[a:b]
        rel[k] = np.linalg.norm(g - w) / max(np.linalg.norm(w), 1e-30)
    print(rel)
    # one bf16 step (2^-8) on a few activations or pre-activation gradients
    # moves a block's gradient by well under 3%
    assert max(rel.values()) < 3e-2, rel
    cos = grad @ want / (np.linalg.norm(grad) * np.linalg.norm(want))
    assert cos > 0.999


def _dataset(rows_feat, rows_target):
    from sphpc_b200 import warm_start as ws
    ws.dataset_reserve(len(rows_target))
    ws.dataset_clear()
    ws.dataset_append(rows_feat, rows_target)
    return ws


def test_dataset_round_trip_and_stats():
    feat, norm, params, target = _grad_case(5000, 7)
    ws = _dataset(feat, target)
    assert ws.dataset_size() == 5000
    f, t = ws.dataset_read(1234, 100)
    assert np.array_equal(f, feat[1234:1334]) and np.array_equal(t, target[1234:1334])
    s = ws.dataset_stats()
    np.testing.assert_allclose(s[:16], feat.astype(np.float64).mean(0), rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(s[16:32], 1.0 / feat.astype(np.float64).std(0), rtol=1e-4)
    np.testing.assert_allclose(s[32], target.astype(np.float64).std(), rtol=1e-4)
    ws.dataset_clear()
    assert ws.dataset_size() == 0


def test_adamw_steps_match_oracle():
    """Three full-batch AdamW steps of the trainer against the oracle's
    AdamW on the oracle's gradients (bf16 network)."""
    n, steps, lr, wd = 4096, 3, 1e-3, 1e-4
    feat, norm, params, target = _grad_case(n, 8)
    ws = _dataset(feat, target)
    got, losses = ws.train(params, norm, steps, batch=n, lr=lr, weight_decay=wd, seed=3)
    p = params.copy()
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    want_losses = []
    for k in range(1, steps + 1):
        L, g = mo.loss_and_grad(p, norm, feat, target, bf16_emulation=True)
        want_losses.append(L)
        p, m, v = mo.adamw_step(p, g, m, v, k, lr=lr, wd=wd)
    np.testing.assert_allclose(losses, want_losses, rtol=2e-3)
    d = np.abs(got.astype(np.float64) - p)
    # Adam moves every parameter by about lr per step whatever the gradient's
    # size, so a gradient that differs in the bf16 noise can flip a tiny
    # component's step: bound the typical and the rare differences
    assert np.mean(d) < 0.05 * lr * steps, np.mean(d)
    assert np.mean(d > 0.5 * lr * steps) < 0.02
    ws.dataset_clear()


def test_training_fits_a_smooth_target():
    feat, norm, params, target = _grad_case(32768, 9)
    target = (np.sin(feat[:, 0] * norm[16]) + 0.5 * np.tanh(feat[:, 3] * norm[19])
              - 0.3 * (feat[:, 5] * norm[21]) ** 2).astype(np.float32)
    ws = _dataset(feat, target)
    nrm = ws.dataset_stats()
    out, losses = ws.train(params, nrm, 400, batch=4096, lr=3e-3, weight_decay=0.0, seed=1)
    assert np.all(np.isfinite(losses))
    assert losses[-20:].mean() < 0.1 * losses[:5].mean(), (losses[:5], losses[-20:])
    ws.dataset_free()
