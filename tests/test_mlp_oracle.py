"""The warm-start network's CPU oracle: bf16 rounding, finite-difference
gradient check of the float64 variant, and one AdamW step by hand."""
import numpy as np
import pytest

from oracle import mlp_oracle as mo


def _batch(B, seed):
    rng = np.random.default_rng(seed)
    feat = rng.normal(size=(B, mo.N_IN)).astype(np.float32) * rng.uniform(0.5, 3.0, mo.N_IN)
    feat += rng.normal(size=mo.N_IN).astype(np.float32)
    norm = np.concatenate([feat.mean(0), 1.0 / feat.std(0), [0.7]]).astype(np.float32)
    target = rng.normal(size=B).astype(np.float32) * 0.7
    return feat, norm, target


def test_layout():
    assert mo.N_PARAMS == 9473
    q = mo.unpack(np.arange(mo.N_PARAMS, dtype=np.float32))
    assert q["W1"].shape == (64, 16) and q["W1"][1, 0] == 16
    assert q["b4"] == 9472


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -9, -2.5, 1e-30, 3.0e38], np.float32)
    r = mo.bf16(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7 and goes to the even mantissa (1.0)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0 + 2.0 ** -7)
    assert r[3] == -2.5
    assert abs(r[4] - 1e-30) / 1e-30 < 2.0 ** -8
    assert np.all(mo.bf16(r) == r)


@pytest.mark.parametrize("seed", [0, 1])
def test_finite_difference_gradient(seed):
    feat, norm, target = _batch(9, seed)
    p = mo.init_params(seed).astype(np.float64)
    p[mo.OFF_B1:mo.OFF_W2] = 0.1
    _, g = mo.loss_and_grad(p, norm, feat, target, bf16_emulation=False)
    rng = np.random.default_rng(seed + 10)
    idx = np.concatenate([rng.choice(mo.N_PARAMS, 40, replace=False),
                          [mo.OFF_B1, mo.OFF_B2 + 3, mo.OFF_B3 + 63, mo.OFF_W4, mo.OFF_B4]])
    eps = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        lp, _ = mo.loss_and_grad(pp, norm, feat, target, bf16_emulation=False)
        lm, _ = mo.loss_and_grad(pm, norm, feat, target, bf16_emulation=False)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])) + 1e-8, (i, fd, g[i])


def test_bf16_gradient_close_to_exact():
    feat, norm, target = _batch(512, 3)
    p = mo.init_params(3)
    _, g64 = mo.loss_and_grad(p, norm, feat, target, bf16_emulation=False)
    _, g16 = mo.loss_and_grad(p, norm, feat, target, bf16_emulation=True)
    rel = np.linalg.norm(g16 - g64) / np.linalg.norm(g64)
    # BF16 rounding of a pre-activation near 0 flips its ReLU gate, so a few
    # hidden units per batch pass or block their gradient in one form only
    assert rel < 3e-2


def test_adamw_step():
    p = np.array([0.5] * mo.N_PARAMS, np.float32)
    g = np.full(mo.N_PARAMS, 0.2, np.float32)
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    p1, m1, v1 = mo.adamw_step(p, g, m, v, 1, lr=1e-2, wd=0.1)
    # first step: m_hat = g, v_hat = g^2 -> update lr * (sign(g) + wd * p) on weights
    w = mo.OFF_W2 + 5
    b = mo.OFF_B2 + 5
    assert abs(p1[w] - (0.5 - 1e-2 * (0.2 / (0.2 + 1e-8) + 0.1 * 0.5))) < 1e-6
    assert abs(p1[b] - (0.5 - 1e-2 * (0.2 / (0.2 + 1e-8)))) < 1e-6
    assert abs(m1[w] - 0.02) < 1e-7 and abs(v1[w] - 0.2 * 0.2 * 1e-3) < 1e-9
