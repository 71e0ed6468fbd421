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
    # bf16 activations: tanh.approx against exact tanh can move a hidden value by one
    # bf16 step (2^-8 relative); the output then moves by well under 1% of its range
    err = np.abs(got - ref)
    assert err.max() <= 1e-2 * scale, err.max() / scale
    assert np.median(err) <= 1e-3 * scale
    # and the bf16 network stays within a few percent of the float64 one
    assert np.abs(got - exact).max() <= 5e-2 * max(np.abs(exact).max(), 1e-3)
