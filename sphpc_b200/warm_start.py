"""Learned warm start of the PBF constraint solve: the network file, the
device-resident training set and the trainer, over the C ABI.

The network maps 16 features of a particle's predicted neighbourhood to the
stiffness-weighted multiplier sum Lambda = sum_k s_k lambda_k of a plain solve
(lambda_k and s_k as in ComputeLambda / UpdateDPs, particles.c:588-746); one
position pass with Lambda at stiffness 1 then stands in for the first
iterations of the plain solve.  Parameter vector (FP32, 9473 values):
W1[64][16] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] w4[64] b4, and the
normalisation norm[33] = feature means, 1/standard deviations, target
standard deviation.
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np

from ._lib import call, load

N_IN = 16
N_HID = 64
N_PARAMS = N_HID * N_IN + N_HID + 2 * (N_HID * N_HID + N_HID) + N_HID + 1
N_NORM = 2 * N_IN + 1
WEIGHTS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights")
DEFAULT_WEIGHTS = os.path.join(WEIGHTS_DIR, "warm_start.npz")

FEATURES = (
    "rho/rho0 - 1", "C", "lambda", "sum |grad_q C|^2", "|grad_p C|^2", "neighbour count",
    "mean offset x / h", "mean offset y / h", "mean offset z / h",
    "mean rel. displacement x / h", "mean rel. displacement y / h",
    "mean rel. displacement z / h", "SDF / h", "nearest neighbour / h", "wall distance / h",
    "own displacement along gravity / h",
)

_F = C.POINTER(C.c_float)


def _fp(a):
    return a.ctypes.data_as(_F)


def init_params(seed: int = 0) -> np.ndarray:
    """Uniform +-1/sqrt(fan_in) weights, zero biases (float32)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    off = 0
    for fan_out, fan_in in ((N_HID, N_IN), (N_HID, N_HID), (N_HID, N_HID), (1, N_HID)):
        lim = 1.0 / np.sqrt(fan_in)
        p[off:off + fan_out * fan_in] = rng.uniform(-lim, lim, fan_out * fan_in)
        off += fan_out * fan_in + (fan_out if fan_out > 1 else 0)
    return p


def save_network(path: str, params: np.ndarray, norm: np.ndarray, meta: dict | None = None):
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    np.savez(path, params=np.asarray(params, np.float32), norm=np.asarray(norm, np.float32),
             meta=np.frombuffer(json.dumps(meta or {}).encode(), np.uint8))


def load_network(path: str = DEFAULT_WEIGHTS):
    """(params[9473], norm[33], meta dict) from a file written by save_network."""
    with np.load(path) as z:
        params = z["params"].astype(np.float32)
        norm = z["norm"].astype(np.float32)
        meta = json.loads(bytes(z["meta"]).decode()) if "meta" in z else {}
    if params.shape != (N_PARAMS,) or norm.shape != (N_NORM,):
        raise ValueError(f"{path}: expected {N_PARAMS} parameters and {N_NORM} norm values")
    return params, norm, meta


# ---------------- training set ----------------
def dataset_reserve(capacity: int):
    call("sphpc_mlp_dataset_reserve", int(capacity))


def dataset_size() -> int:
    n = C.c_longlong(0)
    call("sphpc_mlp_dataset_size", C.byref(n))
    return n.value


def dataset_clear():
    call("sphpc_mlp_dataset_clear")


def dataset_free():
    call("sphpc_mlp_dataset_free")


def dataset_append(feat: np.ndarray, target: np.ndarray):
    feat = np.ascontiguousarray(feat, np.float32).reshape(-1, N_IN)
    target = np.ascontiguousarray(target, np.float32).reshape(-1)
    if len(feat) != len(target):
        raise ValueError("feature and target row counts differ")
    call("sphpc_mlp_dataset_append", _fp(feat), _fp(target), len(target))


def dataset_read(offset: int, count: int):
    feat = np.zeros((count, N_IN), np.float32)
    target = np.zeros(count, np.float32)
    call("sphpc_mlp_dataset_read", int(offset), int(count), _fp(feat), _fp(target))
    return feat, target


def dataset_stats() -> np.ndarray:
    norm = np.zeros(N_NORM, np.float32)
    call("sphpc_mlp_dataset_stats", _fp(norm))
    return norm


def train(params: np.ndarray, norm: np.ndarray, steps: int, batch: int = 65536,
          lr: float = 1e-3, weight_decay: float = 1e-4, seed: int = 0,
          lr_final: float | None = None):
    """AdamW on the training set, learning rate from lr to lr_final (default:
    constant lr) on a half cosine; returns (params, per-step batch loss)."""
    p_in = np.ascontiguousarray(params, np.float32)
    nrm = np.ascontiguousarray(norm, np.float32)
    out = np.zeros(N_PARAMS, np.float32)
    loss = np.zeros(max(steps, 1), np.float32)
    call("sphpc_mlp_train", _fp(p_in), _fp(nrm), int(steps), int(batch), float(lr),
         float(lr if lr_final is None else lr_final), float(weight_decay), C.c_ulonglong(seed),
         _fp(out), _fp(loss))
    return out, loss[:steps]


def collect(sim, iterations: int) -> int:
    """One step of `sim` with the plain solver at `iterations`, appending one
    training row per particle; returns the rows appended."""
    rc = load().sphpc_mlp_collect(C.byref(sim.particles), C.byref(sim.params),
                                  C.byref(sim.neighbors), C.byref(sim.boundary), sim._ob(),
                                  int(iterations))
    if rc < 0:
        from ._lib import check
        check("sphpc_mlp_collect", rc)
    return rc
