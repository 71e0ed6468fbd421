"""The neighbour build's FP32 candidate pre-test (no GPU needed).

The build decides r^2 < h^2 (FillNeighbors, neighbors.c:278-285, FP64) from
FP32 copies of the absolute positions and sends only the pairs whose FP32
r^2 lies within h^2 (1 -+ 2^-10) to the exact FP64 test.  The host query
sphpc_neighbor_pretest_fp32_safe says for which coordinate magnitudes that
is exact; beyond it the build tests every pair in FP64.  These checks hold
the query against an emulation of the kernel's FP32 arithmetic on pairs
placed at r = h, where a wrong decision would change a bucket.
"""
import numpy as np
import pytest

from sphpc_b200 import _lib
from sphpc_b200.scenes import CONFIGS, config_path
from oracle.pyoracle import scene_from_ini


def _safe(m, h):
    return _lib.load().sphpc_neighbor_pretest_fp32_safe(float(m), float(h)) == 1


def _fp32_r2(xp, xq):
    """FP32 r^2 as the kernel forms it: fx*fx + fy*fy + fz*fz contracted to
    fma(fz, fz, fma(fy, fy, fx*fx)), every operation rounded to FP32."""
    f = np.float32
    xp32 = xp.astype(f)
    xq32 = xq.astype(f)
    d = (xp32 - xq32).astype(f)                      # three FP32 subtractions
    d64 = d.astype(np.float64)
    r = (d64[:, 0] * d64[:, 0]).astype(f)             # FMUL
    r = (d64[:, 1] * d64[:, 1] + r.astype(np.float64)).astype(f)   # FFMA
    r = (d64[:, 2] * d64[:, 2] + r.astype(np.float64)).astype(f)   # FFMA
    return r


def _wrong_decisions(m, h, n=400_000, seed=0):
    """Pairs at |x| ~ m with exact r^2 within 2^-9 h^2 of h^2 that the FP32
    band would decide the wrong way (outside the band on the wrong side)."""
    rng = np.random.default_rng(seed)
    xp = m * (0.5 + 0.5 * rng.random((n, 3)))
    # the pair's FP64 positions are fl64(x + d) of FP32 x and d: any double
    # near m is representable that way, so draw doubles directly
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    r = h * (1.0 + (rng.random(n) - 0.5) * 2.0 ** -9)
    xq = xp + u * r[:, None]
    exact = np.sum((xp - xq) ** 2, axis=1) < h * h
    r2f = _fp32_r2(xp, xq)
    lo = np.float32(np.float32(h * h) * (np.float32(1.0) - np.float32(1.0 / 1024.0)))
    hi = np.float32(np.float32(h * h) * (np.float32(1.0) + np.float32(1.0 / 1024.0)))
    said_yes = r2f < lo
    said_no = r2f > hi
    return int(np.sum(said_yes & ~exact) + np.sum(said_no & exact))


def test_pretest_safe_for_every_shipped_config():
    for name in sorted(CONFIGS):
        sc = scene_from_ini(config_path(name))
        p = sc.params
        m = p.h * max(p.nx, p.ny, p.nz)
        assert _safe(m, p.h), name


@pytest.mark.parametrize("h", [2.0, 1.0, 0.0125, 3.0])
def test_pretest_bound_holds_at_its_limit_and_is_needed_beyond(h):
    # the largest power of two the query accepts
    k = 0
    while _safe(h * 2.0 ** (k + 1), h):
        k += 1
    assert 10 <= k <= 14, k
    # the top of the binade that holds h 2^k: the same FP32 spacing, so the
    # largest coordinate the accepted spacing covers
    m_ok = 2.0 ** (np.floor(np.log2(h * 2.0 ** k)) + 1) * (1 - 2.0 ** -30)
    assert _safe(m_ok, h)
    assert _wrong_decisions(m_ok, h) == 0
    # far beyond the limit the FP32 test really does decide pairs wrongly,
    # which is why the build then sends every pair to the FP64 test
    m_bad = h * 2.0 ** (k + 6)
    assert not _safe(m_bad, h)
    assert _wrong_decisions(m_bad, h) > 0


def test_pretest_rejects_nonsense():
    assert not _safe(-1.0, 2.0)
    assert not _safe(100.0, 0.0)
    assert not _safe(float("inf"), 2.0)
