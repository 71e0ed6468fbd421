"""Particle-to-level-set surface (sphpc_particle_surface) against its numpy
restatement (the dense-grid form of ConstructSurface.cc's operations)."""
import numpy as np
import pytest

from oracle import surface_oracle as so


def _blob(seed=0):
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(range(5), range(4), range(6), indexing="ij"), -1).reshape(-1, 3)
    return (g + rng.uniform(-0.05, 0.05, g.shape) + [3.0, 2.0, 1.0]).astype(np.float64)


def test_oracle_shape_of_a_blob():
    xyz = _blob()
    r, hw = 1.0, 2
    voxel = r / 2
    pad = hw * voxel + 2 * r
    lo = xyz.min(0) - pad
    dims = tuple(int(x) for x in np.ceil((xyz.max(0) + pad - lo) / voxel) + 1)
    phi = so.surface(xyz, r, hw, dims, lo).reshape(dims[2], dims[1], dims[0])
    # the centre of the blob is inside, the grid corner outside
    c = ((xyz.mean(0) - lo) / voxel).round().astype(int)
    assert phi[c[2], c[1], c[0]] < 0 and phi[0, 0, 0] > 0


@pytest.mark.gpu
@pytest.mark.parametrize("radius", [1.0, 0.75])
def test_device_surface_matches_oracle(radius):
    from sphpc_b200 import surface
    xyz = _blob(1)
    phi, dims, origin = surface.particle_surface(xyz, radius)
    want = so.surface(xyz, radius, 2, dims, origin)
    # fixed-point minimum (2^-20) and FP32 distances / means
    assert np.max(np.abs(phi - want)) < 2e-5
    assert (phi < 0).sum() == (want < 0).sum() or np.max(np.abs(want[(phi < 0) != (want < 0)])) < 2e-5
