"""The surface reconstruction (ConstructSurface.cc:39-72: spheres of radius r
rasterised at voxel r/2 with a narrow band, offset(-r), gaussian(),
offset(+r)) pinned to closed forms on isolated and overlapping spheres.

The rasterised level set of spheres is the union's distance function
phi0(x) = min_i (|x - p_i| - r), clamped to the band (band = 2 voxels + r).
On the dense grid the smoothing is linear and keeps constants (three 3-tap
means per axis with the edge value repeated: one 7-tap kernel
[1, 3, 6, 7, 6, 3, 1] / 27 per axis), so the dilation by r and the erosion
by r cancel and the result is that smoothing applied to phi0 (each pass
repeating the edge value, so the 7-tap form holds away from the faces).  Both the numpy
oracle (oracle/surface_oracle.py) and the device (sphpc_particle_surface)
must equal this formula, evaluated here by a direct convolution of the
analytic phi0.  Two consequences are checked in closed form: a lattice
block's surface lies between 0.5 r and r beyond its outer layer, and an
isolated particle is smoothed away (the kernel's mean offset length, 1.13 r,
exceeds r).  OpenVDB itself re-normalises the level set after each offset
and filter step, which keeps a smaller sphere around an isolated particle;
that sparse-grid bookkeeping is not available here, so these checks pin the
dense form, not OpenVDB's bits.
"""
import numpy as np
import pytest

from oracle import surface_oracle as so

KERNEL = np.array([1, 3, 6, 7, 6, 3, 1], np.float64) / 27.0


def _grid(xyz, radius, half_width=2):
    voxel = radius / 2.0
    pad = half_width * voxel + 2.0 * radius
    xyz = np.asarray(xyz, np.float64).reshape(-1, 3)
    lo = xyz.min(axis=0) - pad
    dims = tuple(int(x) for x in np.ceil((xyz.max(axis=0) + pad - lo) / voxel) + 1)
    return dims, lo


def _phi0(xyz, radius, dims, origin, half_width=2):
    """min_i (|x - p_i| - r) clamped to [-band, band], [k][j][i] order."""
    voxel = radius / 2.0
    band = half_width * voxel + radius
    z = origin[2] + voxel * np.arange(dims[2])
    y = origin[1] + voxel * np.arange(dims[1])
    x = origin[0] + voxel * np.arange(dims[0])
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    phi = np.full(Z.shape, band)
    for p in np.asarray(xyz, np.float64).reshape(-1, 3):
        d = np.sqrt((X - p[0]) ** 2 + (Y - p[1]) ** 2 + (Z - p[2]) ** 2) - radius
        phi = np.minimum(phi, np.clip(d, -band, band))
    return phi


def _smooth(phi):
    """Three 3-tap means along every axis, each pass repeating the edge
    value (the 7-tap kernel away from the grid's faces)."""
    out = phi
    for axis in range(3):
        pad = [(0, 0)] * 3
        pad[axis] = (1, 1)
        n = out.shape[axis]
        for _ in range(3):
            q = np.pad(out, pad, mode="edge")
            out = sum(np.take(q, range(t, t + n), axis=axis) for t in range(3)) / 3.0
    return out


def closed_form(xyz, radius, dims, origin):
    return _smooth(_phi0(xyz, radius, dims, origin)).ravel()


def _mean_offset_norm(radius):
    """Kernel-weighted mean of |o| over the 7x7x7 voxel offsets o: the
    smoothed value of |x| - r at an isolated sphere's centre is this minus r."""
    v = radius / 2.0
    o = np.arange(-3, 4) * v
    W = KERNEL[:, None, None] * KERNEL[None, :, None] * KERNEL[None, None, :]
    OZ, OY, OX = np.meshgrid(o, o, o, indexing="ij")
    return float(np.sum(W * np.sqrt(OX ** 2 + OY ** 2 + OZ ** 2)))


SCENES = {
    "isolated": np.array([[0.0, 0.0, 0.0]]),
    "two_isolated": np.array([[0.0, 0.0, 0.0], [9.0, 0.3, -0.2]]),
    "overlapping": np.array([[0.0, 0.0, 0.0], [1.3, 0.2, 0.1], [0.6, 1.1, -0.4]]),
}


@pytest.mark.parametrize("name", sorted(SCENES))
@pytest.mark.parametrize("radius", [1.0, 0.6])
def test_oracle_equals_closed_form(name, radius):
    xyz = SCENES[name] * radius
    dims, origin = _grid(xyz, radius)
    want = closed_form(xyz, radius, dims, origin)
    got = so.surface(xyz, radius, 2, dims, origin)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)


@pytest.mark.parametrize("radius", [1.0, 0.6])
def test_isolated_particle_is_smoothed_away(radius):
    """With voxel r/2 the smoothing kernel's mean offset length is 1.13 r, so
    the smoothed |x - p| - r is positive even at an isolated particle's
    centre: in the dense form (dilation and erosion cancel) a lone particle
    leaves no surface.  (OpenVDB re-normalises after the dilation and keeps
    a smaller sphere; see the module docstring.)"""
    m = _mean_offset_norm(radius)
    assert m > radius
    xyz = SCENES["isolated"] * radius
    dims, origin = _grid(xyz, radius)
    phi = closed_form(xyz, radius, dims, origin)
    assert (phi < 0).sum() == 0
    assert abs(phi.min() - (m - radius)) < 1e-12


@pytest.mark.parametrize("radius", [1.0, 0.6])
def test_lattice_block_surface_sits_outside_its_outer_layer(radius):
    """A block of particles on a lattice of spacing r/2: the union of their
    spheres is nearly a box whose faces are r beyond the outer particles,
    the smoothing of a nearly linear distance leaves the face in place, so
    the zero level along the block's axis lies between 0.5 r and r beyond the
    outer layer."""
    s = radius / 2.0
    g = np.stack(np.meshgrid(*(np.arange(8) * s,) * 3, indexing="ij"), -1).reshape(-1, 3)
    dims, origin = _grid(g, radius)
    phi = closed_form(g, radius, dims, origin).reshape(dims[2], dims[1], dims[0])
    v = radius / 2.0
    mid = np.round((np.full(3, 3.5 * s) - origin) / v).astype(int)
    row = phi[mid[2], mid[1], :]
    k = int(np.argmax((np.arange(dims[0]) * v + origin[0] > 7 * s) & (row > 0)))
    t = (k - 1) + row[k - 1] / (row[k - 1] - row[k])
    beyond = origin[0] + t * v - 7 * s
    assert 0.5 * radius < beyond < radius, beyond


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(SCENES))
def test_device_equals_closed_form(name):
    from sphpc_b200 import surface
    radius = 1.0
    xyz = SCENES[name] * radius + 5.0
    phi, dims, origin = surface.particle_surface(xyz, radius)
    want = closed_form(xyz, radius, dims, np.asarray(origin))
    # fixed-point minimum (2^-20 length units) and FP32 arithmetic
    assert np.max(np.abs(phi - want)) < 2e-5
    assert np.array_equal(phi < 0, want < 0) or \
        np.max(np.abs(want[(phi < 0) != (want < 0)])) < 2e-5
