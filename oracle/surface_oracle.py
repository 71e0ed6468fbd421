"""CPU oracle of the surface reconstruction (test infrastructure, not
product code): float64 numpy restatement of sphpc_particle_surface
(sphpc_b200/csrc/surface.cu), the dense-grid form of the operations in
PostProcessing/OpenVDB/src/ConstructSurface.cc:39-72 (rasterise spheres,
offset(-r), gaussian(), offset(+r)).  The OpenVDB original is not
available here, so the restatement is pinned only to its own definition
(parity against OpenVDB is unpinned)."""
import numpy as np


def rasterise(xyz, radius, half_width, dims, origin):
    voxel = radius / 2.0
    band = half_width * voxel + radius
    xyz = np.asarray(xyz, np.float64).reshape(-1, 3)
    k, j, i = np.meshgrid(range(dims[2]), range(dims[1]), range(dims[0]), indexing="ij")
    pts = np.stack([origin[0] + i * voxel, origin[1] + j * voxel, origin[2] + k * voxel], -1)
    phi = np.full(pts.shape[:3], band)
    for p in xyz:
        d = np.linalg.norm(pts - p, axis=-1) - radius
        phi = np.minimum(phi, np.where(d > band, band, np.maximum(d, -band)))
    return phi  # [k][j][i]


def mean3(a, axis):
    lo = np.concatenate([np.take(a, [0], axis), np.take(a, range(a.shape[axis] - 1), axis)], axis)
    hi = np.concatenate([np.take(a, range(1, a.shape[axis]), axis), np.take(a, [-1], axis)], axis)
    return (lo + a + hi) / 3.0


def surface(xyz, radius, half_width, dims, origin):
    phi = rasterise(xyz, radius, half_width, dims, origin) - radius
    for _ in range(3):
        for axis in (2, 1, 0):   # x, y, z in [k][j][i] order
            phi = mean3(phi, axis)
    return (phi + radius).ravel()
