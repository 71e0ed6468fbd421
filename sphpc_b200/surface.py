"""Particle-to-level-set surface of a snapshot (sim-N.bin, interleaved x, y,
z doubles), computed on the device by sphpc_particle_surface: the
operations of the reference's PostProcessing/OpenVDB/src/ConstructSurface.cc
(voxel size r/2, spheres of radius r, narrow band of 2 voxels, dilate by r,
smooth, erode by r) on a dense grid.

    python -m sphpc_b200.surface sim-0.bin out.lvl [radius]

out.lvl: int32 nx, ny, nz; float64 origin x, y, z; float64 voxel size; then
nx*ny*nz float32 values (x fastest), negative inside.  (The reference writes
OpenVDB's .vdb format, which needs the OpenVDB library.)
"""
from __future__ import annotations

import ctypes as C
import sys

import numpy as np

from ._lib import call


def surface_grid(xyz, radius, half_width=2):
    """Dense grid covering the particles with room for the band and the
    dilation: origin and dims for voxel size radius / 2."""
    voxel = radius / 2.0
    pad = half_width * voxel + 2.0 * radius
    xyz = np.asarray(xyz, np.float64).reshape(-1, 3)
    lo = xyz.min(axis=0) - pad
    hi = xyz.max(axis=0) + pad
    dims = tuple(int(x) for x in np.ceil((hi - lo) / voxel) + 1)
    return dims, tuple(float(x) for x in lo)


def particle_surface(xyz, radius=1.0, half_width=2, dims=None, origin=None):
    xyz = np.ascontiguousarray(np.asarray(xyz, np.float64).reshape(-1))
    if dims is None:
        dims, origin = surface_grid(xyz, radius, half_width)
    phi = np.zeros(int(np.prod(dims)), np.float32)
    d = (C.c_int * 3)(*dims)
    o = (C.c_double * 3)(*origin)
    call("sphpc_particle_surface", xyz.ctypes.data_as(C.POINTER(C.c_double)), len(xyz) // 3,
         float(radius), int(half_width), d, o, phi.ctypes.data_as(C.POINTER(C.c_float)))
    return phi, dims, origin


def write_level_set(path, phi, dims, origin, voxel):
    with open(path, "wb") as f:
        np.asarray(dims, np.int32).tofile(f)
        np.asarray(origin, np.float64).tofile(f)
        np.asarray([voxel], np.float64).tofile(f)
        np.asarray(phi, np.float32).tofile(f)


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) not in (2, 3):
        print(__doc__)
        return 2
    radius = float(argv[2]) if len(argv) == 3 else 1.0
    xyz = np.fromfile(argv[0], dtype=np.float64)
    phi, dims, origin = particle_surface(xyz, radius)
    write_level_set(argv[1], phi, dims, origin, radius / 2.0)
    print(f"{argv[0]}: {len(xyz) // 3} particles -> {argv[1]}: {dims[0]}x{dims[1]}x{dims[2]} "
          f"voxels, {int((phi < 0).sum())} inside")
    return 0


if __name__ == "__main__":
    sys.exit(main())
