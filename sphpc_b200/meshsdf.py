"""Signed distance fields of triangle meshes for the SDF obstacle, computed
on the device (sphpc_mesh_sdf) and written in the SDFGen format the
obstacle loader reads (obstacle.c:13-79).

    python -m sphpc_b200.meshsdf mesh.obj DX PADDING out.sdf

Grid as SDFGen builds it: the mesh's bounding box grown by PADDING cells of
size DX on every side, origin at its minimum corner, (extent / DX) samples
per axis (truncated).
"""
from __future__ import annotations

import ctypes as C
import sys

import numpy as np

from ._lib import call
from .scenes import write_sdfgen


def read_obj(path):
    """Vertices (nv, 3) float32 and triangles (nt, 3) int32 of a Wavefront OBJ
    (v and f records; polygons split into fans; 1-based or negative indices)."""
    verts, tris = [], []
    with open(path) as f:
        for line in f:
            parts = line.split()
            if not parts:
                continue
            if parts[0] == "v":
                verts.append([float(x) for x in parts[1:4]])
            elif parts[0] == "f":
                ids = []
                for tok in parts[1:]:
                    v = int(tok.split("/")[0])
                    ids.append(v - 1 if v > 0 else len(verts) + v)
                for t in range(1, len(ids) - 1):
                    tris.append([ids[0], ids[t], ids[t + 1]])
    return np.asarray(verts, np.float32), np.asarray(tris, np.int32)


def sdfgen_grid(verts, dx, padding):
    lo = np.asarray(verts, np.float64).min(axis=0) - padding * dx
    hi = np.asarray(verts, np.float64).max(axis=0) + padding * dx
    dims = tuple(int(x) for x in ((hi - lo) / dx))
    return dims, tuple(float(x) for x in lo)


def mesh_sdf(verts, tris, dims, origin, dx):
    """phi (float32, i fastest) at origin + (i, j, k) dx, negative inside."""
    v = np.ascontiguousarray(verts, np.float32)
    t = np.ascontiguousarray(tris, np.int32)
    d = (C.c_int * 3)(*dims)
    o = (C.c_double * 3)(*origin)
    phi = np.zeros(int(np.prod(dims)), np.float32)
    call("sphpc_mesh_sdf", v.ctypes.data_as(C.POINTER(C.c_float)), len(v),
         t.ctypes.data_as(C.POINTER(C.c_int)), len(t), d, o, float(dx),
         phi.ctypes.data_as(C.POINTER(C.c_float)))
    return phi


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 4:
        print(__doc__)
        return 2
    mesh, dx, padding, out = argv[0], float(argv[1]), int(argv[2]), argv[3]
    verts, tris = read_obj(mesh)
    dims, origin = sdfgen_grid(verts, dx, padding)
    phi = mesh_sdf(verts, tris, dims, origin, dx)
    write_sdfgen(out, dims, origin, dx, phi)
    print(f"{mesh}: {len(tris)} triangles -> {out}: {dims[0]}x{dims[1]}x{dims[2]} samples")
    return 0


if __name__ == "__main__":
    sys.exit(main())
