"""Mesh signed distance (sphpc_mesh_sdf): the CPU oracle against analytic
distances (CPU), and the device kernel against both (GPU)."""
import numpy as np
import pytest

from oracle import meshsdf_oracle as mso


def cube_mesh(h=1.0):
    """Closed cube [-h, h]^3, outward-facing triangles."""
    v = np.array([[x, y, z] for z in (-h, h) for y in (-h, h) for x in (-h, h)], np.float32)
    quads = [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]
    t = []
    for a, b, c, d in quads:
        t += [(a, b, c), (a, c, d)]
    return v, np.array(t, np.int32)


def icosphere(levels=2, r=1.0):
    p = (1 + 5 ** 0.5) / 2
    v = [(-1, p, 0), (1, p, 0), (-1, -p, 0), (1, -p, 0), (0, -1, p), (0, 1, p), (0, -1, -p),
         (0, 1, -p), (p, 0, -1), (p, 0, 1), (-p, 0, -1), (-p, 0, 1)]
    v = [np.array(x, float) / np.linalg.norm(x) for x in v]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
         (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
         (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(levels):
        cache, nf = {}, []
        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = v[a] + v[b]
                v.append(m / np.linalg.norm(m))
                cache[key] = len(v) - 1
            return cache[key]
        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    return (np.array(v) * r).astype(np.float32), np.array(f, np.int32)


def box_sdf(p, h=1.0):
    q = np.abs(p) - h
    outside = np.linalg.norm(np.maximum(q, 0.0), axis=-1)
    inside = np.minimum(np.max(q, axis=-1), 0.0)
    return outside + inside


GRID = ((9, 7, 8), (-1.9, -1.6, -1.7), 0.45)


def _points(dims, origin, dx):
    k, j, i = np.meshgrid(range(dims[2]), range(dims[1]), range(dims[0]), indexing="ij")
    return np.stack([origin[0] + i * dx, origin[1] + j * dx, origin[2] + k * dx], -1).reshape(-1, 3)


def test_oracle_cube_matches_analytic():
    v, t = cube_mesh()
    dims, origin, dx = GRID
    got = mso.grid_sdf(v, t, dims, origin, dx)
    want = box_sdf(_points(dims, origin, dx))
    assert np.allclose(got, want, atol=1e-9)


def test_oracle_sphere_sign_and_faceting():
    v, t = icosphere(2)
    dims, origin, dx = GRID
    got = mso.grid_sdf(v, t, dims, origin, dx)
    r = np.linalg.norm(_points(dims, origin, dx), axis=1)
    # the 320-face sphere lies between radius ~0.98 and 1
    assert np.all(np.abs(got - (r - 1.0)) < 0.03)
    assert np.all(np.sign(got[np.abs(r - 1) > 0.05]) == np.sign(r - 1)[np.abs(r - 1) > 0.05])


@pytest.mark.gpu
@pytest.mark.parametrize("mesh", ["cube", "sphere"])
def test_device_sdf_matches_oracle(mesh):
    from sphpc_b200 import meshsdf
    v, t = cube_mesh() if mesh == "cube" else icosphere(2)
    dims, origin, dx = GRID
    got = meshsdf.mesh_sdf(v, t, dims, origin, dx).astype(np.float64)
    want = mso.grid_sdf(v, t, dims, origin, dx)
    assert np.max(np.abs(np.abs(got) - np.abs(want))) < 2e-6
    far = np.abs(want) > 1e-3
    assert np.all(np.sign(got[far]) == np.sign(want[far]))


@pytest.mark.gpu
def test_device_sdf_writes_a_loadable_obstacle(tmp_path):
    """A mesh-made SDFGen file drives the obstacle path (AllocInitObstacle)."""
    from sphpc_b200 import meshsdf
    from sphpc_b200.scenes import write_sdfgen
    v, t = icosphere(2, r=1.0)
    dims, origin = meshsdf.sdfgen_grid(v, 0.1, 3)
    phi = meshsdf.mesh_sdf(v, t, dims, origin, 0.1)
    assert phi.min() < -0.9 and phi.max() > 0.3
    path = tmp_path / "sphere.sdf"
    write_sdfgen(str(path), dims, origin, 0.1, phi)
    import ctypes as C
    from sphpc_b200._lib import Obstacle, call
    ob = Obstacle()
    ob.SDF_file_name = str(path).encode()
    ob.world_bounds.min_x, ob.world_bounds.max_x = 10.0, 20.0
    call("AllocInitObstacle", C.byref(ob))
    try:
        assert (ob.SDF_dim_x, ob.SDF_dim_y, ob.SDF_dim_z) == tuple(dims)
        assert ob.SDF_spacing == pytest.approx(0.1)
        buf = np.ctypeslib.as_array(ob.SDF_buffer, shape=(int(np.prod(dims)),))
        assert np.allclose(buf, phi, rtol=1e-7, atol=1e-8)
    finally:
        call("FinalizeObstacle", C.byref(ob))
