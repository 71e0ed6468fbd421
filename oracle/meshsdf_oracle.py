"""CPU oracle of the mesh signed-distance tool (test infrastructure, not
product code): float64 numpy restatement of sphpc_mesh_sdf
(sphpc_b200/csrc/meshsdf.cu), which has no counterpart in the reference
(its obstacle loader, obstacle.c:13-79, reads SDFGen files made by an
external tool).

The distance is computed independently of the kernel's Voronoi-region
method: the projection onto the triangle's plane when it falls inside the
triangle, otherwise the nearest of the three edge segments.  The sign is
the generalized winding number (sum of solid angles / 4 pi > 1/2: inside).
"""
import numpy as np


def _seg_dist2(p, a, b):
    ab = b - a
    t = np.clip(np.einsum("ij,ij->i", p - a, ab) / np.maximum(np.einsum("ij,ij->i", ab, ab), 1e-300),
                0.0, 1.0)
    q = a + t[:, None] * ab
    d = p - q
    return np.einsum("ij,ij->i", d, d)


def point_sdf(p, tri):
    """Signed distance of one point p (3,) to the closed mesh tri (nt, 3, 3)."""
    a, b, c = tri[:, 0], tri[:, 1], tri[:, 2]
    P = np.broadcast_to(p, a.shape)
    n = np.cross(b - a, c - a)
    nn = np.einsum("ij,ij->i", n, n)
    s = np.einsum("ij,ij->i", P - a, n) / np.maximum(nn, 1e-300)
    q = P - s[:, None] * n
    # barycentric test of the projection
    def edge_side(u, v):
        return np.einsum("ij,ij->i", np.cross(v - u, q - u), n)
    inside = (edge_side(a, b) >= 0) & (edge_side(b, c) >= 0) & (edge_side(c, a) >= 0)
    d_plane = s * s * nn
    d_edges = np.minimum(np.minimum(_seg_dist2(P, a, b), _seg_dist2(P, b, c)), _seg_dist2(P, c, a))
    d2 = np.where(inside, d_plane, d_edges)
    ra, rb, rc = a - P, b - P, c - P
    la, lb, lc = (np.linalg.norm(x, axis=1) for x in (ra, rb, rc))
    num = np.einsum("ij,ij->i", ra, np.cross(rb, rc))
    den = (la * lb * lc + np.einsum("ij,ij->i", ra, rb) * lc + np.einsum("ij,ij->i", ra, rc) * lb
           + np.einsum("ij,ij->i", rb, rc) * la)
    wind = np.sum(2.0 * np.arctan2(num, den)) / (4.0 * np.pi)
    return (-1.0 if abs(wind) > 0.5 else 1.0) * np.sqrt(d2.min())


def grid_sdf(verts, tris, dims, origin, dx):
    tri = np.asarray(verts, np.float64)[np.asarray(tris)]
    out = np.zeros(dims[0] * dims[1] * dims[2])
    idx = 0
    for k in range(dims[2]):
        for j in range(dims[1]):
            for i in range(dims[0]):
                p = np.array([origin[0] + i * dx, origin[1] + j * dx, origin[2] + k * dx])
                out[idx] = point_sdf(p, tri)
                idx += 1
    return out
