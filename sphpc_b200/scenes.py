"""Synthetic scenes: the configuration files under configs/ and the signed
distance fields their [Obstacle] sections name.

The reference ships one obstacle, Runtime/bunny_watertight.sdf, which is not
in its tree, so the obstacle scenes use an analytic union of a torus (axis
along y) and a sphere, sampled in FP32 and written in SDFGen's ASCII format
(the format AllocInitObstacle parses, obstacle.c:13-79: "nx ny nz", origin,
spacing, then nx*ny*nz values with x fastest).  Sample (i, j, k) sits at the
texel centre min + (i + 0.5) * spacing, where the reference's normalised
tex3D lookup (obstacle_cuda.cu:74-88) reads it, and the model length
dim_x * spacing equals the world length so model distances are world
distances.
"""
from __future__ import annotations

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CONFIG_DIR = os.path.join(HERE, "configs")

# name -> (dims, world min, spacing, sphere (centre, radius), torus (centre, R, r))
SDF_SCENES = {
    "torus_sphere_config3": ((128, 64, 128), (0.0, 0.0, 0.0), 3.0,
                             ((192.0, 30.0, 192.0), 30.0), ((192.0, 12.0, 192.0), 40.0, 12.0)),
    "torus_sphere_config5": ((256, 64, 128), (0.0, 0.0, 0.0), 6.0,
                             ((768.0, 120.0, 384.0), 120.0), ((768.0, 48.0, 384.0), 160.0, 48.0)),
    "torus_sphere_small": ((64, 32, 64), (0.0, 0.0, 0.0), 1.5,
                           ((48.0, 7.5, 48.0), 7.5), ((48.0, 3.0, 48.0), 10.0, 3.0)),
}

# Named workloads (configuration files under configs/).
CONFIGS = {
    "dam_break_32k": "dam_break_32k.ini",      # 32,768 particles, CPU-runnable size
    "dam_break_1m": "dam_break_1m.ini",        # 1,048,576 particles
    "obstacle_4m": "obstacle_4m.ini",          # 4,194,304 particles + SDF + tension
    "full_16m": "full_16m.ini",                # 16,777,216 particles, full pipeline
    "small_dam": "small_dam.ini",
    "small_obstacle": "small_obstacle.ini",
    "reference_compat": "reference_compat.ini",
}


def torus_sphere_sdf(dims, wmin, spacing, sphere, torus):
    """Signed distance (negative inside) of sphere U torus at texel centres,
    FP32, flattened x fastest."""
    nx, ny, nz = dims
    x = wmin[0] + (np.arange(nx, dtype=np.float64) + 0.5) * spacing
    y = wmin[1] + (np.arange(ny, dtype=np.float64) + 0.5) * spacing
    z = wmin[2] + (np.arange(nz, dtype=np.float64) + 0.5) * spacing
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    (sc, sr), (tc, R, r) = sphere, torus
    ds = np.sqrt((X - sc[0]) ** 2 + (Y - sc[1]) ** 2 + (Z - sc[2]) ** 2) - sr
    qx = np.sqrt((X - tc[0]) ** 2 + (Z - tc[2]) ** 2) - R
    qy = Y - tc[1]
    dt = np.sqrt(qx * qx + qy * qy) - r
    return np.minimum(ds, dt).astype(np.float32).reshape(-1)


def write_sdfgen(path, dims, origin, spacing, values):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + f".tmp{os.getpid()}"
    with open(tmp, "w") as f:
        f.write(f"{dims[0]} {dims[1]} {dims[2]}\n")
        f.write(f"{origin[0]:.9g} {origin[1]:.9g} {origin[2]:.9g}\n")
        f.write(f"{spacing:.9g}\n")
        f.write("\n".join(np.char.mod("%.9g", values)))
        f.write("\n")
    os.replace(tmp, path)


def sdf_path(name):
    return os.path.join(CONFIG_DIR, "_sdf", name + ".sdf")


def ensure_sdf(name):
    """Writes configs/_sdf/<name>.sdf if it does not exist yet; returns its path."""
    path = sdf_path(name)
    if not os.path.exists(path):
        dims, wmin, spacing, sphere, torus = SDF_SCENES[name]
        vals = torus_sphere_sdf(dims, wmin, spacing, sphere, torus)
        origin = tuple(w + 0.5 * spacing for w in wmin)
        write_sdfgen(path, dims, origin, spacing, vals)
    return path


def config_path(name):
    """Path of a named configuration, with the SDF it needs generated."""
    path = os.path.join(CONFIG_DIR, CONFIGS.get(name, name))
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    with open(path) as f:
        for line in f:
            s = line.split("#")[0].strip()
            if s.startswith("SDF_file_name"):
                fn = s.split("=", 1)[1].strip()
                base = os.path.splitext(os.path.basename(fn))[0]
                if base in SDF_SCENES:
                    ensure_sdf(base)
    return path
