"""ctypes bindings for the CPU checkers under oracle/.

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py import this module.  The product
(sphpc_b200/libsphpc_cuda.so) never loads these libraries.

* ``OracleSim``  wraps libsphpc_oracle.so, the FP64 restatement of the
  reference path (pbf_oracle.c), or its FP32 build.
* ``RefSim``     wraps oracle/_ref/libsphpc_ref.so, the reference's own
  Simulation/src/particles.c + neighbors.c compiled in place (oracle/Makefile).
* ``scene_from_ini`` restates the reference's parameter set-up
  (input_parser.cc:16-69, simulation.c:130-178, geometry.c:19-74,
  particles.c:1034-1051, obstacle.c:13-79) independently of the product.
"""
from __future__ import annotations

import configparser
import ctypes as C
import math
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MAX_NEIGHBORS = 60


class OracleParams(C.Structure):
    _fields_ = [
        ("h", C.c_double), ("W_norm", C.c_double), ("DelW_norm", C.c_double),
        ("DelW_poly_norm", C.c_double), ("g", C.c_double), ("dt", C.c_double),
        ("gamma", C.c_double), ("dq", C.c_double), ("c", C.c_double),
        ("bmin", C.c_double * 3), ("bmax", C.c_double * 3),
        ("rest_density", C.c_double), ("rest_mass", C.c_double),
        ("solve_iterations", C.c_int), ("scorr_n", C.c_int),
        ("lambda_epsilon", C.c_double), ("scorr_k", C.c_double),
        ("scorr_dq", C.c_double), ("k_stiff", C.c_double),
        ("vorticity_eps", C.c_double), ("v_max", C.c_double),
        ("gravity_axis", C.c_int), ("xsph_mode", C.c_int),
        ("enable_tension", C.c_int), ("enable_vorticity", C.c_int),
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("pad0", C.c_int),
        ("sdf", C.POINTER(C.c_float)), ("sdim", C.c_int * 3), ("pad1", C.c_int),
        ("sdf_spacing", C.c_double), ("ob_min", C.c_double * 3),
        ("ob_max", C.c_double * 3),
    ]


_DP = C.POINTER(C.c_double)
STATE_FIELDS = ["xs", "ys", "zs", "x", "y", "z", "vx", "vy", "vz", "dpx", "dpy",
                "dpz", "wx", "wy", "wz", "cx", "cy", "cz", "rho", "lam"]


class OracleState(C.Structure):
    _fields_ = [("n", C.c_int), ("pad", C.c_int)] + [(f, _DP) for f in STATE_FIELDS]


class OracleNeighbors(C.Structure):
    _fields_ = [("keys", C.POINTER(C.c_uint32)), ("ids", C.POINTER(C.c_uint32)),
                ("start", C.POINTER(C.c_uint32)), ("end", C.POINTER(C.c_uint32)),
                ("nbr", C.POINTER(C.c_uint32)), ("count", C.POINTER(C.c_int32))]


class OracleDiag(C.Structure):
    _fields_ = [("max_density_error", C.c_double), ("mean_density_error", C.c_double),
                ("kinetic_energy", C.c_double), ("com", C.c_double * 3),
                ("momentum", C.c_double * 3)]

    def as_dict(self):
        return {"max_density_error": self.max_density_error,
                "mean_density_error": self.mean_density_error,
                "kinetic_energy": self.kinetic_energy,
                "com": list(self.com), "momentum": list(self.momentum)}


def _load(path):
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built (run `make -C oracle`)")
    return C.CDLL(path)


_LIBS: dict = {}


def oracle_lib(fp32: bool = False):
    key = "f32" if fp32 else "f64"
    if key not in _LIBS:
        lib = _load(os.path.join(HERE, "libsphpc_oracle_f32.so" if fp32 else "libsphpc_oracle.so"))
        P = C.POINTER(OracleParams)
        S = C.POINTER(OracleState)
        N = C.POINTER(OracleNeighbors)
        lib.oracle_uniform01.restype = C.c_double
        lib.oracle_uniform01.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32]
        lib.oracle_lattice.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, _DP,
                                       C.c_double, C.c_uint64, _DP, _DP, _DP]
        lib.oracle_lattice_poly6_sum.restype = C.c_double
        lib.oracle_lattice_poly6_sum.argtypes = [P, C.c_double]
        lib.oracle_hash_val.restype = C.c_uint32
        lib.oracle_hash_val.argtypes = [P, C.c_double, C.c_double, C.c_double]
        lib.oracle_sdf_sample.restype = C.c_float
        lib.oracle_sdf_sample.argtypes = [P, C.c_float, C.c_float, C.c_float]
        lib.oracle_particle_collisions.argtypes = [P, _DP, _DP, _DP, C.c_int]
        lib.oracle_sort_by_key.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.c_int]
        for nm in ("oracle_lower_bounds", "oracle_upper_bounds"):
            getattr(lib, nm).argtypes = [C.POINTER(C.c_uint32), C.c_int, C.c_int,
                                         C.POINTER(C.c_uint32)]
        for nm in ("oracle_apply_gravity", "oracle_predict_positions",
                   "oracle_update_position_stars", "oracle_update_velocities"):
            getattr(lib, nm).argtypes = [P, S]
        for nm in ("oracle_compute_densities", "oracle_compute_lambda",
                   "oracle_surface_tension", "oracle_apply_viscosity",
                   "oracle_compute_vorticity", "oracle_vorticity_confinement",
                   "oracle_find_all_neighbors", "oracle_hash_particles",
                   "oracle_fill_neighbors", "oracle_step"):
            getattr(lib, nm).argtypes = [P, S, N]
        lib.oracle_update_dps.argtypes = [P, S, N, C.c_int]
        lib.oracle_features.argtypes = [P, S, N, _DP]
        lib.oracle_lambda_target.argtypes = [P, S, N, C.c_int, _DP]
        lib.oracle_update_positions.argtypes = [S]
        lib.oracle_diagnostics.argtypes = [P, S, C.POINTER(OracleDiag)]
        lib.oracle_real_size.restype = C.c_int
        _LIBS[key] = lib
    return _LIBS[key]


def ref_lib(fast: bool = False):
    key = "ref_fast" if fast else "ref"
    if key not in _LIBS:
        lib = _load(os.path.join(HERE, "_ref", "libsphpc_ref_fast.so" if fast else "libsphpc_ref.so"))
        lib.ref_create.restype = C.c_void_p
        lib.ref_create.argtypes = [C.POINTER(OracleParams), C.c_int]
        lib.ref_destroy.argtypes = [C.c_void_p]
        lib.ref_set_field.argtypes = [C.c_void_p, C.c_int, _DP]
        lib.ref_get_field.argtypes = [C.c_void_p, C.c_int, _DP]
        U = C.POINTER(C.c_uint32)
        lib.ref_get_neighbors.argtypes = [C.c_void_p, U, U, U, U, U, C.POINTER(C.c_int32)]
        for nm in ("ref_apply_gravity", "ref_predict_positions", "ref_find_all_neighbors",
                   "ref_compute_densities", "ref_compute_lambda",
                   "ref_update_position_stars", "ref_update_velocities",
                   "ref_surface_tension", "ref_apply_viscosity", "ref_compute_vorticity",
                   "ref_vorticity_confinement", "ref_update_positions"):
            getattr(lib, nm).argtypes = [C.c_void_p]
        lib.ref_update_dps.argtypes = [C.c_void_p, C.c_int]
        lib.ref_step.argtypes = [C.c_void_p, C.c_int, C.c_int]
        _LIBS[key] = lib
    return _LIBS[key]


def _ptr(a, ctype=C.c_double):
    return a.ctypes.data_as(C.POINTER(ctype))


# --------------------------------------------------------------------------
# Scene: the reference's parameter set-up, restated in Python
# --------------------------------------------------------------------------

@dataclass
class Scene:
    """Everything the oracle needs for one configuration."""
    params: OracleParams
    x0: np.ndarray      # (3, n) float64 initial positions (original order)
    steps: int
    spacing: float
    sdf: np.ndarray | None = None
    meta: dict = field(default_factory=dict)

    @property
    def n(self):
        return self.x0.shape[1]


def _getf(cp, sec, key, default=None):
    if cp.has_option(sec, key):
        return float(cp.get(sec, key).split("#")[0].strip())
    if default is None:
        raise KeyError(f"{sec}.{key}")
    return float(default)


def _gets(cp, sec, key, default):
    if cp.has_option(sec, key):
        return cp.get(sec, key).split("#")[0].strip()
    return default


def read_sdfgen(path):
    """SDFGen ASCII (obstacle.c:13-79): 'nx ny nz' / origin / dx / values, x fastest."""
    with open(path) as f:
        dims = [int(t) for t in f.readline().split()[:3]]
        origin = [float(t) for t in f.readline().split()[:3]]
        dx = float(f.readline().split()[0])
        vals = np.loadtxt(f, dtype=np.float32, max_rows=dims[0] * dims[1] * dims[2])
    return dims, origin, dx, vals.reshape(-1)


_AXES = {"x": 0, "y": 1, "z": 2, "0": 0, "1": 1, "2": 2}


def scene_from_ini(path: str, fp32_positions: bool = True) -> Scene:
    """Restates ReadParameters + SetParameters + SetParticleNumbers +
    ConstructFluidVolume + AllocInitParticles for one INI file, with the
    build's optional extension keys ([Solver], jitter/seed, rest-density
    mode).  Positions are rounded to FP32 when fp32_positions is set, so the
    oracle sees exactly the values the FP32 device path starts from."""
    cp = configparser.ConfigParser(inline_comment_prefixes=("#", ";"))
    cp.optionxform = str
    with open(path) as f:
        cp.read_string(f.read())
    p = OracleParams()
    steps = int(_getf(cp, "SimParameters", "number_steps"))
    p.dt = _getf(cp, "SimParameters", "time_step")
    n_req = int(_getf(cp, "SimParameters", "number_particles"))
    p.g = _getf(cp, "PhysicalParameters", "g")
    p.c = _getf(cp, "PhysicalParameters", "c")
    p.gamma = _getf(cp, "PhysicalParameters", "k")
    for i, a in enumerate("xyz"):
        p.bmin[i] = _getf(cp, "BoundaryVolume", f"min_{a}")
        p.bmax[i] = _getf(cp, "BoundaryVolume", f"max_{a}")
    fmin = [_getf(cp, "InitialFluidVolume", f"min_{a}") for a in "xyz"]
    fmax = [_getf(cp, "InitialFluidVolume", f"max_{a}") for a in "xyz"]
    jitter = _getf(cp, "InitialFluidVolume", "jitter", 0.0)
    seed = int(_getf(cp, "InitialFluidVolume", "seed", 0))
    # SetParameters, simulation.c:139-155 (spacing is a float there)
    volume = (fmax[0] - fmin[0]) * (fmax[1] - fmin[1]) * (fmax[2] - fmin[2])
    spacing = float(np.float32(math.pow(volume / n_req, 1.0 / 3.0)))
    lib = oracle_lib()
    lib.oracle_set_kernel_norms(C.byref(p), C.c_double(2.0 * spacing))
    # ConstructFluidVolume, geometry.c:19-74 (single rank)
    nl = [int(math.floor((fmax[i] - fmin[i]) / spacing)) for i in range(3)]
    n = nl[0] * nl[1] * nl[2]
    x = np.empty((3, n), np.float64)
    org = (C.c_double * 3)(*fmin)
    lib.oracle_lattice(nl[0], nl[1], nl[2], spacing, org, jitter, seed,
                       _ptr(x[0]), _ptr(x[1]), _ptr(x[2]))
    if fp32_positions:
        x = x.astype(np.float32).astype(np.float64)
    fluid_volume = nl[0] * spacing * nl[1] * spacing * nl[2] * spacing
    # solver constants (reference values by default)
    lib.oracle_params_reference_compat(C.byref(p))
    p.solve_iterations = int(_getf(cp, "Solver", "solve_iterations", 10))
    p.scorr_k = _getf(cp, "Solver", "scorr_k", 0.0)
    p.scorr_n = int(_getf(cp, "Solver", "scorr_n", 4))
    p.scorr_dq = _getf(cp, "Solver", "scorr_dq", 0.1) * p.h
    p.k_stiff = _getf(cp, "Solver", "stiffness_k", 0.95)
    p.v_max = _getf(cp, "Solver", "velocity_max", 100.0)
    p.gravity_axis = _AXES[_gets(cp, "Solver", "gravity_axis", "z").lower()]
    p.vorticity_eps = _getf(cp, "Solver", "vorticity_epsilon", 0.1 * p.h)
    xs = _gets(cp, "Solver", "xsph", "jacobi").lower()
    p.xsph_mode = {"reference": 0, "gauss_seidel": 0, "jacobi": 1, "jacobi_exact": 2}[xs]
    p.enable_tension = 1 if _gets(cp, "Solver", "surface_tension", "on").lower() in ("on", "1", "true") else 0
    p.enable_vorticity = 1 if _gets(cp, "Solver", "vorticity", "on").lower() in ("on", "1", "true") else 0
    # rest state, particles.c:1034-1037, or the lattice poly6 sum
    mode = _gets(cp, "PhysicalParameters", "rest_density", "reference").lower()
    if mode == "lattice":
        p.rest_mass = fluid_volume * 1000.0 / n
        p.rest_density = p.rest_mass * lib.oracle_lattice_poly6_sum(C.byref(p), C.c_double(spacing))
    else:
        p.rest_density = 1000.0
        p.rest_mass = fluid_volume * p.rest_density / n * 0.991
    eps = _getf(cp, "Solver", "lambda_epsilon", 0.01)
    units = _gets(cp, "Solver", "lambda_epsilon_units", "normalized").lower()
    p.lambda_epsilon = eps / (p.rest_density * p.rest_density) if units == "mass_gradient" else eps
    lib.oracle_set_grid(C.byref(p))
    sdf = None
    meta = {"n_requested": n_req, "lattice": nl, "fluid_volume": fluid_volume}
    if cp.has_section("Obstacle") and cp.has_option("Obstacle", "SDF_file_name"):
        fn = _gets(cp, "Obstacle", "SDF_file_name", "")
        if not os.path.isabs(fn):
            fn = os.path.join(os.path.dirname(os.path.abspath(path)), fn)
        dims, origin, dx, vals = read_sdfgen(fn)
        sdf = np.ascontiguousarray(vals, np.float32)
        p.sdim[0], p.sdim[1], p.sdim[2] = dims
        p.sdf_spacing = dx
        p.ob_min[0] = _getf(cp, "Obstacle", "min_x")
        p.ob_max[0] = _getf(cp, "Obstacle", "max_x")
        p.ob_min[1] = _getf(cp, "Obstacle", "min_y")
        p.ob_min[2] = _getf(cp, "Obstacle", "min_z")
        # obstacle.c:73-75
        length = p.ob_max[0] - p.ob_min[0]
        p.ob_max[1] = length * dims[1] / float(np.float32(dims[0]))
        p.ob_max[2] = length * dims[2] / float(np.float32(dims[0]))
        p.sdf = sdf.ctypes.data_as(C.POINTER(C.c_float))
    return Scene(params=p, x0=x, steps=steps, spacing=spacing, sdf=sdf, meta=meta)


# --------------------------------------------------------------------------
# Simulations
# --------------------------------------------------------------------------

class OracleSim:
    """FP64 (or FP32) restatement with arrays in original-index order."""

    def __init__(self, scene: Scene, fp32: bool = False, params: OracleParams | None = None):
        self.lib = oracle_lib(fp32)
        self.scene = scene
        self.p = OracleParams.from_buffer_copy(params if params is not None else scene.params)
        if scene.sdf is not None:
            self.p.sdf = scene.sdf.ctypes.data_as(C.POINTER(C.c_float))
        n = scene.n
        self.n = n
        self.a = {f: np.zeros(n, np.float64) for f in STATE_FIELDS}
        for i, (f, fs) in enumerate((("x", "xs"), ("y", "ys"), ("z", "zs"))):
            self.a[f][:] = scene.x0[i]
            self.a[fs][:] = scene.x0[i]
        self.a["rho"][:] = self.p.rest_density
        self.s = OracleState(n=n, **{f: _ptr(self.a[f]) for f in STATE_FIELDS})
        C_ = self.p.nx * self.p.ny * self.p.nz
        self.nb_arrays = {
            "keys": np.zeros(n, np.uint32), "ids": np.zeros(n, np.uint32),
            "start": np.zeros(C_, np.uint32), "end": np.zeros(C_, np.uint32),
            "nbr": np.zeros(n * MAX_NEIGHBORS, np.uint32), "count": np.zeros(n, np.int32)}
        na = self.nb_arrays
        self.nb = OracleNeighbors(
            keys=_ptr(na["keys"], C.c_uint32), ids=_ptr(na["ids"], C.c_uint32),
            start=_ptr(na["start"], C.c_uint32), end=_ptr(na["end"], C.c_uint32),
            nbr=_ptr(na["nbr"], C.c_uint32), count=_ptr(na["count"], C.c_int32))

    def call(self, name, *args):
        fn = getattr(self.lib, "oracle_" + name)
        if name in ("update_positions",):
            return fn(C.byref(self.s))
        if name in ("apply_gravity", "predict_positions", "update_position_stars",
                    "update_velocities"):
            return fn(C.byref(self.p), C.byref(self.s))
        return fn(C.byref(self.p), C.byref(self.s), C.byref(self.nb), *args)

    def step(self, n=1):
        for _ in range(n):
            self.lib.oracle_step(C.byref(self.p), C.byref(self.s), C.byref(self.nb))

    def diagnostics(self):
        d = OracleDiag()
        self.lib.oracle_diagnostics(C.byref(self.p), C.byref(self.s), C.byref(d))
        return d.as_dict()

    def features(self):
        """Warm-start features [n][16] of the current (predicted) state."""
        f = np.zeros((self.n, 16), np.float64)
        self.lib.oracle_features(C.byref(self.p), C.byref(self.s), C.byref(self.nb), _ptr(f))
        return f

    def lambda_target(self, iterations):
        """Plain solve of `iterations` substeps; returns sum_k s_k lambda_k."""
        t = np.zeros(self.n, np.float64)
        self.lib.oracle_lambda_target(C.byref(self.p), C.byref(self.s), C.byref(self.nb),
                                      iterations, _ptr(t))
        return t

    def neighbor_lists(self):
        cnt = self.nb_arrays["count"]
        nbr = self.nb_arrays["nbr"].reshape(-1, MAX_NEIGHBORS)
        return cnt, nbr


class RefSim:
    """The reference's own particles.c / neighbors.c (oracle/_ref)."""

    FIELDS = ["xs", "ys", "zs", "x", "y", "z", "vx", "vy", "vz", "dpx", "dpy", "dpz",
              "wx", "wy", "wz", "cx", "cy", "cz", "rho", "lam"]

    def __init__(self, scene: Scene, fast: bool = False, params: OracleParams | None = None):
        self.lib = ref_lib(fast)
        self.scene = scene
        self.p = OracleParams.from_buffer_copy(params if params is not None else scene.params)
        if scene.sdf is not None:
            self.p.sdf = scene.sdf.ctypes.data_as(C.POINTER(C.c_float))
        self.n = scene.n
        self.h = self.lib.ref_create(C.byref(self.p), self.n)
        for i, (f, fs) in enumerate((("x", "xs"), ("y", "ys"), ("z", "zs"))):
            v = np.ascontiguousarray(scene.x0[i])
            self.set(f, v)
            self.set(fs, v)
        self.set("rho", np.full(self.n, self.p.rest_density))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_destroy(self.h)
            self.h = None

    def set(self, f, v):
        v = np.ascontiguousarray(v, np.float64)
        self.lib.ref_set_field(self.h, self.FIELDS.index(f), _ptr(v))

    def get(self, f):
        out = np.empty(self.n, np.float64)
        self.lib.ref_get_field(self.h, self.FIELDS.index(f), _ptr(out))
        return out

    def call(self, name, *args):
        return getattr(self.lib, "ref_" + name)(self.h, *args)

    def step(self, n=1, iterations=10):
        self.lib.ref_step(self.h, n, iterations)

    def neighbors(self):
        p = self.p
        C_ = p.nx * p.ny * p.nz
        keys = np.empty(self.n, np.uint32)
        ids = np.empty(self.n, np.uint32)
        start = np.empty(C_, np.uint32)
        end = np.empty(C_, np.uint32)
        nbr = np.empty(self.n * MAX_NEIGHBORS, np.uint32)
        cnt = np.empty(self.n, np.int32)
        U = C.c_uint32
        self.lib.ref_get_neighbors(self.h, _ptr(keys, U), _ptr(ids, U), _ptr(start, U),
                                   _ptr(end, U), _ptr(nbr, U), _ptr(cnt, C.c_int32))
        return {"keys": keys, "ids": ids, "start": start, "end": end,
                "nbr": nbr.reshape(-1, MAX_NEIGHBORS), "count": cnt}
