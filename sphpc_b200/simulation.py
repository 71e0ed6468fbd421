"""Python host driver over the C ABI, mirroring the reference's main()
(Simulation/src/simulation.c:19-128): load the configuration, allocate and
initialise particles, neighbours and obstacle, then step.

Every call goes through libsphpc_cuda.so; host arrays are the reference's
FP64 SoA in original particle order (numpy views of the C arrays).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import (AABB, Diag, FileIO, KernelTime, Neighbors, Obstacle, Params, Particles,
                   Solver, StepInfo, PARTICLE_FIELDS, call, load)
from .scenes import config_path


class Simulation:
    """One particle set on the device.

    ``solver_overrides`` replaces fields of the configuration's solver
    settings (struct SphpcSolver) before the particles are created.
    """

    def __init__(self, config: str, solver_overrides: dict | None = None,
                 obstacle: bool = True):
        self.lib = load()
        self.path = config_path(config)
        self.params = Params()
        self.particles = Particles()
        self.boundary = AABB()
        self.fluid = AABB()
        self.obstacle = Obstacle()
        self.neighbors = Neighbors()
        self.solver = Solver()
        call("sphpc_load_config", self.path.encode(), C.byref(self.params),
             C.byref(self.particles), C.byref(self.boundary), C.byref(self.fluid),
             C.byref(self.obstacle), C.byref(self.solver))
        for k, v in (solver_overrides or {}).items():
            setattr(self.solver, k, v)
        self.lib.sphpc_set_default_solver(C.byref(self.solver))
        call("SetParticleNumbers", C.byref(self.fluid), C.byref(self.particles),
             C.byref(self.params), None)
        call("AllocInitParticles", C.byref(self.particles), C.byref(self.params),
             C.byref(self.fluid))
        self._alive = True
        call("sphpc_set_solver", C.byref(self.particles), C.byref(self.solver))
        call("AllocInitNeighbors", C.byref(self.neighbors), C.byref(self.particles),
             C.byref(self.params), C.byref(self.boundary))
        self.has_obstacle = bool(obstacle and self.obstacle.SDF_file_name)
        if self.has_obstacle:
            call("AllocInitObstacle", C.byref(self.obstacle))
        self.n = self.particles.local_count

    # ---------------- lifetime ----------------
    def close(self):
        if getattr(self, "_alive", False):
            if self.has_obstacle:
                self.lib.FinalizeObstacle(C.byref(self.obstacle))
            self.lib.FinalizeNeighbors(C.byref(self.neighbors))
            self.lib.FinalizeParticles(C.byref(self.particles))
            self._alive = False

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---------------- host arrays ----------------
    def host(self, field: str) -> np.ndarray:
        """numpy view of a host array of struct Particles (FP64, original order)."""
        ptr = getattr(self.particles, field)
        return np.ctypeslib.as_array(ptr, shape=(self.particles.max_local,))[: self.n]

    def fetch(self, fields=None) -> dict:
        """Device -> host (sphpc_update_host), returns copies of the fields."""
        call("sphpc_update_host", C.byref(self.particles))
        fields = fields or PARTICLE_FIELDS
        return {f: self.host(f).copy() for f in fields}

    def fetch_fields(self, fields):
        """Device -> host of the named fields only (no copies returned)."""
        mask = 0
        for f in fields:
            mask |= 1 << PARTICLE_FIELDS.index(f)
        call("sphpc_update_host_fields", C.byref(self.particles), mask)

    def fetch_fields_async(self, fields):
        """Device -> host of the named fields, returning once enqueued: the
        copy overlaps the steps that follow; the host arrays hold the fields
        after host_wait() (every other transfer waits for it first)."""
        mask = 0
        for f in fields:
            mask |= 1 << PARTICLE_FIELDS.index(f)
        call("sphpc_update_host_fields_async", C.byref(self.particles), mask)

    def host_wait(self):
        call("sphpc_host_wait", C.byref(self.particles))

    def push_fields(self, fields):
        """Host -> device of the named fields (groups must be complete)."""
        mask = 0
        for f in fields:
            mask |= 1 << PARTICLE_FIELDS.index(f)
        call("sphpc_update_device_fields", C.byref(self.particles), mask)

    def launches(self) -> int:
        return self.profile_read().get("kernel_launches", (0, 0.0))[0]

    def push(self, arrays: dict | None = None):
        """Writes `arrays` into the host arrays, then host -> device."""
        for f, v in (arrays or {}).items():
            self.host(f)[:] = v
        call("sphpc_update_device", C.byref(self.particles))

    def save_state(self, path: str):
        """Checkpoint: the particle arrays of struct Particles (the reference's
        own state, original order, FP64 copies of the device's values) and the
        solver settings, to an .npz file."""
        arrays = self.fetch()
        solver = {f: getattr(self.solver, f) for f, _ in self.solver._fields_}
        np.savez(path, n=self.n, solver=np.array([solver], dtype=object), **arrays)

    def load_state(self, path: str):
        """Resume from save_state() into a set of the same configuration: the
        arrays go to the device and the solver settings are restored, so the
        steps that follow are those the saved run would have taken (the
        warm-start's skip rule also reads the previous step's first residual,
        which is not part of the checkpoint)."""
        with np.load(path, allow_pickle=True) as z:
            if int(z["n"]) != self.n:
                raise ValueError(f"checkpoint of {int(z['n'])} particles, set of {self.n}")
            self.push({f: z[f] for f in z.files if f not in ("n", "solver")})
            self.set_solver(**z["solver"][0])

    def set_solver(self, **kw):
        for k, v in kw.items():
            setattr(self.solver, k, v)
        call("sphpc_set_solver", C.byref(self.particles), C.byref(self.solver))

    def set_stream(self, stream_ptr: int):
        call("sphpc_set_stream", C.byref(self.particles), C.c_void_p(stream_ptr))

    # ---------------- stepping ----------------
    def _ob(self):
        return C.byref(self.obstacle) if self.has_obstacle else None

    def step(self, steps: int = 1):
        call("sphpc_step", C.byref(self.particles), C.byref(self.params),
             C.byref(self.neighbors), C.byref(self.boundary), self._ob(), steps)

    def diagnostics(self) -> dict:
        d = Diag()
        call("sphpc_diagnostics", C.byref(self.particles), C.byref(d))
        return d.as_dict()

    def last_step_info(self) -> dict:
        i = StepInfo()
        call("sphpc_step_info", C.byref(self.particles), C.byref(i))
        return {"iterations": i.iterations, "converged": i.converged,
                "warm_start_used": i.warm_start_used,
                "warm_start_rejected": i.warm_start_rejected,
                "max_density_error": i.max_density_error,
                "mean_density_error": i.mean_density_error,
                "trace": list(i.trace[:i.trace_len])}

    def device_errors(self) -> int:
        bits = C.c_uint(0)
        call("sphpc_device_errors", C.byref(self.particles), C.byref(bits))
        return bits.value

    def profile(self, enable: bool = True):
        call("sphpc_profile", C.byref(self.particles), 1 if enable else 0)

    def profile_read(self) -> dict:
        buf = (KernelTime * 64)()
        n = C.c_int(0)
        call("sphpc_profile_read", C.byref(self.particles), buf, 64, C.byref(n))
        return {buf[i].name.decode(): (buf[i].launches, buf[i].total_ms)
                for i in range(min(n.value, 64))}

    # reference-named stages (particles.h / neighbors.h), one device stage each
    def apply_gravity(self):
        call("ApplyGravity", C.byref(self.particles), C.byref(self.params))

    def predict_positions(self):
        call("PredictPositions", C.byref(self.particles), C.byref(self.params),
             C.byref(self.boundary))

    def find_all_neighbors(self):
        call("FindAllNeighbors", C.byref(self.particles), C.byref(self.params),
             C.byref(self.neighbors))

    def compute_densities(self):
        call("ComputeDensities", C.byref(self.particles), C.byref(self.params),
             C.byref(self.neighbors))

    def compute_lambda(self):
        call("ComputeLambda", C.byref(self.particles), C.byref(self.params),
             C.byref(self.neighbors))

    def update_dps(self, substep: int):
        call("UpdateDPs", C.byref(self.particles), C.byref(self.params),
             C.byref(self.neighbors), substep)

    def update_position_stars(self):
        call("UpdatePositionStars", C.byref(self.particles), C.byref(self.boundary),
             self._ob(), C.byref(self.params))

    def update_velocities(self):
        call("UpdateVelocities", C.byref(self.particles), C.byref(self.params))

    def surface_tension(self):
        call("ComputeSurfaceTension", C.byref(self.particles), C.byref(self.params),
             C.byref(self.neighbors))

    def apply_viscosity(self):
        call("ApplyViscosity", C.byref(self.particles), C.byref(self.params),
             C.byref(self.neighbors))

    def compute_vorticity(self):
        call("ComputeVorticity", C.byref(self.particles), C.byref(self.params),
             C.byref(self.neighbors))

    def vorticity_confinement(self):
        call("ApplyVorticityConfinement", C.byref(self.particles), C.byref(self.params),
             C.byref(self.neighbors))

    def update_positions(self):
        call("UpdatePositions", C.byref(self.particles))

    # ---------------- snapshot output (fileio_MPI_IO.c) ----------------
    def fileio_open(self) -> FileIO:
        """AllocInitFileIO: snapshots go to ./output/sim-N.bin."""
        f = FileIO()
        call("AllocInitFileIO", C.byref(f), C.byref(self.particles), C.byref(self.params))
        return f

    def write_particles(self, f: FileIO):
        call("WriteParticles", C.byref(self.particles), C.byref(self.params), C.byref(f))

    def fileio_wait(self, f: FileIO):
        call("sphpc_fileio_wait", C.byref(f))

    def fileio_close(self, f: FileIO):
        call("FinalizeFileIO", C.byref(f))

    # ---------------- learned warm start ----------------
    def mlp_load(self, params, norm):
        """Installs the warm-start network (params[9473], norm[33])."""
        p = np.ascontiguousarray(params, np.float32)
        q = np.ascontiguousarray(norm, np.float32)
        F = C.POINTER(C.c_float)
        call("sphpc_mlp_load", C.byref(self.particles), p.ctypes.data_as(F), q.ctypes.data_as(F))

    def mlp_unload(self):
        call("sphpc_mlp_unload", C.byref(self.particles))

    def mlp_features(self) -> np.ndarray:
        """Warm-start features [N][16] by particle id (after find_all_neighbors)."""
        f = np.zeros((self.n, 16), np.float32)
        call("sphpc_mlp_features", C.byref(self.particles), C.byref(self.params),
             C.byref(self.boundary), self._ob(), f.ctypes.data_as(C.POINTER(C.c_float)))
        return f

    def neighbor_buckets(self):
        idx = np.zeros(self.n * _lib.MAX_NEIGHBORS, np.uint32)
        cnt = np.zeros(self.n, np.int32)
        call("sphpc_get_neighbor_buckets", C.byref(self.particles),
             idx.ctypes.data_as(C.POINTER(C.c_uint)), cnt.ctypes.data_as(C.POINTER(C.c_int)))
        return cnt, idx.reshape(self.n, _lib.MAX_NEIGHBORS)

    def cell_data(self):
        nx, ny, nz = (self.neighbors.hash_size_x, self.neighbors.hash_size_y,
                      self.neighbors.hash_size_z)
        keys = np.zeros(self.n, np.uint32)
        ids = np.zeros(self.n, np.uint32)
        start = np.zeros(nx * ny * nz + 1, np.uint32)
        P = C.POINTER(C.c_uint)
        call("sphpc_get_cell_data", C.byref(self.particles), keys.ctypes.data_as(P),
             ids.ctypes.data_as(P), start.ctypes.data_as(P))
        return keys, ids, start
