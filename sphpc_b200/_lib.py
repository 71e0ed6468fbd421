"""ctypes binding of libsphpc_cuda.so (the product's C ABI, include/*.h).

The structs below mirror include/sphpc_types.h field for field.  Loading the
library never needs a GPU; calls that touch the device fail with
SPHPC_ECUDA when none is present (there is no CPU fallback).
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsphpc_cuda.so")

SPHPC_OK = 0
ERRORS = {-1: "EINVAL", -2: "EIO", -3: "ECUDA", -4: "ENOMEM", -5: "ENOTREADY",
          -6: "EKERNEL"}
MAX_NEIGHBORS = 60


class Params(C.Structure):
    _fields_ = [("smoothing_radius", C.c_double), ("W_norm", C.c_double),
                ("DelW_norm", C.c_double), ("DelW_poly_norm", C.c_double),
                ("g", C.c_double), ("time_step", C.c_double), ("k", C.c_double),
                ("dq", C.c_double), ("c", C.c_double), ("node_start_x", C.c_double),
                ("node_end_x", C.c_double), ("fluid_volume", C.c_double),
                ("number_steps", C.c_int), ("rank", C.c_int), ("proc_count", C.c_int)]


class AABB(C.Structure):
    _fields_ = [(f, C.c_double) for f in ("min_x", "max_x", "min_y", "max_y", "min_z", "max_z")]


_DP = C.POINTER(C.c_double)
PARTICLE_FIELDS = ["x_star", "y_star", "z_star", "x", "y", "z", "v_x", "v_y", "v_z",
                   "dp_x", "dp_y", "dp_z", "w_x", "w_y", "w_z", "color_x", "color_y",
                   "color_z", "density", "lambda"]


class Particles(C.Structure):
    _fields_ = [(f, _DP) for f in PARTICLE_FIELDS] + [
        ("id", C.POINTER(C.c_int)), ("rest_density", C.c_double), ("rest_mass", C.c_double),
        ("rest_radius", C.c_double), ("global_count", C.c_int), ("local_count", C.c_int),
        ("max_local", C.c_int), ("halo_count_left", C.c_int), ("halo_count_right", C.c_int)]


class NeighborBucket(C.Structure):
    _fields_ = [("neighbor_indices", C.c_uint * MAX_NEIGHBORS), ("count", C.c_int)]


class Neighbors(C.Structure):
    _fields_ = [("start_indices", C.POINTER(C.c_uint)), ("end_indices", C.POINTER(C.c_uint)),
                ("hash_values", C.POINTER(C.c_uint)), ("particle_ids", C.POINTER(C.c_uint)),
                ("hash_size_x", C.c_int), ("hash_size_y", C.c_int), ("hash_size_z", C.c_int),
                ("neighbor_buckets", C.POINTER(NeighborBucket)), ("hash_spacing", C.c_double)]


class Obstacle(C.Structure):
    _fields_ = [("SDF_file_name", C.c_char * 128), ("origin_x", C.c_double),
                ("origin_y", C.c_double), ("origin_z", C.c_double),
                ("model_length", C.c_double), ("model_width", C.c_double),
                ("model_height", C.c_double), ("world_bounds", AABB),
                ("SDF_spacing", C.c_double), ("SDF_dim_x", C.c_int), ("SDF_dim_y", C.c_int),
                ("SDF_dim_z", C.c_int), ("SDF_buffer", C.POINTER(C.c_float)),
                ("obstacle_cuda", C.c_void_p)]


class Solver(C.Structure):
    _fields_ = [("solve_iterations", C.c_int), ("scorr_n", C.c_int),
                ("lambda_epsilon", C.c_double), ("scorr_k", C.c_double),
                ("scorr_dq", C.c_double), ("stiffness_k", C.c_double),
                ("vorticity_epsilon", C.c_double), ("velocity_max", C.c_double),
                ("gravity_axis", C.c_int), ("xsph_exact", C.c_int),
                ("surface_tension", C.c_int), ("vorticity", C.c_int),
                ("jitter", C.c_double), ("seed", C.c_ulonglong),
                ("rest_density_lattice", C.c_int), ("adaptive", C.c_int),
                ("density_tolerance", C.c_double), ("max_iterations", C.c_int),
                ("warm_start", C.c_int), ("lambda_epsilon_mass_units", C.c_int),
                ("warm_start_gate", C.c_int), ("warm_start_source", C.c_int),
                ("warm_start_scale", C.c_double), ("min_progress", C.c_double),
                ("warm_start_min_error", C.c_double)]


class FileIO(C.Structure):
    _fields_ = [("write_buffer", C.POINTER(C.c_double)), ("output_path", C.c_char_p),
                ("file_num", C.c_int)]


class Diag(C.Structure):
    _fields_ = [("max_density_error", C.c_double), ("mean_density_error", C.c_double),
                ("kinetic_energy", C.c_double), ("com", C.c_double * 3),
                ("momentum", C.c_double * 3), ("iterations", C.c_double),
                ("warm_start_used", C.c_double)]

    def as_dict(self):
        return {"max_density_error": self.max_density_error,
                "mean_density_error": self.mean_density_error,
                "kinetic_energy": self.kinetic_energy, "com": list(self.com),
                "momentum": list(self.momentum), "iterations": self.iterations,
                "warm_start_used": self.warm_start_used}


class StepInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int),
                ("warm_start_used", C.c_int), ("warm_start_rejected", C.c_int),
                ("max_density_error", C.c_double), ("mean_density_error", C.c_double),
                ("trace_len", C.c_int), ("pad", C.c_int), ("trace", C.c_double * 16)]


class KernelTime(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_int), ("pad", C.c_int),
                ("total_ms", C.c_double)]


class SphpcError(RuntimeError):
    def __init__(self, fn, code, msg):
        super().__init__(f"{fn} failed ({ERRORS.get(code, code)}): {msg}")
        self.code = code


# Every symbol include/*.h declares, with its argtypes (restype int unless
# noted).  tests/test_abi.py checks the library exports all of them.
P, PP, PA, PN, PO = (C.POINTER(Params), C.POINTER(Particles), C.POINTER(AABB),
                     C.POINTER(Neighbors), C.POINTER(Obstacle))
U = C.POINTER(C.c_uint)
SIGNATURES = {
    "sphpc_last_error": ([], C.c_char_p),
    "sphpc_version": ([], C.c_char_p),
    "sphpc_default_solver": ([C.POINTER(Solver)], None),
    "sphpc_set_default_solver": ([C.POINTER(Solver)], None),
    "ReadParameters": ([P, PP, PA, PA, PO], C.c_int),
    "SetParameters": ([P, PP, PN, PA, PA, PO], C.c_int),
    "sphpc_load_config": ([C.c_char_p, P, PP, PA, PA, PO, C.POINTER(Solver)], C.c_int),
    "SetParticleNumbers": ([PA, PP, P, C.c_void_p], C.c_int),
    "ConstructFluidVolume": ([PP, P, PA], C.c_int),
    "AllocInitParticles": ([PP, P, PA], C.c_int),
    "FinalizeParticles": ([PP], C.c_int),
    "sphpc_enter_data": ([PP, P], C.c_int),
    "sphpc_exit_data": ([PP], C.c_int),
    "sphpc_update_host": ([PP], C.c_int),
    "sphpc_update_device": ([PP], C.c_int),
    "sphpc_update_host_fields": ([PP, C.c_uint], C.c_int),
    "sphpc_update_host_fields_async": ([PP, C.c_uint], C.c_int),
    "sphpc_host_wait": ([PP], C.c_int),
    "sphpc_update_device_fields": ([PP, C.c_uint], C.c_int),
    "sphpc_set_solver": ([PP, C.POINTER(Solver)], C.c_int),
    "sphpc_get_solver": ([PP, C.POINTER(Solver)], C.c_int),
    "sphpc_set_stream": ([PP, C.c_void_p], C.c_int),
    "ApplyGravity": ([PP, P], C.c_int),
    "PredictPositions": ([PP, P, PA], C.c_int),
    "ComputeDensities": ([PP, P, PN], C.c_int),
    "ComputeLambda": ([PP, P, PN], C.c_int),
    "UpdateDPs": ([PP, P, PN, C.c_int], C.c_int),
    "UpdatePositionStars": ([PP, PA, PO, P], C.c_int),
    "UpdateVelocities": ([PP, P], C.c_int),
    "ComputeSurfaceTension": ([PP, P, PN], C.c_int),
    "ApplyViscosity": ([PP, P, PN], C.c_int),
    "ComputeVorticity": ([PP, P, PN], C.c_int),
    "ApplyVorticityConfinement": ([PP, P, PN], C.c_int),
    "UpdatePositions": ([PP], C.c_int),
    "AllocInitNeighbors": ([PN, PP, P, PA], C.c_int),
    "FinalizeNeighbors": ([PN], C.c_int),
    "FindAllNeighbors": ([PP, P, PN], C.c_int),
    "sphpc_get_neighbor_buckets": ([PP, U, C.POINTER(C.c_int)], C.c_int),
    "sphpc_get_cell_data": ([PP, U, U, U], C.c_int),
    "AllocInitObstacle": ([PO], C.c_int),
    "FinalizeObstacle": ([PO], C.c_int),
    "sphpc_read_sdf": ([PO], C.c_int),
    "sphpc_neighbor_pretest_fp32_safe": ([C.c_double, C.c_double], C.c_int),
    "sphpc_step": ([PP, P, PN, PA, PO, C.c_int], C.c_int),
    "AllocInitFileIO": ([C.POINTER(FileIO), PP, P], C.c_int),
    "WriteParticles": ([PP, P, C.POINTER(FileIO)], C.c_int),
    "sphpc_fileio_wait": ([C.POINTER(FileIO)], C.c_int),
    "FinalizeFileIO": ([C.POINTER(FileIO)], C.c_int),
    "sphpc_mlp_collect": ([PP, P, PN, PA, PO, C.c_int], C.c_int),
    "sphpc_mlp_load": ([PP, C.POINTER(C.c_float), C.POINTER(C.c_float)], C.c_int),
    "sphpc_mlp_unload": ([PP], C.c_int),
    "sphpc_mlp_features": ([PP, P, PA, PO, C.POINTER(C.c_float)], C.c_int),
    "sphpc_diagnostics": ([PP, C.POINTER(Diag)], C.c_int),
    "sphpc_device_errors": ([PP, U], C.c_int),
    "sphpc_step_info": ([PP, C.POINTER(StepInfo)], C.c_int),
    "sphpc_profile": ([PP, C.c_int], C.c_int),
    "sphpc_profile_read": ([PP, C.POINTER(KernelTime), C.c_int, C.POINTER(C.c_int)], C.c_int),
    "sphpc_mlp_forward": ([C.c_void_p, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float),
                           C.c_void_p, C.c_void_p], C.c_int),
    "sphpc_mesh_sdf": ([C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_int), C.c_int,
                        C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_double,
                        C.POINTER(C.c_float)], C.c_int),
    "sphpc_particle_surface": ([C.POINTER(C.c_double), C.c_int, C.c_double, C.c_int,
                                C.POINTER(C.c_int), C.POINTER(C.c_double),
                                C.POINTER(C.c_float)], C.c_int),
    "sphpc_mlp_grad": ([C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_void_p],
                       C.c_int),
    "sphpc_fail_device_alloc": ([C.c_int], C.c_int),
    "sphpc_mlp_dataset_reserve": ([C.c_longlong], C.c_int),
    "sphpc_mlp_dataset_size": ([C.POINTER(C.c_longlong)], C.c_int),
    "sphpc_mlp_dataset_clear": ([], C.c_int),
    "sphpc_mlp_dataset_free": ([], C.c_int),
    "sphpc_mlp_dataset_append": ([C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_longlong], C.c_int),
    "sphpc_mlp_dataset_read": ([C.c_longlong, C.c_longlong, C.POINTER(C.c_float), C.POINTER(C.c_float)], C.c_int),
    "sphpc_mlp_dataset_stats": ([C.POINTER(C.c_float)], C.c_int),
    "sphpc_mlp_train": ([C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int, C.c_int,
                         C.c_float, C.c_float, C.c_float, C.c_ulonglong,
                         C.POINTER(C.c_float), C.POINTER(C.c_float)], C.c_int),
    "SortByKey": ([U, U, C.c_int, C.c_void_p], C.c_int),
    "SortByKeyNoAlloc": ([U, U, C.c_int, C.c_void_p], C.c_int),
    "sphpc_check_sort_wait": ([C.c_int, U], C.c_int),
    "sphpc_slab_init": ([PP, C.c_uint, C.c_double, C.c_double, C.c_int, C.c_int], C.c_int),
    "sphpc_slab_halo_width": ([P, C.POINTER(Solver), C.POINTER(C.c_double)], C.c_int),
    "sphpc_slab_pack": ([PP, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_void_p,
                         C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
    "sphpc_slab_unpack": ([PP, C.c_void_p, C.c_int, C.c_void_p, C.c_int], C.c_int),
    "sphpc_slab_owned": ([PP, U, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int,
                          C.POINTER(C.c_int)], C.c_int),
    "sphpc_balance_nodes": ([C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                             C.c_int, P], C.c_int),
    "sphpc_check_mbarrier_wait": ([C.c_int, U], C.c_int),
    "FindLowerBounds": ([U, C.c_int, C.c_int, U, C.c_void_p], C.c_int),
    "FindUpperBounds": ([U, C.c_int, C.c_int, U, C.c_void_p], C.c_int),
    "CalculateParticleCollisions": ([_DP, _DP, _DP, C.c_int, Obstacle], C.c_int),
    "AllocInitObstacle_CUDA": ([PO], C.c_int),
    "FinalizeObstacle_CUDA": ([C.c_void_p], C.c_int),
}

_LIB = None


def load(path: str = LIB_PATH):
    """Loads the CUDA library (raises if it was not built: no fallback)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `make -C sphpc_b200/csrc` "
            "(the pipeline has no CPU fallback)")
    lib = C.CDLL(path)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _LIB = lib
    return lib


def check(fn_name: str, rc: int):
    if rc != SPHPC_OK:
        msg = load().sphpc_last_error().decode(errors="replace")
        raise SphpcError(fn_name, rc, msg)
    return rc


def call(name: str, *args):
    return check(name, getattr(load(), name)(*args))
