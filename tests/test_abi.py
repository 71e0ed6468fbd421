"""The C ABI without a GPU: the library loads, exports every function that
include/*.h declares, its host-side logic (configuration, scene set-up, SDF
file input, error codes) matches the oracle's restatement of the
reference's set-up, and device calls fail loudly instead of falling back to
the CPU."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from oracle.pyoracle import read_sdfgen, scene_from_ini
from sphpc_b200 import _lib
from sphpc_b200._lib import AABB, Obstacle, Params, Particles, Solver
from sphpc_b200.scenes import CONFIGS, config_path, torus_sphere_sdf, write_sdfgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        src = re.sub(r"#[^\n]*", "", src)
        for m in re.finditer(r"\b([A-Za-z_]\w*)\s*\(([^;{}]*)\)\s*;", src):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_function():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) > 50
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding declares a signature for each of them
    assert names <= set(_lib.SIGNATURES), sorted(names - set(_lib.SIGNATURES))


def test_struct_layouts_match_header_sizes():
    # field-for-field mirrors of the reference's structs (x86-64 sizes)
    assert C.sizeof(Params) == 12 * 8 + 3 * 4 + 4
    assert C.sizeof(AABB) == 48
    assert C.sizeof(Particles) == 21 * 8 + 3 * 8 + 5 * 4 + 4
    assert C.sizeof(Obstacle) == 128 + 6 * 8 + 48 + 8 + 3 * 4 + 4 + 8 + 8


def _load(name):
    p, pa, b, f, ob, s = Params(), Particles(), AABB(), AABB(), Obstacle(), Solver()
    _lib.call("sphpc_load_config", config_path(name).encode(), C.byref(p), C.byref(pa),
              C.byref(b), C.byref(f), C.byref(ob), C.byref(s))
    return p, pa, b, f, ob, s


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_config_matches_oracle_setup(name):
    """SetParameters (simulation.c:130-178) in the library vs the oracle's
    independent restatement."""
    p, pa, b, f, ob, s = _load(name)
    sc = scene_from_ini(config_path(name))
    op = sc.params
    assert p.smoothing_radius == op.h
    assert p.W_norm == op.W_norm and p.DelW_norm == op.DelW_norm
    assert p.DelW_poly_norm == op.DelW_poly_norm
    assert (p.g, p.time_step, p.k, p.c) == (op.g, op.dt, op.gamma, op.c)
    assert s.solve_iterations == op.solve_iterations
    assert s.gravity_axis == op.gravity_axis
    assert abs(s.scorr_dq * p.smoothing_radius - op.scorr_dq) < 1e-12
    assert s.scorr_k == op.scorr_k and s.scorr_n == op.scorr_n
    assert s.xsph_exact == (1 if op.xsph_mode == 2 else 0)
    assert s.surface_tension == op.enable_tension and s.vorticity == op.enable_vorticity


def test_lattice_matches_oracle_bit_for_bit():
    """ConstructFluidVolume with seeded jitter (host side of the library)
    equals the oracle's lattice generator."""
    p, pa, b, f, ob, s = _load("small_dam")
    _lib.load().sphpc_set_default_solver(C.byref(s))
    _lib.call("SetParticleNumbers", C.byref(f), C.byref(pa), C.byref(p), None)
    n = pa.max_local
    arrs = {k: np.zeros(n) for k in ("x", "y", "z")}
    ids = np.zeros(n, np.int32)
    for k, v in arrs.items():
        setattr(pa, k, v.ctypes.data_as(C.POINTER(C.c_double)))
    pa.id = ids.ctypes.data_as(C.POINTER(C.c_int))
    _lib.call("ConstructFluidVolume", C.byref(pa), C.byref(p), C.byref(f))
    sc = scene_from_ini(config_path("small_dam"), fp32_positions=False)
    m = pa.local_count
    assert m == sc.n == 4096
    for i, k in enumerate("xyz"):
        np.testing.assert_array_equal(arrs[k][:m], sc.x0[i])
    np.testing.assert_array_equal(ids[:m], np.arange(m))


def test_sdf_reader_and_aspect_fix(tmp_path):
    dims, wmin, sp = (8, 4, 6), (0.0, 0.0, 0.0), 2.0
    vals = torus_sphere_sdf(dims, wmin, sp, ((8.0, 4.0, 6.0), 3.0), ((8.0, 2.0, 6.0), 4.0, 1.0))
    path = str(tmp_path / "t.sdf")
    write_sdfgen(path, dims, (1.0, 1.0, 1.0), sp, vals)
    ob = Obstacle()
    ob.SDF_file_name = path.encode()
    ob.world_bounds.min_x, ob.world_bounds.max_x = 0.0, 16.0
    _lib.call("sphpc_read_sdf", C.byref(ob))
    assert (ob.SDF_dim_x, ob.SDF_dim_y, ob.SDF_dim_z) == dims
    assert ob.SDF_spacing == sp
    got = np.ctypeslib.as_array(ob.SDF_buffer, shape=(8 * 4 * 6,))
    np.testing.assert_array_equal(got, vals)
    # obstacle.c:73-75
    assert ob.world_bounds.max_y == 16.0 * 4 / 8.0
    assert ob.world_bounds.max_z == 16.0 * 6 / 8.0
    d, o, dx, v = read_sdfgen(path)
    np.testing.assert_array_equal(v, vals)


@pytest.mark.parametrize("content,code", [
    ("3 3\n", -2), ("2 2 2\n0 0 0\n1\n0.5\n0.5\n", -2), ("0 2 2\n0 0 0\n1\n", -2),
    ("2 1 1\n0 0 0\nx\n1\n2\n", -2)])
def test_sdf_reader_errors(tmp_path, content, code):
    path = tmp_path / "bad.sdf"
    path.write_text(content)
    ob = Obstacle()
    ob.SDF_file_name = str(path).encode()
    rc = _lib.load().sphpc_read_sdf(C.byref(ob))
    assert rc == code
    assert _lib.load().sphpc_last_error()


def test_missing_sdf_file():
    ob = Obstacle()
    ob.SDF_file_name = b"/nonexistent/none.sdf"
    assert _lib.load().sphpc_read_sdf(C.byref(ob)) == -2
    assert b"Can't open" in _lib.load().sphpc_last_error()


@pytest.mark.parametrize("mutate,needle", [
    (lambda t: t.replace("time_step = 0.008", ""), b"missing key SimParameters.time_step"),
    (lambda t: t.replace("g = 9.8", "g = nine"), b"not a number"),
    (lambda t: t.replace("gravity_axis = y", "gravity_axis = w"), b"gravity_axis"),
    (lambda t: t.replace("xsph = jacobi", "xsph = reference"), b"data race"),
    (lambda t: t.replace("[Solver]", "[Solver"), b"unterminated"),
    (lambda t: t.replace("min_x = 0.0\nmax_x = 48.0", "min_x = -1.0\nmax_x = 48.0"),
     b"BoundaryVolume minimum"),
])
def test_malformed_config_is_an_error(tmp_path, mutate, needle):
    text = open(config_path("small_dam")).read()
    path = tmp_path / "bad.ini"
    path.write_text(mutate(text))
    p, pa, b, f, ob, s = Params(), Particles(), AABB(), AABB(), Obstacle(), Solver()
    rc = _lib.load().sphpc_load_config(str(path).encode(), C.byref(p), C.byref(pa), C.byref(b),
                                       C.byref(f), C.byref(ob), C.byref(s))
    assert rc in (-1, -2)
    assert needle in _lib.load().sphpc_last_error()


def test_reference_constants_are_the_defaults():
    s = Solver()
    _lib.load().sphpc_default_solver(C.byref(s))
    assert s.solve_iterations == 10 and s.lambda_epsilon == 0.01 and s.scorr_k == 0.0
    assert s.stiffness_k == 0.95 and s.gravity_axis == 2 and s.velocity_max == 100.0
    assert s.surface_tension == 1 and s.vorticity == 1 and s.xsph_exact == 0


def test_device_calls_fail_loudly_without_a_device():
    """No CPU fallback: without a CUDA device the particle set cannot be
    created and the seam returns an error."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    p, pa, b, f, ob, s = _load("small_dam")
    _lib.call("SetParticleNumbers", C.byref(f), C.byref(pa), C.byref(p), None)
    rc = _lib.load().AllocInitParticles(C.byref(pa), C.byref(p), C.byref(f))
    assert rc == -3
    assert b"no CUDA device" in _lib.load().sphpc_last_error()
    _lib.load().FinalizeParticles(C.byref(pa))
    assert _lib.load().ComputeDensities(C.byref(pa), C.byref(p), None) == -5
