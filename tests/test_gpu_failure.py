"""Failure detection of the library's bounded device waits, without a GPU
fault: each check makes one wait run out on a flag that nothing sets (a
radix-sort look-back flag of an earlier tile; a tensor-core completion
mbarrier nothing arrives on), with a short poll limit.  The kernel must give
up, record its error bit and return; the call must report SPHPC_EKERNEL; and
the device must stay usable (a sort run right after is exact)."""
import ctypes as C

import numpy as np
import pytest

from sphpc_b200 import _lib

EKERNEL = -6
EINVAL = -1


def _sort_still_exact():
    import torch
    rng = np.random.default_rng(5)
    n = 100_000
    keys = rng.integers(0, 1 << 20, size=n, dtype=np.int64).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    dk = torch.from_numpy(keys.view(np.int32)).cuda()
    dv = torch.from_numpy(vals.view(np.int32)).cuda()
    u32 = lambda t: C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_uint))  # noqa: E731
    _lib.call("SortByKey", u32(dk), u32(dv), n,
              C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    order = np.argsort(keys, kind="stable")
    np.testing.assert_array_equal(dv.cpu().numpy().view(np.uint32), vals[order])


@pytest.mark.gpu
def test_sort_lookback_wait_gives_up_and_device_stays_usable():
    lib = _lib.load()
    bits = C.c_uint(0)
    rc = lib.sphpc_check_sort_wait(4096, C.byref(bits))
    assert rc == EKERNEL, (rc, lib.sphpc_last_error())
    assert bits.value & 2, bits.value
    assert b"gave up" in lib.sphpc_last_error()
    _sort_still_exact()


@pytest.mark.gpu
def test_mbarrier_wait_gives_up_and_device_stays_usable():
    lib = _lib.load()
    bits = C.c_uint(0)
    rc = lib.sphpc_check_mbarrier_wait(4096, C.byref(bits))
    assert rc == EKERNEL, (rc, lib.sphpc_last_error())
    assert bits.value & 16, bits.value
    _sort_still_exact()


def test_wait_checks_reject_limits_outside_their_range():
    # checked on the host before any device work (no GPU needed)
    lib = _lib.load()
    bits = C.c_uint(7)
    assert lib.sphpc_check_sort_wait(0, C.byref(bits)) == EINVAL
    assert lib.sphpc_check_sort_wait((1 << 22) + 1, C.byref(bits)) == EINVAL
    assert lib.sphpc_check_mbarrier_wait(0, C.byref(bits)) == EINVAL
    assert lib.sphpc_check_mbarrier_wait((1 << 20) + 1, C.byref(bits)) == EINVAL


ENOMEM = -4


def _first_error(config, steps):
    """Creates a particle set and steps it; the code of the first error, or 0."""
    from sphpc_b200 import Simulation
    from sphpc_b200._lib import SphpcError
    try:
        with Simulation(config) as sim:
            sim.step(steps)
            assert sim.device_errors() == 0
    except SphpcError as e:
        return e.code
    return 0


@pytest.mark.gpu
@pytest.mark.parametrize("after", [0, 1, 4, 12])
def test_device_allocation_failure_is_an_error_and_the_next_set_works(after):
    """An allocation of the particle set's device copy that fails (injected
    on the host: the allocation returns the error cudaMalloc would) is
    reported as SPHPC_ENOMEM by the call that needed it; the partly built set
    is released, and a set made afterwards steps normally."""
    lib = _lib.load()
    try:
        assert lib.sphpc_fail_device_alloc(after) == 0
        assert _first_error("small_dam", 1) == ENOMEM
    finally:
        lib.sphpc_fail_device_alloc(-1)
    assert _first_error("small_dam", 2) == 0
    _sort_still_exact()


def test_allocation_injection_rejects_bad_arguments():
    lib = _lib.load()
    assert lib.sphpc_fail_device_alloc(-2) == EINVAL
    assert lib.sphpc_fail_device_alloc(-1) == 0
