"""sphpc_b200 -- B200 (sm_100a) implementation of SPHPC's per-step
Position-Based-Fluids particle pipeline behind the reference's C host API.

The product is the C-ABI library libsphpc_cuda.so (include/*.h); this package
holds its sources (csrc/), scene configurations (configs/) and a thin Python
host driver (Simulation) used by the tests and the benchmark.
"""
from ._lib import SphpcError, load  # noqa: F401
from .simulation import Simulation  # noqa: F401

__all__ = ["Simulation", "SphpcError", "load"]
