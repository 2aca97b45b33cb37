"""caustic_b200 -- B200-native semi-discrete optimal-transport solver.

The first stage of the rmk523/caustic freeform-lens pipeline (the
``caustic_GPU`` executable of Optimal_Transport_rl/), rebuilt as sm_100a CUDA
behind a C ABI (include/causticot.h, libcausticot.so).

* ``capi.Solver``      -- the C ABI from Python (numpy or torch CUDA tensors)
* ``problems``         -- seeded synthetic problems of the benchmark shapes
"""
from . import capi, problems  # noqa: F401

__all__ = ["problems", "capi"]
