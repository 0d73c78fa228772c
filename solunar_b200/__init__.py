"""B200-native particle-fluid step with solunar's FluidWorld API.

`FluidWorld` drives the CUDA library `libsolunar_fluid.so` (built in-tree by
`solunar_b200.build`) through its C ABI, include/solunar_fluid.h.  There is no CPU fallback:
creating a world without the built library, or without a CUDA device, raises.
"""
from .abi import (  # noqa: F401
    Arithmetic,
    FluidReport,
    FluidSettings,
    FluidSolver,
    PhysicsError,
    Positions,
)


def __getattr__(name):
    # the world type loads the CUDA library; import it lazily so that settings and scenes can
    # be used on a machine without a GPU
    if name in ("FluidWorld", "library_path", "load_library"):
        from . import fluid

        return getattr(fluid, name)
    raise AttributeError(name)
