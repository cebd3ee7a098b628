"""B200-native DEM-Engine hot path: Python bindings of the C ABI (include/deme_b200.h)."""
from . import _capi as capi  # noqa: F401
from .scene import SceneBuilder, BuiltScene  # noqa: F401
from .solver import Solver, HandleSolver, DemeError, load_product_library, LIB_PATH  # noqa: F401

__all__ = ["SceneBuilder", "BuiltScene", "Solver", "HandleSolver", "DemeError", "load_product_library", "LIB_PATH",
           "capi"]
