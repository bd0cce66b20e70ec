"""B200-native LithoInv hot path: polyhedron gz / TMI forward, analytic vertex
gradient contracted into the objective gradient, DOF scatter/gather and a
host projected L-BFGS driver, behind the C ABI of include/litho_gpu.h."""
from .api import (FIXED, GATHER_CHAIN, GATHER_REFERENCE, GRAVITY, MAGNETIC, PREC_FP64, PREC_MIXED,
                  XY_ANALYTIC, XY_FORWARD_DIFFERENCE, XYZ_FREE, Z_ONLY, Context, LithoError, Model, read_surface,
                  write_tsurf)
from .build import build_library, library_path

__all__ = ["Context", "Model", "LithoError", "build_library", "library_path", "FIXED", "Z_ONLY", "XYZ_FREE",
           "GRAVITY", "MAGNETIC", "PREC_FP64", "PREC_MIXED", "GATHER_REFERENCE", "GATHER_CHAIN", "XY_ANALYTIC",
           "XY_FORWARD_DIFFERENCE", "read_surface", "write_tsurf"]
