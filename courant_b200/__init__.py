"""courant_b200: B200 FDTD time-stepping engine behind the courant.h C ABI.

The product is the shared library courant_b200/lib/libcourant_b200.so (C ABI
declared in include/courant.h). This package adds the build recipe
(courant_b200.build), a Python host mirror of the reference wrapper
(courant_b200.api) and scenario builders (courant_b200.scenes).
"""
from .api import (Axis, Boundary, C0, EPS0, MU0, Courant, CourantError, DebyeModel, Face, Sim,  # noqa: F401
                  default_library, s_params)

__all__ = ["Axis", "Boundary", "C0", "EPS0", "MU0", "Courant", "CourantError", "DebyeModel", "Face", "Sim",
           "default_library", "s_params"]
