"""B200-native UFEM Navier-Stokes hot path (COOLFluiD 3 UFEM drop-in).

The product is the native library ``libufem_b200.so`` (C ABI in
``include/ufem_b200.h``); this package loads it and mirrors the reference's
NavierStokes solver-action interface for Python callers and tests.
"""
from ._native import UfemError, lib  # noqa: F401
from .problems import Problem, config, cube_tets, lid_driven_bcs, make_problem, rectangle_tris  # noqa: F401
from .ufem import Batch, NavierStokes, NavierStokesSemiImplicit, krylov_options  # noqa: F401

__all__ = ["NavierStokes", "NavierStokesSemiImplicit", "Batch", "UfemError", "Problem", "config", "make_problem", "rectangle_tris", "cube_tets",
           "lid_driven_bcs", "krylov_options", "lib"]
