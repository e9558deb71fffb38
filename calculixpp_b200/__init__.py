"""calculixpp_b200 — B200-native element integration and CSR assembly for CalculiX++.

The hot path of the reference's assemble_linear_static / assemble_material_tangent
(per-element Gauss integration of K_e and f_int for C3D8/C3D8R/C3D20/C3D20R/C3D6/C3D15,
the J2 radial return with its consistent tangent, and the scatter into the reduced CSR
system) runs in the CUDA kernels of libcxg.so, reached through its C ABI
(include/cxg.h). This package is the Python side of that boundary.
"""
from . import meshgen
from ._lib import CxgError, load as load_library
from .assembly import (LinearSystem, Material, MaterialPoints, Model, Plan, ThermalPlan, assemble_linear_static,
                       assemble_material_tangent, element_stiffness, element_tangent_force,
                       make_material_points)
from .batch import Batch
from .solve import solve_sparse

__all__ = ["meshgen", "Batch", "ThermalPlan", "CxgError", "load_library", "LinearSystem", "Material", "MaterialPoints", "Model",
           "Plan", "assemble_linear_static", "assemble_material_tangent", "element_stiffness",
           "element_tangent_force", "make_material_points", "solve_sparse"]
