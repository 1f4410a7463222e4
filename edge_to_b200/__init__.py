"""B200-native SIMP minimum-compliance / GMG-PCG path with the call surface of ahnobari/EDGE-TO.

Drop-in names (EDGETO/__init__.py, TopOpt/__init__.py, solvers/__init__.py,
kernels/__init__.py, geom/__init__.py): CuStructuredMesh2D/3D, CuStructuredStiffnessKernel,
CuStructuredFilter2D/3D, CuMultiGrid, MultiGrid (the CPU solver's smoother-weight semantics),
CuCG, CuTopOpt, SingleMaterial, PenalizedMultiMaterial,
auto_stiffness, and for unstructured meshes CuGeneralMesh, CuUniformStiffnessKernel,
CuGeneralStiffnessKernel, CuGeneralFilter (with CuCG); beyond the
reference, SIMPObjective (differentiable compliance / mechanism objectives, autograd.py).
Arrays are torch CUDA tensors; the compute runs in libedge_b200.so (sm_100a).
"""
from . import autograd
from .autograd import SIMPObjective
from .filters import CuGeneralFilter, CuStructuredFilter2D, CuStructuredFilter3D, FilterKernel
from .kernels import (CuGeneralStiffnessKernel, CuStructuredStiffnessKernel, CuUniformStiffnessKernel,
                      StiffnessKernel)
from .material import MaterialModel, PenalizedMultiMaterial, SingleMaterial
from .mesh import CuGeneralMesh, CuStructuredMesh2D, CuStructuredMesh3D, GeneralMesh, StructuredMesh
from .physics import auto_stiffness, hexahedron_element_stiffness, quadrilateral_element_stiffness
from .solvers import CuCG, CuMultiGrid, MultiGrid
from .topopt import CuTopOpt

__all__ = [
    "CuStructuredMesh2D", "CuStructuredMesh3D", "StructuredMesh", "CuGeneralMesh", "GeneralMesh", "CuStructuredStiffnessKernel", "StiffnessKernel",
    "CuStructuredFilter2D", "CuStructuredFilter3D", "FilterKernel", "CuMultiGrid", "MultiGrid", "CuCG", "CuTopOpt", "SingleMaterial",
    "PenalizedMultiMaterial", "MaterialModel", "auto_stiffness", "hexahedron_element_stiffness", "quadrilateral_element_stiffness",
    "SIMPObjective", "CuUniformStiffnessKernel", "CuGeneralStiffnessKernel", "CuGeneralFilter",
]
