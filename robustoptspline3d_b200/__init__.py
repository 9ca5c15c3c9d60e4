"""B200-native voxel-FEM worst-case topology optimisation (capabilities of
NanXYZH/RobustOptSpline3D): matrix-free SIMP operator, multigrid V-cycle,
worst-case load, adjoint sensitivities, B-spline density map with the
self-support constraint, and MMA.

The compute lives in ``librso.so`` (hand-written CUDA for sm_100a behind the
C ABI of ``include/rso.h``).  This package is the host-side mirror of the
reference's Grid/optimization interface over that C ABI.  Importing it
without the compiled library raises immediately: there is no CPU fallback.

Submodules beside the solver: ``voxelize`` (OBJ reading, solid
voxelisation), ``boundary`` (regions, load fields, shell elements, normals,
``mesh_problem``), ``records`` (run records in the reference's raw layout)
and ``autograd`` (a torch.autograd.Function over the design gradient).
"""
from .rso import (  # noqa: F401
    Config,
    HierarchyGrid,
    MMA,
    IterParams,
    RSOError,
    element_matrix,
    library_path,
    load_library,
)
