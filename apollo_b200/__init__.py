"""apollo_b200: B200-native nodal-DG right-hand side and SSP Runge-Kutta stepper.

The compute path is libapollo_dg.so (hand-written sm_100a CUDA behind the C ABI
in include/apollo_dg.h); this package holds its Python binding (``dg``), mesh
generation (``mesh``) and the benchmark problems (``problems``).
"""
from .mesh import Mesh, jittered_square, grid_for_elements
from .dg import NodalDG2d, NodalDG2dBatch, ApolloError, load_library, LIB_PATH, FIELDS
from .gmsh import read_gmsh, write_gmsh
from .vtk import read_vtu, write_frame, write_vtu

__all__ = ["Mesh", "jittered_square", "grid_for_elements", "NodalDG2d", "NodalDG2dBatch", "read_gmsh", "write_gmsh", "write_vtu", "write_frame", "read_vtu", "ApolloError", "load_library",
           "LIB_PATH", "FIELDS"]
