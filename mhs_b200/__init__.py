"""mhs_b200 -- mollified Mindlin half-space triangular-dislocation Green's
function matrices, assembled on NVIDIA B200 (sm_100a) GPUs.

A drop-in for mhs's matrix calls: the same names, arguments, index order and
error behaviour, with the assembly running in hand-written CUDA kernels
(``libmhs_b200.so``, C ABI in ``include/mhs_b200.h``).  There is no CPU path:
without a CUDA device the matrix functions raise.

    import mhs_b200 as mhs
    mat = mhs.Material(mu=30.0, lam=30.0)
    G = mhs.disp_matrix(obs, tris, mat, eps=0.1)     # (n_obs, 3, n_src, 3)

``mhs_b200.fullspace`` is mhs.fullspace.api's single-triangle calls
(displacement, stress, eigenstress, force_displacement, force_stress,
influence) on the device.
"""
from . import chunking, defaults, fullspace, tdcs
from .materials import Material
from .matrices import (
    collocation_points,
    disp_matrix,
    disp_matvec,
    eigenstress_matrix,
    elastic_strain_matrix,
    interaction_matrix,
    interaction_matvec,
    stress_matrix,
    stress_matvec,
    total_stress_matrix,
    traction_matrix,
    traction_matvec,
)
from .shared import SharedNodes, shared_nodes

__all__ = [
    "Material",
    "disp_matrix",
    "stress_matrix",
    "traction_matrix",
    "interaction_matrix",
    "total_stress_matrix",
    "eigenstress_matrix",
    "elastic_strain_matrix",
    "collocation_points",
    "interaction_matvec",
    "disp_matvec",
    "stress_matvec",
    "traction_matvec",
    "shared_nodes",
    "SharedNodes",
    "chunking",
    "defaults",
    "fullspace",
    "tdcs",
]

__version__ = "0.1.0"
