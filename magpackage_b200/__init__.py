"""magpackage_b200: B200-native (sm_100a) Nedelec element assembly for MagPackage.

The hot path -- curl-curl stiffness K(nu), sigma-mass M, Newton Jacobian and
residual scattered into a global CSR -- runs in hand-written CUDA kernels in
``libmagasm.so`` behind the C ABI of ``include/magasm.h``. This package holds
the host-side mirror of the reference's ``Mesh``/``DofHandler``/``Assembler``
interface, the synthetic workloads, and the learned reluctivity warm start.
"""
from .material import (NU0, MU0, Material, PackedMaterials, create_linear, create_linear_nu,
                       create_nonlinear, froehlich_bh, pack_material_data)
from .quadrature import get_quadrature_data, nedelec_tet_p1, reference_data

__all__ = [
    "NU0", "MU0", "Material", "PackedMaterials", "create_linear", "create_linear_nu",
    "create_nonlinear", "froehlich_bh", "pack_material_data", "get_quadrature_data",
    "nedelec_tet_p1", "reference_data",
]
