"""B200-native (sm_100a) implementation of the OversetDevFort per-timestep hot
path: VMS Navier-Stokes / VOF / temperature element assembly into the
node-block CSR system and its diagonally preconditioned GMRES solve.

The compute runs in ``_lib/libovs_b200.so`` (C ABI: ``include/ovs.h``);
:mod:`oversetdevfort_b200.api` mirrors the reference's routine names.
"""
from . import _ffi
from .api import (Context, genSparStruc, assembleNavSto, assembleQuenching, SparseGMRES_up,
                  SparseGMRES_ns_conv, SparseGMRES_tem, calculate_residual,
                  ASSEMBLE_FIELD_NS, ASSEMBLE_FIELD_VOF, ASSEMBLE_FIELD_TEM,
                  ASSEMBLE_TENSOR_VEC, ASSEMBLE_TENSOR_MAT)
from . import mesh

__all__ = ["Context", "genSparStruc", "assembleNavSto", "assembleQuenching", "SparseGMRES_up",
           "SparseGMRES_ns_conv", "SparseGMRES_tem", "calculate_residual", "mesh", "_ffi",
           "ASSEMBLE_FIELD_NS", "ASSEMBLE_FIELD_VOF", "ASSEMBLE_FIELD_TEM",
           "ASSEMBLE_TENSOR_VEC", "ASSEMBLE_TENSOR_MAT"]
