"""B200-native SSA (SSTREAM) Newton assembly and solve for Úa.

The compute path is libuassa.so (CUDA, sm_100a) behind the C-ABI in
include/ua_ssa.h; ``uasource_b200.ua`` mirrors the reference's MATLAB
interface on top of it.
"""
from .ua import (CtrlVar, Fields, BCs, HBCs, MUA, CreateMUA, CreateMUABatch, uvMatrixAssembly, uv, uv_batch,  # noqa: F401,E501
                 uv_resident, uv_batch_resident, uvhAssembly, uvh,
                 solveKApeSymmetric, adjoint_gradient_C, constraint_matrix, autotune, RunInfo)
from .lib import UaError  # noqa: F401
