"""tlfea_b200 -- B200-native (sm_100a) TLFEA hot path behind the reference's class API.

The compute runs in ``libtlfea_b200.so`` (hand-written CUDA, C ABI in
include/tlfea_b200.h); this package is the Python mirror of the reference's
FEASolver / element / solver classes plus mesh utilities.
"""
from . import quadrature as Quadrature
from . import mesh
from ._capi import TLFEAError, launch_count, last_error
from .api import (
    FEASolver,
    ElementBase,
    GPU_FEAT10_Data,
    GPU_FEAT4_Data,
    SolverBase,
    SyncedNesterovParams,
    SyncedNesterovSolver,
    SyncedAdamWParams,
    SyncedAdamWNocoopParams,
    SyncedAdamWSolver,
    SyncedAdamWNocoopSolver,
    LinearStaticSolver,
    LinearStaticSolverT10,
    LinearStaticSolverT4,
    BatchedLinearStaticSolver,
    BatchedDynamics,
    WarmStartMLP,
    gemm_bf16,
    gemm_bf16_async,
    TYPE_3243,
    TYPE_3443,
    TYPE_T10,
    TYPE_T4,
    MATERIAL_MODEL_SVK,
    MATERIAL_MODEL_MOONEY_RIVLIN,
)

__all__ = [
    "Quadrature", "mesh", "TLFEAError", "launch_count", "last_error", "FEASolver", "ElementBase",
    "GPU_FEAT10_Data", "GPU_FEAT4_Data", "SolverBase", "SyncedNesterovParams", "SyncedNesterovSolver",
    "SyncedAdamWParams", "SyncedAdamWNocoopParams", "SyncedAdamWSolver", "SyncedAdamWNocoopSolver",
    "LinearStaticSolver", "LinearStaticSolverT10", "LinearStaticSolverT4", "BatchedLinearStaticSolver", "BatchedDynamics", "WarmStartMLP", "gemm_bf16", "gemm_bf16_async", "TYPE_3243", "TYPE_3443", "TYPE_T10",
    "TYPE_T4", "MATERIAL_MODEL_SVK", "MATERIAL_MODEL_MOONEY_RIVLIN",
]
