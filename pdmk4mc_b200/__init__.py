"""pdmk4mc_b200 — periodic DMK electrostatics for Monte Carlo on one B200.

The compute path is the CUDA library libhpdmk_b200.so (sm_100a) behind the
C-ABI declared in include/hpdmk.h; this package is its Python host mirror of
the reference's HPDMKPtTree<double> interface. There is no CPU fallback:
importing the package fails when the library is missing, and every call
fails with HPDMKError when the CUDA path does.
"""
from .tree import (DIRECT, MC_GRAPH, MC_PERSISTENT, PRECISION_FP64, PRECISION_MIXED, PROXY, STATIC_MAX_MOVES, HPDMKError, HPDMKParams, HPDMKPtTree, launch_count, library_path, read_particle_info, replicas_energy, replicas_mc_run, load_library, prolate_setup)

__all__ = ["DIRECT", "MC_GRAPH", "MC_PERSISTENT", "PRECISION_FP64", "PRECISION_MIXED", "PROXY", "STATIC_MAX_MOVES", "HPDMKError", "HPDMKParams", "HPDMKPtTree", "launch_count", "library_path", "read_particle_info", "replicas_energy", "replicas_mc_run", "load_library", "prolate_setup"]
