"""B200-native WIEN2k lapw1 Hamiltonian/overlap setup (HAMILT + HNS + HORB).

The compute path is the C-ABI library built from hack_wein2k_b200/csrc
(CUDA for sm_100a); this package is its host-side mirror: problem
marshalling, basis construction (COORS/LOPW), seeded workloads, the
k-point batch driver and the force adjoint.
"""
from .problem import Problem, CProblem, CStats, hermitian_from_packed  # noqa: F401

__all__ = ["Problem", "CProblem", "CStats", "hermitian_from_packed"]
