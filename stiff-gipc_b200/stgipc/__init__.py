"""stgipc -- B200-native (sm_100a) Newton linear solve for StiffGIPC.

Host-side mirror of the reference's linear-system plugin API over libstgipc.so (C ABI in
include/stgipc.h).  ``scenes`` generates seeded synthetic Newton systems in the reference's
triplet layout.
"""
from .linear_system import GlobalLinearSystem, PCGSolverConfig, Solver, StgError  # noqa: F401

__all__ = ["GlobalLinearSystem", "PCGSolverConfig", "Solver", "StgError"]
