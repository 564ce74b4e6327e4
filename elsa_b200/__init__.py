"""elsa_b200: B200-native X-ray projectors and iterative-solver vector operations with elsa's
operator API.

The compute path is the native library libelsa_b200.so (hand-written sm_100a CUDA kernels behind
a C ABI, include/elsa_b200.h). Importing this package does not need a GPU; calling a projector
does, and fails loudly when the library is missing.
"""
from . import _capi  # noqa: F401
from ._capi import (ElsaError, InvalidArgumentError, Projector, circle_trajectory,  # noqa: F401
                    pose_2d, pose_3d, POSE_FLOATS, PROJECTOR_JOSEPH, SOLVER_CGNE, Solver)

__all__ = ["ElsaError", "InvalidArgumentError", "Projector", "circle_trajectory", "pose_2d",
           "pose_3d", "POSE_FLOATS", "PROJECTOR_JOSEPH", "SOLVER_CGNE", "Solver"]
