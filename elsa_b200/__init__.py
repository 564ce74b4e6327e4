"""elsa_b200: B200-native X-ray projectors and iterative-solver vector operations with elsa's
operator API.

The compute path is the native library libelsa_b200.so (hand-written sm_100a CUDA kernels behind
a C ABI, include/elsa_b200.h). Importing this package does not need a GPU; calling a projector
does, and fails loudly when the library is missing.
"""
from . import _capi  # noqa: F401
from ._capi import (ElsaError, InvalidArgumentError, Projector, Solver, BatchCGNE,  # noqa: F401
                    voxel_lut, PROJECTOR_BLOB, PROJECTOR_BSPLINE, PROJECTOR_PHASE_CONTRAST_BLOB,
                    PROJECTOR_PHASE_CONTRAST_BSPLINE, FOOTPRINT_REFERENCE, FOOTPRINT_RECTANGLE,
                    circle_trajectory, pose_2d, pose_3d, power_iterations, solve_batch, POSE_FLOATS,
                    PROJECTOR_JOSEPH, PROJECTOR_SIDDON, SOLVER_CGNE, SOLVER_CGLS,
                    SOLVER_LANDWEBER, SOLVER_APGD, SOLVER_SIRT, SOLVER_FGM,
                    SOLVER_OGM, PROX_IDENTITY, PROX_BOX, PROX_L1, KNOB_FORWARD_THREADS,
                    KNOB_ADJOINT_CHUNKS, KNOB_ADJOINT_THREADS, KNOB_ADJOINT_SCATTER, KNOB_EXACT_WEIGHTS,
                    KNOB_CHECKPOINT_DEPTH,
                    tune_cache_size,
                    tune_cache_clear, tune_cache_save, tune_cache_load, tune_cache_put,
                    tune_cache_get, SOLVER_SQS, SUBSET_ROUND_ROBIN,
                    SUBSET_ROTATIONAL_CLUSTERING, subset_split, gather_views, edf_read,
                    edf_write, mhd_read, mhd_write, pgm_write, PROJECTOR_BINARY,
                    curved_detector_coords, PROJECTOR_RAY_BLOB, PROJECTOR_RAY_BSPLINE)

__all__ = ["ElsaError", "InvalidArgumentError", "Projector", "Solver", "BatchCGNE", "voxel_lut",
           "PROJECTOR_BLOB", "PROJECTOR_BSPLINE", "PROJECTOR_PHASE_CONTRAST_BLOB",
           "PROJECTOR_PHASE_CONTRAST_BSPLINE", "FOOTPRINT_REFERENCE", "FOOTPRINT_RECTANGLE",
           "circle_trajectory",
           "pose_2d", "pose_3d", "power_iterations", "solve_batch", "POSE_FLOATS", "PROJECTOR_JOSEPH",
           "PROJECTOR_SIDDON", "SOLVER_CGNE", "SOLVER_CGLS", "SOLVER_LANDWEBER", "SOLVER_APGD",
           "SOLVER_SIRT", "SOLVER_FGM", "SOLVER_OGM",
           "PROX_IDENTITY",
           "PROX_BOX", "PROX_L1", "KNOB_FORWARD_THREADS", "KNOB_ADJOINT_CHUNKS",
           "KNOB_ADJOINT_THREADS", "KNOB_ADJOINT_SCATTER", "KNOB_EXACT_WEIGHTS", "KNOB_CHECKPOINT_DEPTH", "tune_cache_size", "tune_cache_clear", "tune_cache_save",
           "tune_cache_load", "tune_cache_put", "tune_cache_get", "SOLVER_SQS",
           "SUBSET_ROUND_ROBIN", "SUBSET_ROTATIONAL_CLUSTERING", "subset_split", "gather_views",
           "edf_read", "edf_write", "mhd_read", "mhd_write", "pgm_write", "PROJECTOR_BINARY",
           "curved_detector_coords", "PROJECTOR_RAY_BLOB", "PROJECTOR_RAY_BSPLINE"]
