// Voxel-driven (blob / B-spline) projectors, see voxel.cu.
#pragma once

#include <memory>
#include <vector>

#include "luts.hpp"
#include "projector.hpp"

namespace elsa_b200
{
    // Pixel loop per (voxel, pose): Reference follows elsa's CPU loop as written
    // (projectors/VoxelComputation.h:88-113); Rectangle visits the clamped footprint rectangle.
    enum class FootprintMode { Reference = 0, Rectangle = 1 };

    // lut: the basis profile sampled on [0, support] (luts.hpp); phaseContrast selects the
    // differential weight (PhaseContrastProjector.cpp) instead of the classic one.
    std::unique_ptr<Projector> makeVoxelProjector(int kind, const VolumeShape& vol,
                                                  const DetectorShape& det,
                                                  const std::vector<PoseRecord>& poses,
                                                  const VoxelLut& lut, bool phaseContrast,
                                                  FootprintMode mode);
} // namespace elsa_b200
