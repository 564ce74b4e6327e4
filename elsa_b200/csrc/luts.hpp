// Lookup tables of the voxel-driven projectors (host side, computed once per projector).
//
// Reference semantics: projectors/Luts.hpp:14-83 (N samples of a profile on [0, support],
// linear interpolation), projectors/Blobs.h:67-245 (projected Kaiser-Bessel blob, its derivative
// and its normalized gradient), projectors/BSplines.h:22-186 (projected B-spline), and
// core/Utilities/Bessel.cpp:6-137 (modified Bessel functions I_m). The tables are computed in the
// reference's float/double mix so that they match elsa's float tables bit for bit.
#pragma once

#include <cstdint>
#include <vector>

namespace elsa_b200
{
    constexpr int kVoxelLutSize = 100; // DEFAULT_PROJECTOR_LUT_SIZE, projectors/Luts.hpp:8

    enum class VoxelBasis { Blob, BSpline };

    // Which profile the table holds: the projected basis function (absorption), its derivative
    // (2D phase contrast) or derivative / s (3D phase contrast).
    enum class LutProfile { Value = 0, Derivative = 1, NormalizedGradient = 2 };

    struct VoxelLut {
        std::vector<float> values;
        float support = 0.0f; // radius of the projected basis function
    };

    // Modified Bessel function of the first kind I_m(x), Abramowitz & Stegun 9.8.1-9.8.4 for
    // m <= 1, upward recurrence for m = 2..4, Miller's downward recurrence above.
    double besselI(int m, double x);

    VoxelLut blobLut(float radius, float alpha, int order, LutProfile profile,
                     int samples = kVoxelLutSize);
    // dim: volume dimension (the projected B-spline is (dim-1)-dimensional).
    VoxelLut bsplineLut(int dim, int order, LutProfile profile, int samples = kVoxelLutSize);
} // namespace elsa_b200
