// Host-side projection geometry for elsa_b200.
//
// A pose is described by the projection matrix P = K [R|t] S (index space -> detector pixels),
// its inverse Pinv, the camera (source) centre C in index space, the extrinsic matrix ext and the
// source-detector distance. The formulas and their float evaluation order follow elsa's
// core/Geometry.cpp:12-109,225-270 so that every matrix entry matches the reference's float
// result: all small products are coefficient-wise sequential sums with separate multiply/add,
// and the camera centre comes from a column-pivoting Householder QR solve in float.
//
// Poses travel across the C ABI as 40-float records (see include/elsa_b200.h).
#pragma once

#include <cstdint>
#include <vector>

namespace elsa_b200
{
    constexpr int kPoseFloats = 40;
    constexpr int kPoseOffP = 0;
    constexpr int kPoseOffPinv = 12;
    constexpr int kPoseOffC = 24;
    constexpr int kPoseOffExt = 27;
    constexpr int kPoseOffSdd = 39;

    struct PoseRecord {
        float v[kPoseFloats];
    };

    // One 2D pose: source-to-centre, centre-to-detector, rotation angle (radian), volume spacing
    // and origin (2), detector spacing and origin (1 used), principal point offset, centre of
    // rotation offset (2).
    PoseRecord makePose2d(float s2c, float c2d, float angle, const float* volSpacing,
                          const float* volOrigin, const float* sinoSpacing,
                          const float* sinoOrigin, float ppOffset, const float* corOffset);

    // One 3D pose with YZY Euler angles (gamma, beta, alpha).
    PoseRecord makePose3d(float s2c, float c2d, const float* volSpacing, const float* volOrigin,
                          const float* sinoSpacing, const float* sinoOrigin, float gamma,
                          float beta, float alpha, const float* ppOffset, const float* corOffset);

    // Circular trajectory as elsa's CircleTrajectoryGenerator::createTrajectory builds it:
    // angles LinSpaced(numPoses, 0, arc) (both ends included), detector size defaulting to
    // floor(N*sqrt(2)) and detector spacing to the volume spacing. Fills detDims (dim entries,
    // the last one = numPoses).
    std::vector<PoseRecord> circleTrajectory(int dim, const int64_t* volDims,
                                             const float* volSpacing, int64_t numPoses,
                                             float arcDegrees, float s2c, float c2d,
                                             const int64_t* detSize, const float* detSpacing,
                                             int64_t* detDims);

    // Ordered-subset partitions of the poses (projectors/SubsetSampler.cpp:50-103): subset i of
    // a round robin takes positions i, i + n, i + 2n, ... of `indices`; rotational clustering
    // first sorts the pose indices by the rotation angle to the first pose (2D: the signed angle
    // atan2(R0 R^T (1,0), R0 R^T (0,0)); 3D: acos((trace(R0 R^T) - 1) / 2)), with std::sort as
    // the reference does, then splits them round robin.
    std::vector<std::vector<int>> splitRoundRobin(const std::vector<int>& indices, int nSubsets);
    std::vector<std::vector<int>> splitRotationalClustering(int dim,
                                                            const std::vector<PoseRecord>& poses,
                                                            int nSubsets);

    // Planar detector coordinates of the pixel centres of a curved (cylindrical) detector,
    // CurvedDetectorDescriptor::setup / mapCurvedCoordToPlanarCoord
    // (core/Descriptors/CurvedDetectorDescriptor.cpp:33-91): radius nu / angle, the circle centred
    // s2d - radius in front of the source; every pixel centre on the arc is projected from the
    // source onto the flat detector at distance s2d. Two floats (u', v') per pixel, u fastest
    // (2D: v' = 0). A ray-driven projector casts the ray of pixel (u, v) through (u', v') instead
    // of (u + 0.5, v + 0.5).
    // columnFactor (optional): per column u the factor s2d / depth that stretches its rows.
    std::vector<float> curvedPlanarCoords(int dim, int nu, int nv, float angle, float s2d,
                                          std::vector<float>* columnFactor = nullptr);
} // namespace elsa_b200
