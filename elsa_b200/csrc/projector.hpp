// Device projectors behind the C ABI.
//
// A projector owns its geometry (pose records uploaded to the device) and any per-geometry
// tables; callers own the input and output buffers. forward() computes y = A x and adjoint()
// x = A^T y on device pointers, asynchronously on the given stream. Outputs are fully
// overwritten (the reference requires projectors to zero their outputs,
// projectors/tests/test_JosephsMethod.cpp:322-436).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

#include "geometry.hpp"
#include "internal.cuh"

namespace elsa_b200
{
    class Projector
    {
    public:
        virtual ~Projector();
        virtual void forward(const float* x, float* y, cudaStream_t stream) = 0;
        virtual void adjoint(const float* y, float* x, cudaStream_t stream) = 0;

        int64_t domainSize() const { return domainSize_; }
        int64_t rangeSize() const { return rangeSize_; }
        const VolumeShape& volume() const { return vol_; }
        const DetectorShape& detector() const { return det_; }
        int device() const { return device_; }
        int kind() const { return kind_; }
        // Tunables reported for diagnostics (e.g. the conflict-free ray class spacing).
        virtual int64_t info(int key) const { (void)key; return -1; }

    protected:
        Projector(int kind, const VolumeShape& vol, const DetectorShape& det,
                  const std::vector<PoseRecord>& poses);
        int kind_;
        VolumeShape vol_;
        DetectorShape det_;
        int device_ = 0;
        int64_t domainSize_ = 0, rangeSize_ = 0;
        std::vector<PoseRecord> poses_;
        float* dPoses_ = nullptr;
    };

    std::unique_ptr<Projector> makeJosephProjector(const VolumeShape& vol,
                                                   const DetectorShape& det,
                                                   const std::vector<PoseRecord>& poses);
    std::unique_ptr<Projector> makeSiddonProjector(const VolumeShape& vol,
                                                   const DetectorShape& det,
                                                   const std::vector<PoseRecord>& poses);

    // Detector window of every (brick, view) for the brick-owner adjoints: the projection of the
    // brick grown by one voxel, plus one pixel (joseph.cu). Windows are indexed view * nBricks +
    // brick.
    void launchBrickWindows(const float* poses, const VolumeShape& vol, const DetectorShape& det,
                            int3 brick, int3 nBricks, RayWindow* out, cudaStream_t s);
} // namespace elsa_b200
