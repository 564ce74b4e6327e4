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
#include <utility>
#include <vector>

#include "geometry.hpp"
#include "internal.cuh"

namespace elsa_b200
{
    // Launch parameters ("knobs") that change how a projector's kernels are launched, not the
    // operator: every value gives the same forward and adjoint up to float rounding (adjoint
    // view chunks only change the order in which per-chunk partial volumes are added).
    enum Knob : int {
        kKnobForwardThreads = 0, // rays per block of a thread-per-ray forward kernel
        kKnobAdjointChunks = 1,  // view chunks of a brick-owner adjoint (partial volumes)
        kKnobAdjointThreads = 2, // voxels per block of a thread-per-voxel adjoint kernel
        kKnobAdjointScatter = 3, // 0: deterministic brick-owner adjoint, 1: atomic scatter
        kKnobExactWeights = 4,   // voxel adjoint: 0 the forward's weights, 1 the reference's
        kKnobCheckpointDepth = 5, // planes per checkpoint slab of the 3D Joseph adjoint
        kKnobCount = 6
    };

    // A curved (cylindrical) detector: opening angle (radian) and source-to-detector distance
    // (CurvedDetectorDescriptor); angle 0 is a flat detector.
    struct CurvedDetector {
        float angle = 0.0f;
        float s2d = 0.0f;
        bool enabled() const { return angle > 0.0f; }
    };

    class DeviceBuffer;

    // Device copies of a curved detector's planar pixel coordinates (float2 per pixel) and of
    // the per-column planar u for the brick windows; empty for a flat detector. Needed only
    // while a projector sets up its rays and windows.
    class CurvedTables
    {
    public:
        CurvedTables();
        CurvedTables(int dim, const DetectorShape& det, const CurvedDetector& c);
        ~CurvedTables();
        CurvedTables(CurvedTables&&) noexcept;
        CurvedTables& operator=(CurvedTables&&) noexcept;
        const float2* planar() const;
        CurvedMap map() const;
        void release();

    private:
        std::unique_ptr<DeviceBuffer> planar_, column_;
        float fmin_ = 1.0f, fmax_ = 1.0f;
    };

    class Projector
    {
    public:
        virtual ~Projector();
        virtual void forward(const float* x, float* y, cudaStream_t stream) = 0;
        virtual void adjoint(const float* y, float* x, cudaStream_t stream) = 0;
        // `batch` applies on x + b xStride -> y + b yStride (adjoint: y + b yStride ->
        // x + b xStride), each exactly as a single apply computes it; the default loops.
        virtual void forwardBatch(const float* x, int64_t xStride, float* y, int64_t yStride,
                                  int batch, cudaStream_t stream)
        {
            for (int b = 0; b < batch; ++b)
                forward(x + b * xStride, y + b * yStride, stream);
        }
        virtual void adjointBatch(const float* y, int64_t yStride, float* x, int64_t xStride,
                                  int batch, cudaStream_t stream)
        {
            for (int b = 0; b < batch; ++b)
                adjoint(y + b * yStride, x + b * xStride, stream);
        }

        int64_t domainSize() const { return domainSize_; }
        int64_t rangeSize() const { return rangeSize_; }
        const VolumeShape& volume() const { return vol_; }
        const DetectorShape& detector() const { return det_; }
        int device() const { return device_; }
        int kind() const { return kind_; }
        // Tunables reported for diagnostics (e.g. the conflict-free ray class spacing).
        virtual int64_t info(int key) const { (void)key; return -1; }
        // Values the autotuner may try for `knob` on this geometry (empty: fixed here), the
        // current value (-1: not used by this projector) and setting one of the candidates.
        virtual std::vector<int> knobCandidates(int knob) const
        {
            (void)knob;
            return {};
        }
        virtual int knob(int knob) const
        {
            (void)knob;
            return -1;
        }
        virtual void setKnob(int knob, int value);
        // Test hook of the bounded device waits (elsa_projector_wait_test): false when this
        // projector has none.
        virtual bool setWaitTest(long long cycles, bool withhold)
        {
            (void)cycles, (void)withhold;
            return false;
        }

        // Pipelining of the host-buffer entry points (optional). forwardGroups() > 1: after
        // prepareForward(x), forwardGroup(x, y, g, G) writes the rays of the views
        // [forwardGroupViews(g, G)), so that finished groups can be copied out while later ones
        // run. adjointGroups() > 1: adjointGroup(y, g, G) adds the views
        // [adjointGroupViews(g, G)) (only those must be on the device yet), adjointFinish(x)
        // writes the result. The views of the groups partition [0, np) in order.
        virtual int forwardGroups() const { return 0; }
        virtual int adjointGroups() const { return 0; }
        virtual std::pair<int, int> forwardGroupViews(int g, int G) const
        {
            return {static_cast<int>(static_cast<int64_t>(det_.np) * g / G),
                    static_cast<int>(static_cast<int64_t>(det_.np) * (g + 1) / G)};
        }
        virtual std::pair<int, int> adjointGroupViews(int g, int G) const
        {
            return forwardGroupViews(g, G);
        }
        virtual void prepareForward(const float* x, cudaStream_t s)
        {
            (void)x;
            (void)s;
        }
        virtual void forwardGroup(const float* x, float* y, int g, int G, cudaStream_t s)
        {
            (void)x, (void)y, (void)g, (void)G, (void)s;
        }
        virtual void adjointGroup(const float* y, int g, int G, cudaStream_t s)
        {
            (void)y, (void)g, (void)G, (void)s;
        }
        virtual void adjointFinish(float* x, cudaStream_t s)
        {
            (void)x, (void)s;
        }

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
                                                   const std::vector<PoseRecord>& poses,
                                                   const CurvedDetector& curved = {},
                                                   bool fast = false);
    // binary: BinaryMethod, the Siddon visits with weight 1 (projectors/BinaryMethod.cpp)
    std::unique_ptr<Projector> makeSiddonProjector(const VolumeShape& vol,
                                                   const DetectorShape& det,
                                                   const std::vector<PoseRecord>& poses,
                                                   bool binary = false,
                                                   const CurvedDetector& curved = {});

    struct VoxelLut;
    // Ray-driven blob / B-spline projector (LutProjector): lut on [0, lut.support], the
    // neighbourhood half-width `support` in voxels.
    std::unique_ptr<Projector> makeLutProjector(int kind, const VolumeShape& vol,
                                                const DetectorShape& det,
                                                const std::vector<PoseRecord>& poses,
                                                const VoxelLut& lut, int support);

    // Detector window of every (brick, view) for the brick-owner adjoints (joseph.cu). grow > 0
    // (flat detectors): the pixels whose centres lie in the projection of the brick grown by
    // `grow` voxels, plus `pixMargin` pixels; grow = 0 (and curved detectors): the projection of
    // the brick grown by one voxel, plus one pixel. Windows are indexed view * nBricks + brick.
    void launchBrickWindows(const float* poses, const VolumeShape& vol, const DetectorShape& det,
                            int3 brick, int3 nBricks, RayWindow* out, cudaStream_t s,
                            CurvedMap cm = {}, float grow = 0.0f, float pixMargin = 0.0f);

    // Matched 3D Joseph adjoints of many projectors in one launch per driving-axis grid (batched
    // solves): plan once for fixed sinogram and volume buffers, then run on a stream. Every
    // projector's result equals its own adjoint() bit for bit (same bricks, view chunks and
    // summation order). Throws ELSA_ERROR_NOT_SUPPORTED unless every projector is a 3D matched
    // Joseph operator with its brick-owner adjoint.
    class AdjointManyPlan;
    std::shared_ptr<AdjointManyPlan> planJosephAdjointMany(const std::vector<Projector*>& ops,
                                                           const std::vector<const float*>& ys,
                                                           const std::vector<float*>& xs);
    void runJosephAdjointMany(const AdjointManyPlan& plan, cudaStream_t s);

    // x[v] = sum over c = 0 .. chunks-1 of partial[c * nvox + v], added in chunk order
    // (joseph.cu).
    void launchSumChunks(const float* partial, int chunks, int64_t nvox, float* x,
                         cudaStream_t s);

    // Powers of two up to `limit` plus `extra` (sorted, unique, each >= 1): the candidate
    // view-chunk counts of a brick-owner adjoint.
    std::vector<int> chunkCandidates(int limit, int extra);
} // namespace elsa_b200
