// Ray-driven blob / B-spline projector (elsa's LutProjector: BlobProjector, BSplineProjector,
// projectors/LutProjector.h:85-241, LutProjector.cpp:9-90). The kernels are in raysetup.cu,
// which is compiled without FMA contraction; this file holds the operator.
//
// forward: thread per ray, the reference's slice walk and neighbourhood order, sums in that
// order (bit-identical to a sequential restatement). adjoint: thread per ray with 64-bit
// fixed-point atomic sums, so that the result is deterministic. As in the reference, the
// adjoint walks the volume box grown by the support and the forward the volume box itself, so
// the two are not exact transposes of each other near the box faces.
#include "luts.hpp"
#include "projector.hpp"
#include "raysetup.cuh"
#include "solvers.hpp"
#include "voxel.hpp"

#include <algorithm>
#include <cmath>

namespace elsa_b200
{
    namespace
    {
        // TransformToTraversal::create2DRotation / create3DRotation
        // (projectors/SliceTraversal.cpp:9-78), evaluated with the float std::cos / std::sin
        void traversalRotations(int dim, float (&rot)[6][9])
        {
            const float pi = static_cast<float>(3.14159265358979323846);
            const float half = static_cast<float>(0.5 * static_cast<double>(pi));
            for (auto& m : rot)
                for (int i = 0; i < 9; ++i)
                    m[i] = (i % 4 == 0) ? 1.0f : 0.0f;
            auto set2 = [&](float* m, float rad) {
                const float c = std::cos(rad), s = std::sin(rad);
                m[0] = c, m[1] = -s, m[3] = s, m[4] = c;
            };
            auto rotY = [&](float* m, float rad) {
                const float c = std::cos(rad), s = std::sin(rad);
                const float v[9] = {c, 0, s, 0, 1, 0, -s, 0, c};
                std::copy(v, v + 9, m);
            };
            auto rotZ = [&](float* m, float rad) {
                const float c = std::cos(rad), s = std::sin(rad);
                const float v[9] = {c, -s, 0, s, c, 0, 0, 0, 1};
                std::copy(v, v + 9, m);
            };
            if (dim == 2) {
                set2(rot[0], 0.0f);       // leading x, >= 0
                set2(rot[1], pi);         // leading x, < 0
                set2(rot[2], 3 * pi / 2); // leading y, >= 0
                set2(rot[3], pi / 2);     // leading y, < 0
                return;
            }
            rotY(rot[1], pi);
            rotZ(rot[2], -half);
            rotZ(rot[3], half);
            rotY(rot[4], half);
            rotY(rot[5], -half);
        }

        class LutProjector final : public Projector
        {
        public:
            LutProjector(int kind, const VolumeShape& vol, const DetectorShape& det,
                         const std::vector<PoseRecord>& poses, const VoxelLut& lut, int support)
                : Projector(kind, vol, det, poses),
                  lut_(sizeof(float) * lut.values.size()),
                  absMax_(sizeof(unsigned)),
                  acc_(sizeof(unsigned long long) * static_cast<size_t>(domainSize_))
            {
                if (lut.values.empty() || lut.values.size() > kLutProjMaxSamples)
                    throw Error(ELSA_ERROR_LOGIC, "LutProjector: lookup table size");
                lp_.dim = vol.dim;
                lp_.n[0] = vol.n[0], lp_.n[1] = vol.n[1], lp_.n[2] = vol.n[2];
                lp_.lutN = static_cast<int>(lut.values.size());
                lp_.support = support;
                lp_.radius = lut.support;
                float mx = 0.0f;
                for (float v : lut.values)
                    mx = std::max(mx, std::fabs(v));
                lp_.maxLut = mx;
                traversalRotations(vol.dim, lp_.rot);
                ELSA_CUDA(cudaMemcpy(lut_.as<float>(), lut.values.data(),
                                     sizeof(float) * lut.values.size(), cudaMemcpyHostToDevice));
            }

            void forward(const float* x, float* y, cudaStream_t s) override
            {
                launchLutForward(dPoses_, det_, lp_, lut_.as<float>(), x, y, s);
                ELSA_LAUNCH_CHECK("lutForwardKernel");
            }

            void adjoint(const float* y, float* x, cudaStream_t s) override
            {
                launchLutBackward(dPoses_, det_, lp_, lut_.as<float>(), y, absMax_.as<unsigned>(),
                                  acc_.as<unsigned long long>(), domainSize_, x, s);
                ELSA_LAUNCH_CHECK("lutBackwardKernel");
            }

            int64_t info(int key) const override
            {
                switch (key) {
                case 6: // kernel launches per forward call
                    return 1;
                case 7: // per adjoint call: |y| maximum, fixed-point sums, conversion
                    return 3;
                default:
                    return -1;
                }
            }

        private:
            DeviceBuffer lut_, absMax_, acc_;
            LutProjParams lp_{};
        };
    } // namespace

    std::unique_ptr<Projector> makeLutProjector(int kind, const VolumeShape& vol,
                                                const DetectorShape& det,
                                                const std::vector<PoseRecord>& poses,
                                                const VoxelLut& lut, int support)
    {
        return std::make_unique<LutProjector>(kind, vol, det, poses, lut, support);
    }
} // namespace elsa_b200
