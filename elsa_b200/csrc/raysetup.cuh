// Kernels of raysetup.cu (compiled without FMA contraction).
#pragma once

#include <cuda_runtime.h>

#include "internal.cuh"

namespace elsa_b200
{
    // One JosephRay record per detector pixel and pose; ray index u + nu*(v + nv*p). planar:
    // per-pixel planar coordinates of a curved detector (null for a flat one).
    __global__ void josephSetupKernel(const float* __restrict__ poses, VolumeShape vol,
                                      DetectorShape det, const float2* __restrict__ planar,
                                      JosephRay* __restrict__ rays);

    // Entry point and lateral slopes of a Siddon ray (setup-time geometry for the ray classes):
    // along axis g the ray passes a = a0 + (x_g - g0) * sa, b = b0 + (x_g - g0) * sb.
    struct SiddonLine {
        float g0, a0, b0, sa, sb;
    };

    // One SiddonRay record (kLast and crossings are filled in by the checkpoint pass) and one
    // SiddonLine per detector pixel and pose; ray index u + nu*(v + nv*p).
    __global__ void siddonSetupKernel(const float* __restrict__ poses, VolumeShape vol,
                                      DetectorShape det, const float2* __restrict__ planar,
                                      SiddonRay* __restrict__ rays,
                                      SiddonLine* __restrict__ lines);

    // Ray-driven LUT projector (LutProjector) parameters: dimension, volume size, LUT samples on
    // [0, radius], neighbourhood `support`, the largest |LUT| value and the six traversal
    // rotations (variant 2 * leading axis + (leading coefficient < 0), row-major 3 x 3; 2D uses
    // the top-left 2 x 2).
    constexpr int kLutProjMaxSamples = 128;
    struct LutProjParams {
        int dim;
        int n[3];
        int lutN;
        int support;
        float radius;
        float maxLut;
        float rot[6][9];
    };

    // 2^k with k such that 4 * nrays contributions of at most absMaxY * maxLut stay below 2^62
    // (0 when there is nothing to add)
    __host__ __device__ inline double lutFixedScale(float absMaxY, float maxLut, int64_t nrays)
    {
        const double bound = static_cast<double>(absMaxY) * static_cast<double>(maxLut) * 4.0 *
                             static_cast<double>(nrays > 0 ? nrays : 1);
        if (!(bound > 0.0) || !(bound < 1e300))
            return 0.0;
        int e = 0;
        frexp(bound, &e); // bound < 2^e
        return ldexp(1.0, 62 - e);
    }

    void launchLutForward(const float* poses, const DetectorShape& det, const LutProjParams& lp,
                          const float* lut, const float* x, float* y, cudaStream_t s);
    // absMaxBits: one device word of scratch; acc: nvox 64-bit words of scratch
    void launchLutBackward(const float* poses, const DetectorShape& det, const LutProjParams& lp,
                           const float* lut, const float* y, unsigned* absMaxBits,
                           unsigned long long* acc, int64_t nvox, float* x, cudaStream_t s);
} // namespace elsa_b200
