// Kernels of raysetup.cu (compiled without FMA contraction).
#pragma once

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
} // namespace elsa_b200
