// Kernels of raysetup.cu (compiled without FMA contraction).
#pragma once

#include "internal.cuh"

namespace elsa_b200
{
    // One JosephRay record per detector pixel and pose; ray index u + nu*(v + nv*p).
    __global__ void josephSetupKernel(const float* __restrict__ poses, VolumeShape vol,
                                      DetectorShape det, JosephRay* __restrict__ rays);
} // namespace elsa_b200
