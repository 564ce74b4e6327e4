// Internal declarations shared by the elsa_b200 CUDA translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include "../../include/elsa_b200.h"

namespace elsa_b200
{
    // Error carrying an elsa_status across the C++ layer; the C ABI converts it to a return
    // code and a thread-local message (elsa_last_error).
    struct Error : std::runtime_error {
        elsa_status status;
        Error(elsa_status s, const std::string& msg) : std::runtime_error(msg), status(s) {}
    };

    inline void cudaCheck(cudaError_t e, const char* what)
    {
        if (e != cudaSuccess)
            throw Error(e == cudaErrorMemoryAllocation ? ELSA_ERROR_BAD_ALLOC : ELSA_ERROR_CUDA,
                        std::string(what) + ": " + cudaGetErrorString(e));
    }

#define ELSA_CUDA(call) ::elsa_b200::cudaCheck((call), #call)
#define ELSA_LAUNCH_CHECK(what) ::elsa_b200::cudaCheck(cudaGetLastError(), what)

    // Per-ray traversal record of the Joseph projector (32 bytes). The driving axis d is the
    // axis of largest |direction|; a < b are the two other axes (2D: only a). Sample j
    // (0 <= j < n) lies on the plane of driving index k0 + j*dir, at non-driving positions
    //   pa_j = fma(j, sa, pa),  pb_j = fma(j, sb, pb).
    // The forward and the adjoint kernels evaluate exactly this expression, which makes the
    // pair an exact transpose. (elsa's CPU code accumulates pos += step instead,
    // projectors/DrivingDirectionTraversal.cpp:265.)
    struct __align__(16) JosephRay {
        float pa, pb, sa, sb;
        float len; // |step| = intersection length per sample
        int k0;    // driving-axis voxel index of sample 0
        int n;     // number of samples, 0 when the ray misses the volume
        int meta;  // bits 0-1 driving axis, bit 2 set when the ray runs towards lower indices
    };

    // Per (brick, view) detector window of the rays that can touch the brick, inclusive.
    struct __align__(16) RayWindow {
        int u0, u1, v0, v1; // empty when u0 > u1
    };

    struct VolumeShape {
        int dim;
        int n[3]; // nx, ny, nz (nz = 1 in 2D)
    };

    struct DetectorShape {
        int nu, nv, np; // nv = 1 in 2D
    };

    __host__ __device__ inline void nonDrivingAxes(int d, int& a, int& b)
    {
        a = (d == 0) ? 1 : 0;
        b = (d == 2) ? 1 : 2;
    }
} // namespace elsa_b200
