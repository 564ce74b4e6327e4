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
    // (0 <= j < n) lies on the plane of driving index k0 + j*dir; its non-driving positions are
    // accumulated in float, pa_{j+1} = pa_j + sa (one rounding per step), exactly like elsa's
    // CPU traversal (projectors/DrivingDirectionTraversal.cpp:265). Kernels that start a ray in
    // the middle read the accumulated position from the slab checkpoints.
    // floor(x) as a float and as an int for |x| < 2^22, on the FMA and integer pipes instead of
    // the conversion pipe (the "magic number" rounding method): x + 1.5 * 2^23 rounded toward
    // -infinity lies in [2^23, 2^24), where the floats are exactly the integers, so it equals
    // 1.5 * 2^23 + floor(x); subtracting the constant back is exact, and the integer is the
    // difference of the two bit patterns (0x4B400000 is the pattern of 1.5 * 2^23). x = -0 does
    // not occur where this is used (x = p - 0.5 rounds to +0 at p = 0.5).
#ifdef __CUDACC__
    // Packed two-wide FP32 arithmetic of sm_100 (add/sub/mul/fma .f32x2): two IEEE operations
    // with the stated rounding in one instruction, on a register pair.
    __device__ __forceinline__ unsigned long long pack2(float2 a)
    {
        unsigned long long r;
        asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
        return r;
    }
    __device__ __forceinline__ float2 unpack2(unsigned long long r)
    {
        float2 a;
        asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
        return a;
    }
    __device__ __forceinline__ float2 add2(float2 a, float2 b)
    {
        unsigned long long r;
        asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pack2(a)), "l"(pack2(b)));
        return unpack2(r);
    }
    __device__ __forceinline__ float2 add2Down(float2 a, float2 b) // rounded toward -infinity
    {
        unsigned long long r;
        asm("add.rm.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pack2(a)), "l"(pack2(b)));
        return unpack2(r);
    }
    __device__ __forceinline__ float2 sub2(float2 a, float2 b)
    {
        unsigned long long r;
        asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pack2(a)), "l"(pack2(b)));
        return unpack2(r);
    }
    __device__ __forceinline__ float2 mul2(float2 a, float2 b)
    {
        unsigned long long r;
        asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pack2(a)), "l"(pack2(b)));
        return unpack2(r);
    }
    __device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) // a * b + c, one rounding
    {
        unsigned long long r;
        asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(pack2(a)), "l"(pack2(b)), "l"(pack2(c)));
        return unpack2(r);
    }

    // floorSmall of both components.
    __device__ __forceinline__ float2 floorSmall2(float2 x, int& i0, int& i1)
    {
        constexpr float kMagic = 12582912.0f; // 1.5 * 2^23
        const float2 t = add2Down(x, make_float2(kMagic, kMagic));
        i0 = __float_as_int(t.x) - 0x4B400000;
        i1 = __float_as_int(t.y) - 0x4B400000;
        return sub2(t, make_float2(kMagic, kMagic));
    }

    __device__ __forceinline__ float floorSmall(float x, int& i)
    {
        constexpr float kMagic = 12582912.0f; // 1.5 * 2^23
        const float t = __fadd_rd(x, kMagic);
        i = __float_as_int(t) - 0x4B400000;
        return __fsub_rn(t, kMagic);
    }
#endif

    struct __align__(16) JosephRay {
        float pa, pb, sa, sb;
        float len; // |step| = intersection length per sample
        int k0;    // driving-axis voxel index of sample 0
        int n;     // number of samples, 0 when the ray misses the volume
        int meta;  // bits 0-1 driving axis, bit 2 set when the ray runs towards lower indices
    };

    // Per-ray record of the Siddon projector (48 bytes): elsa's TraverseAABB state at the entry
    // voxel (projectors/TraverseAABB.cpp:6-40,104-166). g is the axis of largest |direction|
    // (used to cut rays into slabs); every visit advances the axes whose T is minimal.
    struct __align__(16) SiddonRay {
        float tDelta[3]; // |1/d| per axis, FLT_MAX when |d| <= FLT_EPSILON
        int meta;        // bits 0-1 g; bit 2+i: step of axis i is -1; bit 5+i: step of axis i is 0;
                         // bit 8: the ray crosses the volume
        int kFirst;      // entry voxel index along g
        int kLast;       // last voxel index along g
        int cur[2];      // entry voxel indices of the two other axes a < b (2D: b unused)
        float T[3];      // parameter of the first boundary crossing per axis (FLT_MAX if none)
        int crossings;   // number of voxels visited
    };

    // Curved detector as the brick-window kernel sees it: planar coordinate of the ray of every
    // detector column (ascending, null for a flat detector) and the range of the row stretch.
    struct CurvedMap {
        const float* planarU = nullptr;
        float fmin = 1.0f, fmax = 1.0f;
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
