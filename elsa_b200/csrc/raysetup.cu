// Per-ray traversal setup for the ray-driven projectors.
//
// This translation unit is compiled with --fmad=false: every multiply and add below must round
// separately so that the records are bit-identical to elsa's float CPU path:
//   ray:        core/Descriptors/DetectorDescriptor.cpp:90-128 (rd = normalize(Pinv [u+.5,v+.5,1]))
//   intersect:  projectors/Intersection.cpp:7-46 (slab test on [0, N])
//   traversal:  projectors/DrivingDirectionTraversal.cpp:6-57 (driving axis, .5-plane shift,
//               step count, intersection length)
//   Siddon:     projectors/TraverseAABB.cpp:6-40,104-166 (entry voxel, tDelta, first T)
#include "internal.cuh"
#include "raysetup.cuh"

#include <cfloat>

namespace elsa_b200
{
    namespace
    {
        __device__ __forceinline__ float minNum(float x, float y)
        {
            return (y != y) ? x : (x < y ? x : y);
        }
        __device__ __forceinline__ float maxNum(float x, float y)
        {
            return (y != y) ? x : (x > y ? x : y);
        }

        // Ray through the centre of pixel (u, v) of a pose record, or, for a curved detector,
        // through the planar coordinate planar[u + nu * v] of that pixel centre
        // (CurvedDetectorDescriptor::computeRayFromDetectorCoord,
        // core/Descriptors/CurvedDetectorDescriptor.cpp:93-120).
        __device__ void pixelRay(const float* pose, int dim, int u, int v, const float2* planar,
                                 int nu, float* o, float* d)
        {
            const float* Pinv = pose + 12;
            float h0 = static_cast<float>(u) + 0.5f;
            float h1 = (dim == 3) ? static_cast<float>(v) + 0.5f : 1.0f;
            if (planar) {
                const float2 c = planar[u + static_cast<int64_t>(nu) * v];
                h0 = c.x;
                if (dim == 3)
                    h1 = c.y;
            }
            float dir[3];
            if (dim == 3) {
                for (int i = 0; i < 3; ++i) {
                    float s = 0.0f;
                    s = s + Pinv[i * 3 + 0] * h0;
                    s = s + Pinv[i * 3 + 1] * h1;
                    s = s + Pinv[i * 3 + 2] * 1.0f;
                    dir[i] = s;
                }
            } else {
                for (int i = 0; i < 2; ++i) {
                    float s = 0.0f;
                    s = s + Pinv[i * 2 + 0] * h0;
                    s = s + Pinv[i * 2 + 1] * 1.0f;
                    dir[i] = s;
                }
                dir[2] = 0.0f;
            }
            float z = dir[0] * dir[0];
            z = z + dir[1] * dir[1];
            if (dim == 3)
                z = z + dir[2] * dir[2];
            const float nrm = sqrtf(z);
            for (int i = 0; i < dim; ++i) {
                d[i] = z > 0.0f ? dir[i] / nrm : dir[i];
                o[i] = pose[24 + i];
            }
        }

        __device__ bool slabIntersect(const float* boxMax, int dim, const float* o, const float* d,
                                      float& tmin, float& tmax)
        {
            float inv = 1.0f / d[0];
            float t1 = (0.0f - o[0]) * inv;
            float t2 = (boxMax[0] - o[0]) * inv;
            tmin = inv >= 0.0f ? t1 : t2;
            tmax = inv >= 0.0f ? t2 : t1;
            for (int i = 1; i < dim; ++i) {
                inv = 1.0f / d[i];
                t1 = (0.0f - o[i]) * inv;
                t2 = (boxMax[i] - o[i]) * inv;
                tmin = maxNum(tmin, inv >= 0.0f ? t1 : t2);
                tmax = minNum(tmax, inv >= 0.0f ? t2 : t1);
            }
            if (tmax == 0.0f && tmin == 0.0f)
                return false;
            return tmax >= maxNum(tmin, 0.0f);
        }
    } // namespace

    __global__ void josephSetupKernel(const float* __restrict__ poses, VolumeShape vol,
                                      DetectorShape det, const float2* __restrict__ planar,
                                      JosephRay* __restrict__ rays)
    {
        const int64_t nrays = static_cast<int64_t>(det.nu) * det.nv * det.np;
        const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
        if (r >= nrays)
            return;
        const int dim = vol.dim;
        const int u = static_cast<int>(r % det.nu);
        const int v = static_cast<int>((r / det.nu) % det.nv);
        const int p = static_cast<int>(r / (static_cast<int64_t>(det.nu) * det.nv));
        float o[3] = {0, 0, 0}, d[3] = {0, 0, 0};
        pixelRay(poses + static_cast<int64_t>(p) * 40, dim, u, v, planar, det.nu, o, d);
        float boxMax[3] = {static_cast<float>(vol.n[0]), static_cast<float>(vol.n[1]),
                           static_cast<float>(vol.n[2])};
        float tmin, tmax;
        const bool hit = slabIntersect(boxMax, dim, o, d, tmin, tmax);
        int drv = 0;
        float best = fabsf(d[0]);
        for (int i = 1; i < dim; ++i)
            if (fabsf(d[i]) > best) {
                best = fabsf(d[i]);
                drv = i;
            }
        int a, b;
        nonDrivingAxes(drv, a, b);
        JosephRay rec;
        rec.pa = rec.pb = rec.sa = rec.sb = rec.len = 0.0f;
        rec.k0 = 0;
        rec.n = 0;
        rec.meta = drv;
        if (hit) {
            float pos[3] = {0, 0, 0}, ex[3] = {0, 0, 0}, step[3] = {0, 0, 0};
            for (int i = 0; i < dim; ++i) {
                pos[i] = o[i] + d[i] * tmin;
                ex[i] = o[i] + d[i] * tmax;
                pos[i] = pos[i] < 0.0f ? 0.0f : pos[i];
                pos[i] = pos[i] > boxMax[i] ? boxMax[i] : pos[i];
                ex[i] = ex[i] < 0.0f ? 0.0f : ex[i];
                ex[i] = ex[i] > boxMax[i] ? boxMax[i] : ex[i];
            }
            const float absd = fabsf(d[drv]);
            for (int i = 0; i < dim; ++i)
                step[i] = d[i] / absd;
            const float dist = pos[drv] - floorf(pos[drv]);
            const float sgn = step[drv] > 0.0f ? 1.0f : (step[drv] < 0.0f ? -1.0f : 0.0f);
            const float shift = 0.5f - dist;
            for (int i = 0; i < dim; ++i)
                pos[i] = pos[i] + (step[i] * shift) * sgn;
            pos[drv] = floorf(pos[drv]) + 0.5f;
            const float nsteps = ceilf(fabsf(ex[drv] - pos[drv]));
            float len;
            if (dim == 3)
                len = sqrtf(step[0] * step[0] + (step[1] * step[1] + step[2] * step[2]));
            else
                len = sqrtf(step[0] * step[0] + step[1] * step[1]);
            rec.pa = pos[a];
            rec.sa = step[a];
            if (dim == 3) {
                rec.pb = pos[b];
                rec.sb = step[b];
            }
            rec.len = len;
            rec.k0 = static_cast<int>(floorf(pos[drv] - 0.5f));
            rec.n = static_cast<int>(nsteps);
            rec.meta = drv | (sgn < 0.0f ? 4 : 0);
        }
        rays[r] = rec;
    }

    __global__ void siddonSetupKernel(const float* __restrict__ poses, VolumeShape vol,
                                      DetectorShape det, const float2* __restrict__ planar,
                                      SiddonRay* __restrict__ rays,
                                      SiddonLine* __restrict__ lines)
    {
        const int64_t nrays = static_cast<int64_t>(det.nu) * det.nv * det.np;
        const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
        if (r >= nrays)
            return;
        const int dim = vol.dim;
        const int u = static_cast<int>(r % det.nu);
        const int v = static_cast<int>((r / det.nu) % det.nv);
        const int p = static_cast<int>(r / (static_cast<int64_t>(det.nu) * det.nv));
        float o[3] = {0, 0, 0}, d[3] = {0, 0, 0};
        pixelRay(poses + static_cast<int64_t>(p) * 40, dim, u, v, planar, det.nu, o, d);
        float boxMax[3] = {static_cast<float>(vol.n[0]), static_cast<float>(vol.n[1]),
                           static_cast<float>(vol.n[2])};
        float tmin, tmax;
        bool inBox = slabIntersect(boxMax, dim, o, d, tmin, tmax);
        int g = 0;
        float best = fabsf(d[0]);
        for (int i = 1; i < dim; ++i)
            if (fabsf(d[i]) > best) {
                best = fabsf(d[i]);
                g = i;
            }
        int a, b;
        nonDrivingAxes(g, a, b);
        SiddonRay rec;
        for (int i = 0; i < 3; ++i) {
            rec.tDelta[i] = FLT_MAX;
            rec.T[i] = FLT_MAX;
        }
        rec.meta = g;
        rec.kFirst = rec.kLast = 0;
        rec.cur[0] = rec.cur[1] = 0;
        rec.crossings = 0;
        SiddonLine line{0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        if (inBox) {
            // entry point clamped to the box, TraverseAABB.cpp:13-20
            float entry[3] = {0, 0, 0}, cur[3] = {0, 0, 0};
            int stepDir[3] = {0, 0, 0};
            for (int i = 0; i < dim; ++i) {
                float e = o[i] + d[i] * tmin;
                e = e < 0.0f ? 0.0f : e;
                e = e > boxMax[i] ? boxMax[i] : e;
                entry[i] = e;
                stepDir[i] = d[i] > 0.0f ? 1 : (d[i] < 0.0f ? -1 : 0);
            }
            // entry voxel (one lower on a boundary when stepping down), :123-137
            for (int i = 0; i < dim; ++i) {
                float lc = floorf(entry[i]);
                if (lc == entry[i] && stepDir[i] < 0)
                    lc = lc - 1.0f;
                cur[i] = lc;
                if (cur[i] >= boxMax[i] || cur[i] < 0.0f)
                    inBox = false;
            }
            if (inBox) {
                for (int i = 0; i < dim; ++i) {
                    const bool moves = fabsf(d[i]) > FLT_EPSILON;
                    rec.tDelta[i] = moves ? static_cast<float>(stepDir[i]) / d[i] : FLT_MAX;
                    const float bound = d[i] > 0.0f ? cur[i] + 1.0f : cur[i];
                    rec.T[i] = moves ? (bound - entry[i]) / d[i] : FLT_MAX;
                    if (stepDir[i] < 0)
                        rec.meta |= 4 << i;
                    if (stepDir[i] == 0)
                        rec.meta |= 32 << i;
                }
                rec.meta |= 256;
                rec.kFirst = rec.kLast = static_cast<int>(cur[g]);
                rec.cur[0] = static_cast<int>(cur[a]);
                rec.cur[1] = dim == 3 ? static_cast<int>(cur[b]) : 0;
                line.g0 = entry[g];
                line.a0 = entry[a];
                line.sa = d[a] / d[g];
                if (dim == 3) {
                    line.b0 = entry[b];
                    line.sb = d[b] / d[g];
                }
            }
        }
        rays[r] = rec;
        if (lines)
            lines[r] = line;
    }
} // namespace elsa_b200
