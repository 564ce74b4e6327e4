// Per-ray traversal setup for the ray-driven projectors.
//
// This translation unit is compiled with --fmad=false: every multiply and add below must round
// separately so that the records are bit-identical to elsa's float CPU path:
//   ray:        core/Descriptors/DetectorDescriptor.cpp:90-128 (rd = normalize(Pinv [u+.5,v+.5,1]))
//   intersect:  projectors/Intersection.cpp:7-46 (slab test on [0, N])
//   traversal:  projectors/DrivingDirectionTraversal.cpp:6-57 (driving axis, .5-plane shift,
//               step count, intersection length)
//   Siddon:     projectors/TraverseAABB.cpp:6-40,104-166 (entry voxel, tDelta, first T)
//   LutProjector (ray-driven blob / B-spline): projectors/LutProjector.h:85-163 with
//               SliceTraversal.cpp:7-200, Intersection.cpp:47-119, CartesianIndices.cpp:341-356
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

    // ---- ray-driven LUT projector -----------------------------------------------------------
    namespace
    {
        // Lut::operator() (projectors/Luts.hpp:61-80): linear interpolation of n samples on
        // [0, support], 0 outside
        __device__ __forceinline__ float lutValue(const float* lut, int n, float support,
                                                  float distance)
        {
            const float index = (distance / support) * static_cast<float>(n - 1);
            if (index < 0.0f || index > static_cast<float>(n - 1))
                return 0.0f;
            const int a = static_cast<int>(floorf(index));
            const int b = static_cast<int>(ceilf(index));
            const float fa = lut[a], fb = lut[b];
            const float t = index - static_cast<float>(a);
            return t * fb + (1.0f - t) * fa;
        }

        struct SliceWalk {
            float start[3];
            float step[3];
            int count;
        };

        // SliceTraversal(box [lo, hi], ray) of the reference: the ray and box in traversal
        // coordinates (rotation R of the leading axis onto +x about the box centre hi / 2),
        // intersectXPlanes with its advance / retreat to voxel centres, then the slice walk along
        // the original ray. False when the ray misses.
        __device__ bool sliceWalk(int dim, const float* bmin, const float* bmax, const float* ro,
                                  const float* rd, const float* R, SliceWalk& w)
        {
            float centre[3] = {0.0f, 0.0f, 0.0f}, tcol[3] = {0.0f, 0.0f, 0.0f};
            for (int i = 0; i < dim; ++i)
                centre[i] = bmax[i] / 2.0f;
            for (int i = 0; i < dim; ++i) {
                float acc = 0.0f;
                for (int k = 0; k < dim; ++k)
                    acc = acc + R[i * 3 + k] * (-centre[k]);
                tcol[i] = acc + 0.0f;
            }
            float o[3], d[3], lo[3], hi[3];
            for (int i = 0; i < dim; ++i) {
                float ao = 0.0f, ad = 0.0f, al = 0.0f, ah = 0.0f;
                for (int k = 0; k < dim; ++k) {
                    ao = ao + R[i * 3 + k] * ro[k];
                    ad = ad + R[i * 3 + k] * rd[k];
                    al = al + R[i * 3 + k] * bmin[k];
                    ah = ah + R[i * 3 + k] * bmax[k];
                }
                o[i] = ao + tcol[i];
                d[i] = ad;
                lo[i] = al + tcol[i];
                hi[i] = ah + tcol[i];
                if (lo[i] > hi[i]) {
                    const float t = lo[i];
                    lo[i] = hi[i];
                    hi[i] = t;
                }
            }
            lo[0] = lo[0] + 0.5f;
            hi[0] = hi[0] - 0.5f;
            float inv = 1.0f / d[0];
            float t1 = (lo[0] - o[0]) * inv, t2 = (hi[0] - o[0]) * inv;
            float tmin = inv >= 0.0f ? t1 : t2, tmax = inv >= 0.0f ? t2 : t1;
            const float txmin = tmin, txmax = tmax;
            for (int i = 1; i < dim; ++i) {
                inv = 1.0f / d[i];
                t1 = (lo[i] - o[i]) * inv;
                t2 = (hi[i] - o[i]) * inv;
                tmin = maxNum(tmin, inv >= 0.0f ? t1 : t2);
                tmax = minNum(tmax, inv >= 0.0f ? t2 : t1);
            }
            const float xc = fabsf(lo[0] - static_cast<float>(static_cast<int>(roundf(lo[0]))));
            if (txmin < tmin) {
                const float e = o[0] + tmin * d[0];
                float ip;
                const float tmp = fabsf(modff(e - xc, &ip));
                const float frac = e < xc ? tmp : 1.0f - tmp;
                tmin = tmin + ((static_cast<double>(tmp) > 0.00001 &&
                                static_cast<double>(frac) > 0.00001)
                                   ? frac / d[0]
                                   : 0.0f);
            }
            if (txmax > tmax) {
                const float e = o[0] + tmax * d[0];
                float ip;
                const float tmp = fabsf(modff(e - xc, &ip));
                const float frac = e < xc ? 1.0f - tmp : tmp;
                tmax = tmax - ((static_cast<double>(tmp) > 0.00001 &&
                                static_cast<double>(frac) > 0.00001)
                                   ? frac / d[0]
                                   : 0.0f);
            }
            if (tmax == 0.0f && tmin == 0.0f)
                return false;
            if (!(static_cast<double>(tmax - maxNum(tmin, 0.0f)) > -0.000001))
                return false;
            const float first = o[0] + tmin * d[0], last = o[0] + tmax * d[0];
            w.count = max(1, static_cast<int>(ceilf(last - first + 0.5f)));
            const float tDelta = 1.0f / d[0];
            for (int i = 0; i < 3; ++i) {
                w.start[i] = i < dim ? ro[i] + tmin * rd[i] : 0.0f;
                w.step[i] = i < dim ? rd[i] * tDelta : 0.0f;
            }
            return true;
        }

        // Every (voxel, weight) of one ray (LutProjector.h:85-163): the slice walk over the
        // volume box (forward) or the box grown by `support` off the leading axis (backward), and
        // per slice the voxels within `support` in the other axes, last axis fastest.
        template <class F>
        __device__ __forceinline__ void lutRay(const LutProjParams& lp, const float* lut,
                                               const float* ro, const float* rd, bool backward,
                                               F&& f)
        {
            const int dim = lp.dim;
            int lead = 0;
            float best = fabsf(rd[0]);
            for (int i = 1; i < dim; ++i)
                if (fabsf(rd[i]) > best) {
                    best = fabsf(rd[i]);
                    lead = i;
                }
            const int variant = lead * 2 + (rd[lead] >= 0.0f ? 0 : 1);
            float bmin[3] = {0.0f, 0.0f, 0.0f}, bmax[3] = {0.0f, 0.0f, 0.0f};
            for (int i = 0; i < dim; ++i) {
                bmax[i] = static_cast<float>(lp.n[i]);
                if (backward && i != lead) {
                    bmin[i] = bmin[i] - static_cast<float>(lp.support);
                    bmax[i] = bmax[i] + static_cast<float>(lp.support);
                }
            }
            SliceWalk w;
            if (!sliceWalk(dim, bmin, bmax, ro, rd, lp.rot[variant], w))
                return;
            float cur[3] = {w.start[0], w.start[1], w.start[2]};
            for (int it = 0; it < w.count; ++it) {
                int from[3] = {0, 0, 0}, to[3] = {1, 1, 1};
                for (int i = 0; i < dim; ++i) {
                    const int pos = static_cast<int>(cur[i]);
                    const int dist = i == lead ? 0 : lp.support;
                    from[i] = max(pos - dist, 0);
                    to[i] = min(pos + dist + 1, lp.n[i]);
                    if (to[i] == from[i])
                        from[i] -= 1;
                }
                for (int a = from[0]; a < to[0]; ++a)
                    for (int b = from[1]; b < to[1]; ++b)
                        for (int c = from[2]; c < (dim == 3 ? to[2] : from[2] + 1); ++c) {
                            const int nb[3] = {a, b, c};
                            float diff[3], dot = 0.0f;
                            for (int i = 0; i < dim; ++i)
                                diff[i] = (static_cast<float>(nb[i]) + 0.5f) - ro[i];
                            for (int i = 0; i < dim; ++i)
                                dot = dot + rd[i] * diff[i];
                            float sq = 0.0f;
                            for (int i = 0; i < dim; ++i) {
                                const float v = diff[i] - dot * rd[i];
                                sq = sq + v * v;
                            }
                            const float wt = lutValue(lut, lp.lutN, lp.radius, sqrtf(sq));
                            const int64_t idx =
                                a + static_cast<int64_t>(lp.n[0]) *
                                        (b + (dim == 3 ? static_cast<int64_t>(lp.n[1]) * c : 0));
                            if (a >= 0 && b >= 0 && c >= 0)
                                f(idx, wt);
                        }
                for (int i = 0; i < dim; ++i)
                    cur[i] = cur[i] + w.step[i];
            }
        }

        __global__ void lutForwardKernel(const float* __restrict__ poses, DetectorShape det,
                                         LutProjParams lp, const float* __restrict__ lutIn,
                                         const float* __restrict__ x, float* __restrict__ y)
        {
            __shared__ float lut[kLutProjMaxSamples];
            for (int i = threadIdx.x; i < lp.lutN; i += blockDim.x)
                lut[i] = lutIn[i];
            __syncthreads();
            const int64_t nrays = static_cast<int64_t>(det.nu) * det.nv * det.np;
            const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            if (r >= nrays)
                return;
            const int u = static_cast<int>(r % det.nu);
            const int v = static_cast<int>((r / det.nu) % det.nv);
            const int p = static_cast<int>(r / (static_cast<int64_t>(det.nu) * det.nv));
            float o[3] = {0, 0, 0}, d[3] = {0, 0, 0};
            pixelRay(poses + static_cast<int64_t>(p) * 40, lp.dim, u, v, nullptr, det.nu, o, d);
            float acc = 0.0f;
            lutRay(lp, lut, o, d, false,
                   [&](int64_t idx, float wt) { acc = acc + wt * __ldg(x + idx); });
            y[r] = acc;
        }

        // Backward in 64-bit fixed point: every contribution w * y is rounded once to a multiple
        // of 2^-k and the integer sums are exact, so the result does not depend on the order of
        // the atomic additions. 2^k keeps any sum of up to 4 * nrays contributions of at most
        // max|y| * max|lut| below 2^62.
        __global__ void lutBackwardKernel(const float* __restrict__ poses, DetectorShape det,
                                          LutProjParams lp, const float* __restrict__ lutIn,
                                          const float* __restrict__ y,
                                          const unsigned* __restrict__ absMaxBits,
                                          unsigned long long* __restrict__ acc)
        {
            __shared__ float lut[kLutProjMaxSamples];
            for (int i = threadIdx.x; i < lp.lutN; i += blockDim.x)
                lut[i] = lutIn[i];
            __syncthreads();
            const int64_t nrays = static_cast<int64_t>(det.nu) * det.nv * det.np;
            const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            if (r >= nrays)
                return;
            const double scale = lutFixedScale(__uint_as_float(*absMaxBits), lp.maxLut, nrays);
            const float yv = y[r];
            if (yv == 0.0f || scale == 0.0)
                return;
            const int u = static_cast<int>(r % det.nu);
            const int v = static_cast<int>((r / det.nu) % det.nv);
            const int p = static_cast<int>(r / (static_cast<int64_t>(det.nu) * det.nv));
            float o[3] = {0, 0, 0}, d[3] = {0, 0, 0};
            pixelRay(poses + static_cast<int64_t>(p) * 40, lp.dim, u, v, nullptr, det.nu, o, d);
            lutRay(lp, lut, o, d, true, [&](int64_t idx, float wt) {
                const float c = wt * yv;
                const long long q = __double2ll_rn(static_cast<double>(c) * scale);
                if (q != 0)
                    atomicAdd(acc + idx, static_cast<unsigned long long>(q));
            });
        }

        __global__ void absMaxKernel(const float* __restrict__ y, int64_t n,
                                     unsigned* __restrict__ out)
        {
            unsigned m = 0;
            for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
                 i += static_cast<int64_t>(gridDim.x) * blockDim.x)
                m = max(m, __float_as_uint(fabsf(y[i])));
            for (int off = 16; off > 0; off >>= 1)
                m = max(m, __shfl_xor_sync(0xffffffffu, m, off));
            if ((threadIdx.x & 31) == 0 && m)
                atomicMax(out, m);
        }

        __global__ void fixedToFloatKernel(const unsigned long long* __restrict__ acc, int64_t n,
                                           const unsigned* __restrict__ absMaxBits,
                                           float lutMax, int64_t nrays, float* __restrict__ x)
        {
            const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            if (i >= n)
                return;
            const double scale = lutFixedScale(__uint_as_float(*absMaxBits), lutMax, nrays);
            x[i] = scale == 0.0 ? 0.0f
                                : static_cast<float>(static_cast<double>(
                                                         static_cast<long long>(acc[i])) /
                                                     scale);
        }
    } // namespace

    void launchLutForward(const float* poses, const DetectorShape& det, const LutProjParams& lp,
                          const float* lut, const float* x, float* y, cudaStream_t s)
    {
        const int64_t nrays = static_cast<int64_t>(det.nu) * det.nv * det.np;
        if (nrays == 0)
            return;
        lutForwardKernel<<<static_cast<unsigned>((nrays + 127) / 128), 128, 0, s>>>(
            poses, det, lp, lut, x, y);
    }

    void launchLutBackward(const float* poses, const DetectorShape& det, const LutProjParams& lp,
                           const float* lut, const float* y, unsigned* absMaxBits,
                           unsigned long long* acc, int64_t nvox, float* x, cudaStream_t s)
    {
        const int64_t nrays = static_cast<int64_t>(det.nu) * det.nv * det.np;
        cudaMemsetAsync(absMaxBits, 0, sizeof(unsigned), s);
        cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * static_cast<size_t>(nvox), s);
        if (nrays > 0) {
            absMaxKernel<<<592, 256, 0, s>>>(y, nrays, absMaxBits);
            lutBackwardKernel<<<static_cast<unsigned>((nrays + 127) / 128), 128, 0, s>>>(
                poses, det, lp, lut, y, absMaxBits, acc);
        }
        if (nvox > 0)
            fixedToFloatKernel<<<static_cast<unsigned>((nvox + 255) / 256), 256, 0, s>>>(
                acc, nvox, absMaxBits, lp.maxLut, nrays, x);
    }
} // namespace elsa_b200
