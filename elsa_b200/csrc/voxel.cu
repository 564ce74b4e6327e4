// Voxel-driven projectors (blob / B-spline basis functions, absorption and phase contrast).
//
// Reference semantics: projectors/VoxelComputation.h:20-185 (visitDetector, forwardVoxel,
// backwardVoxel), projectors/VoxelProjector.cpp:30-114 and PhaseContrastProjector.cpp:30-119.
// For every (voxel, pose) the voxel centre is projected onto the detector, centre
// c = hnormalized(P [v + .5; 1]) - .5, scaling s = sdd / |ext [v + .5; 1]|, and every pixel in
// [ceil(c - r s), floor(c + r s)] (clamped to the detector) receives the weight
// lut(|c - pixel| / s) (phase contrast: times sgn(d0) in 2D, d0 in 3D).
//
// This unit is compiled with --fmad=false: the footprint and weight arithmetic rounds exactly
// like elsa's float CPU path.
//
// Footprint loop. elsa's CPU loop (VoxelComputation.h:88-113) runs its outer loop over the u
// extent and its inner loop over the v extent while stepping the pixel index along u, so for a
// non-square clamped footprint it visits a sheared block instead of the footprint rectangle.
// FootprintMode::Reference reproduces that loop (pixels it would address outside the view are
// dropped); FootprintMode::Rectangle visits the rectangle. The two agree whenever the u and v
// extents are equal.
//
// Adjoint: one thread per voxel gathers over poses and footprint pixels in the reference's order
// (deterministic, bit-identical to the CPU loop). Forward: one CTA per (brick of voxels, pose)
// splats its voxels into a shared-memory detector patch with shared atomics and adds the patch
// to the sinogram with global atomics (the reference's CUDA path uses global atomics per pixel);
// the order of the float additions is not fixed, so forward results agree with the CPU path to
// rounding, not bit for bit.
#include "luts.hpp"
#include "projector.hpp"
#include "solvers.hpp"
#include "voxel.hpp"

#include <algorithm>
#include <climits>
#include <cmath>

namespace elsa_b200
{
    namespace
    {
        constexpr int kVoxelThreads = 256;      // forward: one thread per brick voxel; adjoint default
        constexpr int kMaxAdjointThreads = 512; // largest adjoint block the autotuner may choose
        constexpr int kPatchWords = 2304; // 9 KB shared detector patch (48 x 48 pixels)
// Footprint pixels in pairs on the packed two-wide FP32 path (blob / B-spline 128^3 adjoint:
// 17.5 -> 16.6 / 16.1 ms; the forward: blob unchanged, B-spline 24.5 -> 25.0 ms, phase-contrast
// blob / B-spline 26.7 -> 25.6 / 25.8 -> 25.1 ms, so the forward pairs pixels for the
// phase-contrast (differential) weights only)
#ifndef ELSA_VOXEL_PAIRS_ADJ
#define ELSA_VOXEL_PAIRS_ADJ 1
#endif
#ifndef ELSA_VOXEL_PAIRS_FWD
#define ELSA_VOXEL_PAIRS_FWD 2 // 0: never, 1: always, 2: differential weights only
#endif

        struct VoxelParams {
            int dim;
            int weightKind; // 0 classic, 1 differential
            int mode;       // FootprintMode
            float radius;   // LUT support
            int nu, nv;     // detector pixels per pose (nv = 1 in 2D)
            float invRadius; // 1 / radius when radius is a power of two, else 0
        };

        struct Footprint {
            float c0, c1, s;
            int lo0, hi0, lo1, hi1;
        };

        // VoxelComputation.h:55-86 in float, sequential sums (no contraction in this unit).
        template <int DIM>
        __device__ __forceinline__ Footprint footprint(const float* __restrict__ pose, int ix,
                                                       int iy, int iz, const VoxelParams& vp)
        {
            const float h0 = static_cast<float>(ix) + 0.5f;
            const float h1 = static_cast<float>(iy) + 0.5f;
            const float h2 = static_cast<float>(iz) + 0.5f;
            Footprint f;
            if (DIM == 3) {
                const float* P = pose;
                const float* E = pose + 27;
                float p[3], e[3];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    float s = __ldg(P + 4 * i) * h0;
                    s = s + __ldg(P + 4 * i + 1) * h1;
                    s = s + __ldg(P + 4 * i + 2) * h2;
                    s = s + __ldg(P + 4 * i + 3) * 1.0f;
                    p[i] = s;
                    float t = __ldg(E + 4 * i) * h0;
                    t = t + __ldg(E + 4 * i + 1) * h1;
                    t = t + __ldg(E + 4 * i + 2) * h2;
                    t = t + __ldg(E + 4 * i + 3) * 1.0f;
                    e[i] = t;
                }
                f.c0 = p[0] / p[2] - 0.5f;
                f.c1 = p[1] / p[2] - 0.5f;
                float n2 = e[0] * e[0];
                n2 = n2 + e[1] * e[1];
                n2 = n2 + e[2] * e[2];
                f.s = __ldg(pose + 39) / sqrtf(n2);
            } else {
                const float* P = pose;
                const float* E = pose + 27;
                float p[2], e[2];
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    float s = __ldg(P + 3 * i) * h0;
                    s = s + __ldg(P + 3 * i + 1) * h1;
                    s = s + __ldg(P + 3 * i + 2) * 1.0f;
                    p[i] = s;
                    float t = __ldg(E + 3 * i) * h0;
                    t = t + __ldg(E + 3 * i + 1) * h1;
                    t = t + __ldg(E + 3 * i + 2) * 1.0f;
                    e[i] = t;
                }
                f.c0 = p[0] / p[1] - 0.5f;
                f.c1 = 0.0f;
                float n2 = e[0] * e[0];
                n2 = n2 + e[1] * e[1];
                f.s = __ldg(pose + 39) / sqrtf(n2);
            }
            // clamping in float first keeps the integer conversion in range for voxels that
            // project far off the detector (same result as clamping the integers)
            const float r = f.s * vp.radius;
            f.lo0 = static_cast<int>(fmaxf(ceilf(f.c0 - r), 0.0f));
            f.hi0 = static_cast<int>(fminf(floorf(f.c0 + r), static_cast<float>(vp.nu - 1)));
            if (DIM == 3) {
                f.lo1 = static_cast<int>(fmaxf(ceilf(f.c1 - r), 0.0f));
                f.hi1 = static_cast<int>(fminf(floorf(f.c1 + r), static_cast<float>(vp.nv - 1)));
            } else {
                f.lo1 = f.hi1 = 0;
            }
            return f;
        }

        // Lut::operator()(float), Luts.hpp:61-80, on a table in shared memory. invSupport: 1 /
        // support when support is a power of two (then distance * invSupport is exactly
        // distance / support), else 0. ceil(index) is floor(index) + (index > floor(index)).
        __device__ __forceinline__ float lutAt(const float* lut, float support, float invSupport,
                                               float distance)
        {
            const float q = invSupport != 0.0f ? distance * invSupport : distance / support;
            const float index = q * static_cast<float>(kVoxelLutSize - 1);
            if (index < 0.0f || index > static_cast<float>(kVoxelLutSize - 1))
                return 0.0f;
            const float af = floorf(index);
            const int a = static_cast<int>(af);
            const int b = a + (index > af ? 1 : 0);
            const float fa = lut[a], fb = lut[b];
            const float t = index - af;
            return t * fb + (1.0f - t) * fa;
        }

        // Fast (forward only): the distance as n2 * rsqrt(n2) and the lerp as one fma, within a
        // few ulp of the reference's weights; the forward's sums are reordered by atomics
        // anyway, while the adjoint keeps every float operation of the reference.
        // WK: weight kind (-1: read vp.weightKind; 0 classic, 1 differential). The fast lerp
        // always reads lut[a + 1]: the staged table carries one padding entry, and at an integer
        // index the factor (index - a) is 0, so the result equals the reference's
        // lut[a] + 0 * (lut[ceil] - lut[a]).
        template <int DIM, bool Fast = false, int WK = -1>
        __device__ __forceinline__ float voxelWeight(const float* lut, const VoxelParams& vp,
                                                     float d0, float d1)
        {
            float n2 = d0 * d0;
            if (DIM == 3)
                n2 = Fast ? __fmaf_rn(d1, d1, n2) : n2 + d1 * d1;
            float v;
            if (Fast) {
                const float dist = n2 > 0.0f ? __fmul_rn(n2, rsqrtf(n2)) : 0.0f;
                const float q = vp.invRadius != 0.0f ? dist * vp.invRadius : dist / vp.radius;
                const float index = q * static_cast<float>(kVoxelLutSize - 1);
                if (!(index <= static_cast<float>(kVoxelLutSize - 1))) { // index >= 0 here
                    v = 0.0f;
                } else {
                    const float af = floorf(index);
                    const int a = static_cast<int>(af);
                    const float fa = lut[a];
                    v = __fmaf_rn(index - af, lut[a + 1] - fa, fa);
                }
            } else {
                v = lutAt(lut, vp.radius, vp.invRadius, sqrtf(n2));
            }
            const int wk = WK >= 0 ? WK : vp.weightKind;
            if (wk == 0)
                return v;
            if (DIM == 2)
                return v * static_cast<float>((0.0f < d0) - (d0 < 0.0f));
            return v * d0;
        }

        // voxelWeight<DIM, true, WK> of two pixels of one footprint row (d0 pair, shared d1) on
        // the packed two-wide FP32 instructions: the same operations and roundings per pixel.
        template <int DIM, int WK>
        __device__ __forceinline__ float2 voxelWeight2(const float* lut, const VoxelParams& vp,
                                                       float2 d0, float d1)
        {
            float2 n2 = mul2(d0, d0);
            if (DIM == 3)
                n2 = fma2(make_float2(d1, d1), make_float2(d1, d1), n2);
            float2 dist = mul2(n2, make_float2(rsqrtf(n2.x), rsqrtf(n2.y)));
            dist.x = n2.x > 0.0f ? dist.x : 0.0f;
            dist.y = n2.y > 0.0f ? dist.y : 0.0f;
            const float2 q = vp.invRadius != 0.0f
                                 ? mul2(dist, make_float2(vp.invRadius, vp.invRadius))
                                 : make_float2(dist.x / vp.radius, dist.y / vp.radius);
            constexpr float kTop = static_cast<float>(kVoxelLutSize - 1);
            const float2 index = mul2(q, make_float2(kTop, kTop));
            // index >= 0 and far below 2^22 (a footprint reaches a few supports at most)
            int a0, a1;
            const float2 af = floorSmall2(index, a0, a1);
            const bool in0 = index.x <= kTop, in1 = index.y <= kTop;
            const float2 fa = make_float2(in0 ? lut[a0] : 0.0f, in1 ? lut[a1] : 0.0f);
            const float2 fb = make_float2(in0 ? lut[a0 + 1] : 0.0f, in1 ? lut[a1 + 1] : 0.0f);
            float2 v = fma2(sub2(index, af), sub2(fb, fa), fa);
            v.x = in0 ? v.x : 0.0f;
            v.y = in1 ? v.y : 0.0f;
            const int wk = WK >= 0 ? WK : vp.weightKind;
            if (wk == 0)
                return v;
            if (DIM == 2)
                return make_float2(v.x * static_cast<float>((0.0f < d0.x) - (d0.x < 0.0f)),
                                   v.y * static_cast<float>((0.0f < d0.y) - (d0.y < 0.0f)));
            return mul2(v, d0);
        }

        // Visits the footprint pixels of one voxel in the reference's order; fn(linear pixel
        // index within the pose, u, v, d0, d1) with (u, v) the pixel's unwrapped detector
        // coordinates (u may leave [0, nu) where the reference's linear index wraps into the
        // next row; visitBox rejects such footprints for the shared patch).
        // Fast (forward only): divisions by the scaling s replaced by a multiplication with 1 / s.
        template <int DIM, bool Fast = false, class Fn>
        __device__ __forceinline__ void visitFootprint(const Footprint& f, const VoxelParams& vp,
                                                       Fn fn)
        {
            const float invS = Fast ? 1.0f / f.s : 0.0f;
            auto scaled = [&](float d) { return Fast ? __fmul_rn(d, invS) : d / f.s; };
            if (DIM == 2) {
                for (int u = f.lo0; u <= f.hi0; ++u)
                    fn(u, u, 0, scaled(f.c0 - static_cast<float>(u)), 0.0f);
                return;
            }
            const int ext0 = f.hi0 - f.lo0 + 1, ext1 = f.hi1 - f.lo1 + 1;
            if (ext0 <= 0 || ext1 <= 0)
                return;
            const bool ref = vp.mode == static_cast<int>(FootprintMode::Reference);
            const int rows = ref ? ext0 : ext1;
            const int cols = ref ? ext1 : ext0;
            const int64_t npix = static_cast<int64_t>(vp.nu) * vp.nv;
            int64_t lin = static_cast<int64_t>(f.lo1) * vp.nu + f.lo0;
            float cur0 = static_cast<float>(f.lo0), cur1 = static_cast<float>(f.lo1);
            int u = f.lo0, v = f.lo1;
            for (int r = 0; r < rows; ++r) {
                const float d1 = scaled(f.c1 - cur1);
                for (int c = 0; c < cols; ++c) {
                    if (lin >= 0 && lin < npix)
                        fn(lin, u, v, scaled(f.c0 - cur0), d1);
                    lin += 1;
                    u += 1;
                    cur0 = cur0 + 1.0f;
                }
                lin += vp.nu - ext0;
                u -= ext0;
                v += 1;
                cur0 = cur0 - static_cast<float>(ext0);
                cur1 = cur1 + 1.0f;
            }
        }

        // visitFootprintInside with the pixels of a row taken in pairs: fn2(u, v, (d0, d0'), d1)
        // for pixels u and u + 1, fn1 for the last pixel of an odd row; the same pixels, order
        // and offsets.
        template <int DIM, class Fn2, class Fn1>
        __device__ __forceinline__ void visitFootprintInsidePairs(const Footprint& f,
                                                                  const VoxelParams& vp, Fn2 fn2,
                                                                  Fn1 fn1)
        {
            const float invS = 1.0f / f.s;
            const float2 inv2 = make_float2(invS, invS);
            const float2 c2 = make_float2(f.c0, f.c0);
            if (DIM == 2) {
                int u = f.lo0;
                for (; u + 1 <= f.hi0; u += 2)
                    fn2(u, 0, mul2(sub2(c2, make_float2(static_cast<float>(u),
                                                        static_cast<float>(u + 1))),
                                   inv2),
                        0.0f);
                if (u <= f.hi0)
                    fn1(u, 0, __fmul_rn(f.c0 - static_cast<float>(u), invS), 0.0f);
                return;
            }
            const int ext0 = f.hi0 - f.lo0 + 1, ext1 = f.hi1 - f.lo1 + 1;
            if (ext0 <= 0 || ext1 <= 0)
                return;
            const bool ref = vp.mode == static_cast<int>(FootprintMode::Reference);
            const int rows = min(ref ? ext0 : ext1, vp.nv - f.lo1);
            const int cols = ref ? ext1 : ext0;
            float cur0 = static_cast<float>(f.lo0), cur1 = static_cast<float>(f.lo1);
            int u = f.lo0, v = f.lo1;
            for (int r = 0; r < rows; ++r) {
                const float d1 = __fmul_rn(f.c1 - cur1, invS);
                int c = 0;
                for (; c + 1 < cols; c += 2) {
                    fn2(u, v, mul2(sub2(c2, make_float2(cur0, cur0 + 1.0f)), inv2), d1);
                    u += 2;
                    cur0 = cur0 + 1.0f;
                    cur0 = cur0 + 1.0f;
                }
                if (c < cols) {
                    fn1(u, v, __fmul_rn(f.c0 - cur0, invS), d1);
                    u += 1;
                    cur0 = cur0 + 1.0f;
                }
                u -= ext0;
                v += 1;
                cur0 = cur0 - static_cast<float>(ext0);
                cur1 = cur1 + 1.0f;
            }
        }

        // visitFootprint for a footprint whose visited pixels lie inside the detector (visitBox
        // true): the same pixels in the same order with the same offsets (Fast), without the
        // linear index. In the reference loop with a sheared block, rows past the detector's
        // last row are where the linear index would leave the view: they are not visited.
        template <int DIM, class Fn>
        __device__ __forceinline__ void visitFootprintInside(const Footprint& f,
                                                             const VoxelParams& vp, Fn fn)
        {
            const float invS = 1.0f / f.s;
            if (DIM == 2) {
                for (int u = f.lo0; u <= f.hi0; ++u)
                    fn(u, 0, __fmul_rn(f.c0 - static_cast<float>(u), invS), 0.0f);
                return;
            }
            const int ext0 = f.hi0 - f.lo0 + 1, ext1 = f.hi1 - f.lo1 + 1;
            if (ext0 <= 0 || ext1 <= 0)
                return;
            const bool ref = vp.mode == static_cast<int>(FootprintMode::Reference);
            const int rows = min(ref ? ext0 : ext1, vp.nv - f.lo1);
            const int cols = ref ? ext1 : ext0;
            float cur0 = static_cast<float>(f.lo0), cur1 = static_cast<float>(f.lo1);
            int u = f.lo0, v = f.lo1;
            for (int r = 0; r < rows; ++r) {
                const float d1 = __fmul_rn(f.c1 - cur1, invS);
                for (int c = 0; c < cols; ++c) {
                    fn(u, v, __fmul_rn(f.c0 - cur0, invS), d1);
                    u += 1;
                    cur0 = cur0 + 1.0f;
                }
                u -= ext0;
                v += 1;
                cur0 = cur0 - static_cast<float>(ext0);
                cur1 = cur1 + 1.0f;
            }
        }

        // Bounding box (u0, u1, v0, v1) of the pixels a footprint visits; false when the visit
        // wraps across detector rows (reference loop with a sheared block), which the patch
        // cannot hold.
        template <int DIM>
        __device__ __forceinline__ bool visitBox(const Footprint& f, const VoxelParams& vp,
                                                 int& u0, int& u1, int& v0, int& v1)
        {
            const int ext0 = f.hi0 - f.lo0 + 1, ext1 = f.hi1 - f.lo1 + 1;
            if (DIM == 2 || vp.mode != static_cast<int>(FootprintMode::Reference) ||
                ext0 == ext1) {
                u0 = f.lo0, u1 = f.hi0, v0 = f.lo1, v1 = f.hi1;
                return true;
            }
            // rows r = 0 .. ext0-1 start at u = lo0 + r * (ext1 - ext0) and span ext1 pixels
            const int shift = (ext0 - 1) * (ext1 - ext0);
            u0 = f.lo0 + min(0, shift);
            u1 = f.lo0 + max(0, shift) + ext1 - 1;
            v0 = f.lo1;
            v1 = min(f.lo1 + ext0 - 1, vp.nv - 1);
            return u0 >= 0 && u1 < vp.nu;
        }

        // visitBox's test alone: the footprint's visited pixels stay inside the detector's rows.
        template <int DIM>
        __device__ __forceinline__ bool footprintInside(const Footprint& f, const VoxelParams& vp)
        {
            const int ext0 = f.hi0 - f.lo0 + 1, ext1 = f.hi1 - f.lo1 + 1;
            if (DIM == 2 || vp.mode != static_cast<int>(FootprintMode::Reference) ||
                ext0 == ext1)
                return true;
            const int shift = (ext0 - 1) * (ext1 - ext0);
            return f.lo0 + min(0, shift) >= 0 && f.lo0 + max(0, shift) + ext1 - 1 < vp.nu;
        }

        // Adjoint: x[v] = sum over poses and footprint pixels of w * y[pixel], in the reference's
        // order (VoxelComputation.h:152-183). One thread per voxel, x fastest within a block.
        // Fast: the forward's weights (the default); otherwise the reference's float
        // operations, bit-identical to its CPU loop.
        template <int DIM, bool Fast, int WK>
        __global__ void __launch_bounds__(kMaxAdjointThreads, 2)
            voxelAdjointKernel(const float* __restrict__ poses, int np,
                               const float* __restrict__ lutIn, VoxelParams vp, VolumeShape vol,
                               const float* __restrict__ y, float* __restrict__ x)
        {
            __shared__ float lut[kVoxelLutSize + 1]; // + 1 padding entry for the fast lerp
            for (int i = threadIdx.x; i <= kVoxelLutSize; i += blockDim.x)
                lut[i] = lutIn[min(i, kVoxelLutSize - 1)];
            __syncthreads();
            const int64_t nvox = static_cast<int64_t>(vol.n[0]) * vol.n[1] * vol.n[2];
            const int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            if (v >= nvox)
                return;
            const int ix = static_cast<int>(v % vol.n[0]);
            const int iy = static_cast<int>((v / vol.n[0]) % vol.n[1]);
            const int iz = DIM == 3 ? static_cast<int>(v / (static_cast<int64_t>(vol.n[0]) *
                                                            vol.n[1]))
                                    : 0;
            const int64_t npix = static_cast<int64_t>(vp.nu) * vp.nv;
            float acc = 0.0f;
            for (int p = 0; p < np; ++p) {
                const Footprint f = footprint<DIM>(poses + static_cast<int64_t>(p) * 40, ix, iy,
                                                   iz, vp);
                const float* view = y + p * npix;
                if (Fast && footprintInside<DIM>(f, vp)) {
                    // the same pixels in the same order, without the linear index
#if ELSA_VOXEL_PAIRS_ADJ
                    visitFootprintInsidePairs<DIM>(
                        f, vp,
                        [&](int pu_, int pv_, float2 d0, float d1) {
                            const float2 w = voxelWeight2<DIM, WK>(lut, vp, d0, d1);
                            const float* yp = view + pv_ * vp.nu + pu_;
                            acc = acc + w.x * __ldg(yp);
                            acc = acc + w.y * __ldg(yp + 1);
                        },
                        [&](int pu_, int pv_, float d0, float d1) {
                            const float w = voxelWeight<DIM, true, WK>(lut, vp, d0, d1);
                            acc = acc + w * __ldg(view + pv_ * vp.nu + pu_);
                        });
#else
                    visitFootprintInside<DIM>(f, vp, [&](int pu_, int pv_, float d0, float d1) {
                        const float w = voxelWeight<DIM, true, WK>(lut, vp, d0, d1);
                        acc = acc + w * __ldg(view + pv_ * vp.nu + pu_);
                    });
#endif
                    continue;
                }
                visitFootprint<DIM, Fast>(f, vp, [&](int64_t pix, int pu_, int pv_, float d0,
                                                     float d1) {
                    const float w = voxelWeight<DIM, Fast, WK>(lut, vp, d0, d1);
                    acc = acc + w * __ldg(view + pix);
                });
            }
            x[v] = acc;
        }

        // Forward: one CTA per (brick of voxels, pose). Voxels splat into a shared patch of the
        // detector (shared atomics); the patch is added to the sinogram with global atomics.
        // Voxels whose footprint leaves the patch add to the sinogram directly.
        template <int DIM, int BX, int BY, int BZ, int WK>
        __global__ void __launch_bounds__(kVoxelThreads)
            voxelForwardKernel(const float* __restrict__ poses, const float* __restrict__ lutIn,
                               VoxelParams vp, VolumeShape vol, int3 nBricks,
                               const float* __restrict__ x, float* __restrict__ y)
        {
            static_assert(BX * BY * BZ == kVoxelThreads, "one thread per brick voxel");
            __shared__ float lut[kVoxelLutSize + 1]; // + 1 padding entry for the fast lerp
            __shared__ float patch[kPatchWords];
            __shared__ int box[4]; // u0, -u1, v0, -v1 (atomicMin on all four)
            const int p = blockIdx.y;
            const int b = blockIdx.x;
            const int bx = b % nBricks.x, by = (b / nBricks.x) % nBricks.y,
                      bz = b / (nBricks.x * nBricks.y);
            const int tx = threadIdx.x % BX, ty = (threadIdx.x / BX) % BY,
                      tz = threadIdx.x / (BX * BY);
            const int ix = bx * BX + tx, iy = by * BY + ty, iz = bz * BZ + tz;
            for (int i = threadIdx.x; i <= kVoxelLutSize; i += blockDim.x)
                lut[i] = lutIn[min(i, kVoxelLutSize - 1)];
            if (threadIdx.x < 4)
                box[threadIdx.x] = INT_MAX;
            __syncthreads();

            bool active = ix < vol.n[0] && iy < vol.n[1] && (DIM == 2 || iz < vol.n[2]);
            float xv = 0.0f;
            Footprint f{};
            int u0 = 0, u1 = -1, v0 = 0, v1 = -1;
            bool boxed = false;
            if (active) {
                xv = __ldg(x + ix + static_cast<int64_t>(vol.n[0]) *
                                        (iy + static_cast<int64_t>(vol.n[1]) * iz));
                active = xv != 0.0f;
            }
            if (active) {
                f = footprint<DIM>(poses + static_cast<int64_t>(p) * 40, ix, iy, iz, vp);
                active = f.lo0 <= f.hi0 && f.lo1 <= f.hi1;
            }
            if (active) {
                boxed = visitBox<DIM>(f, vp, u0, u1, v0, v1) && u0 <= u1 && v0 <= v1;
                if (boxed) {
                    atomicMin(&box[0], u0);
                    atomicMin(&box[1], -u1);
                    atomicMin(&box[2], v0);
                    atomicMin(&box[3], -v1);
                }
            }
            __syncthreads();
            const int bu0 = box[0], bu1 = -box[1], bv0 = box[2], bv1 = -box[3];
            const int pw = bu1 - bu0 + 1, ph = bv1 - bv0 + 1;
            const bool usePatch = bu0 != INT_MAX && pw > 0 && ph > 0 &&
                                  static_cast<int64_t>(pw) * ph <= kPatchWords;
            float* view = y + static_cast<int64_t>(p) * vp.nu * vp.nv;
            if (usePatch) {
                for (int i = threadIdx.x; i < pw * ph; i += blockDim.x)
                    patch[i] = 0.0f;
            }
            __syncthreads();
            if (active) {
                if (usePatch && boxed) {
                    // a boxed footprint stays inside the detector and its rows: no linear
                    // index to test
                    constexpr bool kFwdPairs =
                        ELSA_VOXEL_PAIRS_FWD == 1 || (ELSA_VOXEL_PAIRS_FWD == 2 && WK == 1);
                    if constexpr (kFwdPairs) {
                        visitFootprintInsidePairs<DIM>(
                            f, vp,
                            [&](int pu_, int pv_, float2 d0, float d1) {
                                const float2 c = mul2(make_float2(xv, xv),
                                                      voxelWeight2<DIM, WK>(lut, vp, d0, d1));
                                float* pp = &patch[(pv_ - bv0) * pw + (pu_ - bu0)];
                                atomicAdd(pp, c.x);
                                atomicAdd(pp + 1, c.y);
                            },
                            [&](int pu_, int pv_, float d0, float d1) {
                                const float w = voxelWeight<DIM, true, WK>(lut, vp, d0, d1);
                                atomicAdd(&patch[(pv_ - bv0) * pw + (pu_ - bu0)], xv * w);
                            });
                    } else {
                        visitFootprintInside<DIM>(f, vp, [&](int pu_, int pv_, float d0, float d1) {
                            const float w = voxelWeight<DIM, true, WK>(lut, vp, d0, d1);
                            atomicAdd(&patch[(pv_ - bv0) * pw + (pu_ - bu0)], xv * w);
                        });
                    }
                } else {
                    visitFootprint<DIM, true>(f, vp, [&](int64_t pix, int pu_, int pv_, float d0,
                                                         float d1) {
                        const float w = voxelWeight<DIM, true, WK>(lut, vp, d0, d1);
                        atomicAdd(view + pix, xv * w);
                    });
                }
            }
            if (usePatch) {
                __syncthreads();
                for (int i = threadIdx.x; i < pw * ph; i += blockDim.x) {
                    const float v = patch[i];
                    if (v != 0.0f)
                        atomicAdd(view + static_cast<int64_t>(bv0 + i / pw) * vp.nu + bu0 + i % pw,
                                  v);
                }
            }
        }

        template <int DIM>
        class VoxelProjector final : public Projector
        {
        public:
            VoxelProjector(int kind, const VolumeShape& vol, const DetectorShape& det,
                           const std::vector<PoseRecord>& poses, const VoxelLut& lut,
                           int weightKind, FootprintMode mode)
                : Projector(kind, vol, det, poses), lut_(sizeof(float) * kVoxelLutSize)
            {
                if (static_cast<int>(lut.values.size()) != kVoxelLutSize)
                    throw Error(ELSA_ERROR_LOGIC, "voxel projector: lookup table size");
                ELSA_CUDA(cudaMemcpy(lut_.as<float>(), lut.values.data(),
                                     sizeof(float) * kVoxelLutSize, cudaMemcpyHostToDevice));
                vp_.dim = DIM;
                vp_.weightKind = weightKind;
                vp_.mode = static_cast<int>(mode);
                vp_.radius = lut.support;
                vp_.nu = det.nu;
                vp_.nv = det.nv;
                {
                    int e = 0;
                    const float m = std::frexp(lut.support, &e);
                    vp_.invRadius = (m == 0.5f) ? std::ldexp(1.0f, 1 - e) : 0.0f;
                }
                nBricks_ = make_int3((vol.n[0] + kBX - 1) / kBX, (vol.n[1] + kBY - 1) / kBY,
                                     (vol.n[2] + kBZ - 1) / kBZ);
                if (det.np > 65535)
                    throw Error(ELSA_ERROR_NOT_SUPPORTED, "voxel projector: at most 65535 poses");
            }

            void forward(const float* x, float* y, cudaStream_t s) override
            {
                ELSA_CUDA(cudaMemsetAsync(y, 0, sizeof(float) * rangeSize_, s));
                const dim3 grid(static_cast<unsigned>(nBricks_.x * nBricks_.y * nBricks_.z),
                                static_cast<unsigned>(det_.np));
                if (vp_.weightKind == 0)
                    voxelForwardKernel<DIM, kBX, kBY, kBZ, 0><<<grid, kVoxelThreads, 0, s>>>(
                        dPoses_, lut_.as<float>(), vp_, vol_, nBricks_, x, y);
                else
                    voxelForwardKernel<DIM, kBX, kBY, kBZ, 1><<<grid, kVoxelThreads, 0, s>>>(
                        dPoses_, lut_.as<float>(), vp_, vol_, nBricks_, x, y);
                ELSA_LAUNCH_CHECK("voxelForwardKernel");
            }

            void adjoint(const float* y, float* x, cudaStream_t s) override
            {
                const unsigned blocks =
                    static_cast<unsigned>((domainSize_ + adjointThreads_ - 1) / adjointThreads_);
#define ELSA_VOXEL_ADJOINT(FAST_, WK_)                                                      \
    voxelAdjointKernel<DIM, FAST_, WK_><<<blocks, adjointThreads_, 0, s>>>(                    \
        dPoses_, det_.np, lut_.as<float>(), vp_, vol_, y, x)
                if (exactWeights_) {
                    if (vp_.weightKind == 0)
                        ELSA_VOXEL_ADJOINT(false, 0);
                    else
                        ELSA_VOXEL_ADJOINT(false, 1);
                } else {
                    if (vp_.weightKind == 0)
                        ELSA_VOXEL_ADJOINT(true, 0);
                    else
                        ELSA_VOXEL_ADJOINT(true, 1);
                }
#undef ELSA_VOXEL_ADJOINT
                ELSA_LAUNCH_CHECK("voxelAdjointKernel");
            }

            int64_t info(int key) const override
            {
                switch (key) {
                case 1:
                    return static_cast<int64_t>(nBricks_.x) * nBricks_.y * nBricks_.z;
                case 5:
                    return vp_.mode;
                case 6: // kernel launches per forward call (after the output memset)
                    return 1;
                case 7: // kernel launches per adjoint call
                    return 1;
                default:
                    return -1;
                }
            }

            std::vector<int> knobCandidates(int knob) const override
            {
                if (knob == kKnobAdjointThreads)
                    return {64, 128, 256, 512};
                if (knob == kKnobExactWeights)
                    return {0, 1};
                return {};
            }

            int knob(int knob) const override
            {
                if (knob == kKnobAdjointThreads)
                    return adjointThreads_;
                if (knob == kKnobExactWeights)
                    return exactWeights_;
                return -1;
            }

            void setKnob(int knob, int value) override
            {
                const std::vector<int> c = knobCandidates(knob);
                if (std::find(c.begin(), c.end(), value) == c.end())
                    throw Error(ELSA_ERROR_INVALID_ARGUMENT,
                                "voxel projector: value " + std::to_string(value) +
                                    " is not a candidate of knob " + std::to_string(knob));
                if (knob == kKnobExactWeights)
                    exactWeights_ = value;
                else
                    adjointThreads_ = value;
            }

        private:
            int adjointThreads_ = kVoxelThreads; // voxels per block of the gather adjoint
            // 0: the adjoint uses the forward's weights (128^3 blob: 21.7 ms); 1: the reference's
            // float operations, bit-identical to elsa's CPU loop (24.1 ms)
            int exactWeights_ = 0;
            // forward bricks: 8 x 8 x 4 voxels in 3D, 16 x 16 in 2D (one thread per voxel)
            static constexpr int kBX = DIM == 3 ? 8 : 16;
            static constexpr int kBY = DIM == 3 ? 8 : 16;
            static constexpr int kBZ = DIM == 3 ? 4 : 1;
            DeviceBuffer lut_;
            VoxelParams vp_{};
            int3 nBricks_{};
        };
    } // namespace

    std::unique_ptr<Projector> makeVoxelProjector(int kind, const VolumeShape& vol,
                                                  const DetectorShape& det,
                                                  const std::vector<PoseRecord>& poses,
                                                  const VoxelLut& lut, bool phaseContrast,
                                                  FootprintMode mode)
    {
        const int wk = phaseContrast ? 1 : 0;
        if (vol.dim == 3)
            return std::make_unique<VoxelProjector<3>>(kind, vol, det, poses, lut, wk, mode);
        return std::make_unique<VoxelProjector<2>>(kind, vol, det, poses, lut, wk, mode);
    }
} // namespace elsa_b200
