// Joseph's method (driving-direction ray stepping with bilinear interpolation) for sm_100a.
//
// Reference semantics: projectors/JosephsMethod.cpp:37-198 and
// projectors/DrivingDirectionTraversal.cpp:6-106 (elsa's CPU path, the parity target). Per ray r
// with n samples and step length L:
//   forward  y[r] = L * sum_j bilinear(x, plane k0 + j*dir, (pa_j, pb_j))
//   adjoint  x[v] = sum_r sum_j y[r] * L * w_v(r, j)
// Taps outside the volume contribute zero (the reference masks them, :60-97).
//
// Sample positions. The reference advances pos += step in float after every sample
// (DrivingDirectionTraversal.cpp:265). With a constant step every addition rounds the same way
// inside a binade, so the accumulated position drifts linearly from pos0 + j*step (about 1e-3
// voxel after 256 steps at 256^3) -- far more than the 1e-5 parity budget allows. Both kernels
// therefore reproduce the accumulation bit for bit: the forward accumulates along each ray, and
// the adjoint starts every ray segment from a checkpoint (the exact accumulated position at the
// ray's first sample in each slab of kCheckpointDepth planes, computed once per geometry) and
// accumulates from there.
//
// Forward: one thread per ray, samples gathered through the read-only cache (the volume is
// L2-resident: 67 MB at 256^3 against a 126 MB L2).
//
// Adjoint (default): atomic-free and deterministic. Each CTA owns one brick of the volume in shared memory
// for all views. For every view it visits the rays of the brick's detector window one
// conflict-free class at a time: rays whose pixel indices are congruent modulo m stay more than
// two voxels apart on every plane (m is validated per geometry at construction), so their
// bilinear taps never overlap and the threads update shared memory without atomics. Each thread
// walks one ray through the brick; classes are separated by barriers. Every voxel receives its
// contributions in a fixed order, with exactly the positions and weights of the forward kernel.
// The launch knob kKnobAdjointScatter = 1 selects a thread-per-ray scatter instead (the forward's
// sample loop with atomic adds to the four taps): faster in 2D, slower in 3D, where four global
// atomics per sample exceed what the L2 sustains. A shared-memory variant (several warps per
// brick adding with shared atomics, no ray classes) measured 65.5 ms against 54.8 ms at
// 256^3 / 360 views and was dropped.
#include "joseph_tma.cuh"
#include "projector.hpp"
#include "raysetup.cuh"
#include "solvers.hpp"

#include <algorithm>
#include <atomic>
#include <mutex>
#include <cmath>
#include <cstring>

#ifndef ELSA_ADJ_MIN_BLOCKS
#define ELSA_ADJ_MIN_BLOCKS 1 // resident one-warp blocks per SM asked of the register allocator
#endif
#ifndef ELSA_ADJ_BATCH
#define ELSA_ADJ_BATCH 3 // class rays per lane fetched together by the adjoints (3D axis bricks at 256^3 / 360 views: 1: 37.5 ms, 2: 33.5, 3: 33.0)
#endif
#ifndef ELSA_AXIS_TD
#define ELSA_AXIS_TD 16 // depth along the driving axis of the 3D adjoint's axis bricks
#endif
#ifndef ELSA_AXIS_TW
#define ELSA_AXIS_TW 32 // edge along the non-driving axis over which a detector row's rays spread
#endif
#ifndef ELSA_AXIS_TV
#define ELSA_AXIS_TV 8 // edge along the other non-driving axis
#endif
#ifndef ELSA_SPLAT_UNROLL
#define ELSA_SPLAT_UNROLL 2 // unroll factor of the adjoint's per-sample loop (1: 72.8 ms, 2: 63.4 ms, 4: 68.9 ms at 256^3)
#endif

namespace elsa_b200
{
    namespace
    {
        constexpr int kForwardThreads = 256;    // default rays per block of the gather forward
        constexpr int kMaxForwardThreads = 512; // largest block the autotuner may choose
        constexpr int kSplatUnroll = ELSA_SPLAT_UNROLL;
        constexpr int kMinClass = 2;
        constexpr int kMaxClass = 8;
        // Joseph brick windows: the brick grown by half a voxel (the reach of a bilinear tap)
        // plus slack for the accumulated-position drift (at most n steps of half an ulp of a
        // coordinate below n: n^2 2^-24 voxel, 0.004 at n = 256), doubled, and 0.05 voxel for the
        // rounding of the float rays; 0.05 pixel of margin for the projection of the corners.
        inline float windowGrow(const VolumeShape& vol)
        {
            const float n = static_cast<float>(std::max(vol.n[0], std::max(vol.n[1], vol.n[2])));
            return 0.55f + 2.0f * n * n * 5.9604645e-8f;
        }
        constexpr float kWindowPixelMargin = 0.05f;

        struct Weights {
            int ia, ib;
            float wa, cwa, wb, cwb;
        };

        // Bilinear weights at non-driving position (pa, pb), as JosephsMethod.cpp:37-52:
        // floor of pos - 0.5, complement weight (pos - floor) - 0.5, weight 1 - complement.
        __device__ __forceinline__ void tapWeights(float pa, float pb, Weights& w)
        {
            const float fa = floorf(__fsub_rn(pa, 0.5f));
            const float fb = floorf(__fsub_rn(pb, 0.5f));
            w.cwa = __fsub_rn(__fsub_rn(pa, fa), 0.5f);
            w.cwb = __fsub_rn(__fsub_rn(pb, fb), 0.5f);
            w.wa = __fsub_rn(1.0f, w.cwa);
            w.wb = __fsub_rn(1.0f, w.cwb);
            w.ia = static_cast<int>(fa);
            w.ib = static_cast<int>(fb);
        }

        __device__ __forceinline__ int floorDiv(int a, int b)
        {
            return a >= 0 ? a / b : -((-a + b - 1) / b);
        }

        template <int DIM>
        __global__ void __launch_bounds__(kMaxForwardThreads)
            josephForwardKernel(const JosephRay* __restrict__ rays, int64_t nrays,
                                const float* __restrict__ x, VolumeShape vol,
                                float* __restrict__ y)
        {
            const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            if (r >= nrays)
                return;
            const JosephRay R = rays[r];
            if (R.n == 0) {
                y[r] = 0.0f;
                return;
            }
            const int g = R.meta & 3;
            const int dir = (R.meta & 4) ? -1 : 1;
            int a, b;
            nonDrivingAxes(g, a, b);
            const int64_t plane = static_cast<int64_t>(vol.n[0]) * vol.n[1];
            const int64_t sg = g == 0 ? 1 : (g == 1 ? vol.n[0] : plane);
            const int64_t sa = a == 0 ? 1 : (a == 1 ? vol.n[0] : plane);
            const int ng = g == 0 ? vol.n[0] : (g == 1 ? vol.n[1] : vol.n[2]);
            const int na = a == 0 ? vol.n[0] : (a == 1 ? vol.n[1] : vol.n[2]);
            const int64_t sb = DIM == 3 ? (b == 1 ? vol.n[0] : plane) : 0;
            const int nb = DIM == 3 ? (b == 1 ? vol.n[1] : vol.n[2]) : 1;
            float acc = 0.0f;
            float pa = R.pa, pb = R.pb;
            int k = R.k0;
            for (int j = 0; j < R.n; ++j, k += dir, pa = __fadd_rn(pa, R.sa),
                     pb = __fadd_rn(pb, R.sb)) {
                if (static_cast<unsigned>(k) >= static_cast<unsigned>(ng))
                    continue;
                Weights w;
                tapWeights(pa, pb, w);
                const float* base = x + k * sg;
                const bool a0 = static_cast<unsigned>(w.ia) < static_cast<unsigned>(na);
                const bool a1 = static_cast<unsigned>(w.ia + 1) < static_cast<unsigned>(na);
                if (DIM == 2) {
                    const float v0 = a0 ? __ldg(base + w.ia * sa) : 0.0f;
                    const float v1 = a1 ? __ldg(base + (w.ia + 1) * sa) : 0.0f;
                    acc += w.wa * v0 + w.cwa * v1;
                } else {
                    const bool b0 = static_cast<unsigned>(w.ib) < static_cast<unsigned>(nb);
                    const bool b1 = static_cast<unsigned>(w.ib + 1) < static_cast<unsigned>(nb);
                    const float* p0 = base + w.ia * sa + w.ib * sb;
                    const float v00 = (a0 && b0) ? __ldg(p0) : 0.0f;
                    const float v10 = (a1 && b0) ? __ldg(p0 + sa) : 0.0f;
                    const float v01 = (a0 && b1) ? __ldg(p0 + sb) : 0.0f;
                    const float v11 = (a1 && b1) ? __ldg(p0 + sa + sb) : 0.0f;
                    acc += w.wb * (w.wa * v00 + w.cwa * v10) + w.cwb * (w.wa * v01 + w.cwa * v11);
                }
            }
            y[r] = R.len * acc;
        }

        // Adjoint by atomic scatter: the forward's sample loop, one thread per ray, adding
        // y[r] * len * (tap weight) to the in-volume taps of every sample (x zeroed beforehand);
        // the tap values are those of the brick-owner adjoint, the order of the additions varies.
        template <int DIM>
        __global__ void __launch_bounds__(kMaxForwardThreads)
            josephScatterKernel(const JosephRay* __restrict__ rays, int64_t nrays,
                                const float* __restrict__ y, VolumeShape vol,
                                float* __restrict__ x)
        {
            const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            if (r >= nrays)
                return;
            const JosephRay R = rays[r];
            if (R.n == 0)
                return;
            const float yl = __ldg(y + r) * R.len;
            if (yl == 0.0f)
                return;
            const int g = R.meta & 3;
            const int dir = (R.meta & 4) ? -1 : 1;
            int a, b;
            nonDrivingAxes(g, a, b);
            const int64_t plane = static_cast<int64_t>(vol.n[0]) * vol.n[1];
            const int64_t sg = g == 0 ? 1 : (g == 1 ? vol.n[0] : plane);
            const int64_t sa = a == 0 ? 1 : (a == 1 ? vol.n[0] : plane);
            const int ng = g == 0 ? vol.n[0] : (g == 1 ? vol.n[1] : vol.n[2]);
            const int na = a == 0 ? vol.n[0] : (a == 1 ? vol.n[1] : vol.n[2]);
            const int64_t sb = DIM == 3 ? (b == 1 ? vol.n[0] : plane) : 0;
            const int nb = DIM == 3 ? (b == 1 ? vol.n[1] : vol.n[2]) : 1;
            float pa = R.pa, pb = R.pb;
            int k = R.k0;
            for (int j = 0; j < R.n; ++j, k += dir, pa = __fadd_rn(pa, R.sa),
                     pb = __fadd_rn(pb, R.sb)) {
                if (static_cast<unsigned>(k) >= static_cast<unsigned>(ng))
                    continue;
                Weights w;
                tapWeights(pa, pb, w);
                float* base = x + k * sg;
                const bool a0 = static_cast<unsigned>(w.ia) < static_cast<unsigned>(na);
                const bool a1 = static_cast<unsigned>(w.ia + 1) < static_cast<unsigned>(na);
                if (DIM == 2) {
                    if (a0)
                        atomicAdd(base + w.ia * sa, yl * w.wa);
                    if (a1)
                        atomicAdd(base + (w.ia + 1) * sa, yl * w.cwa);
                } else {
                    const bool b0 = static_cast<unsigned>(w.ib) < static_cast<unsigned>(nb);
                    const bool b1 = static_cast<unsigned>(w.ib + 1) < static_cast<unsigned>(nb);
                    float* p0 = base + w.ia * sa + w.ib * sb;
                    if (a0 && b0)
                        atomicAdd(p0, yl * (w.wa * w.wb));
                    if (a1 && b0)
                        atomicAdd(p0 + sa, yl * (w.cwa * w.wb));
                    if (a0 && b1)
                        atomicAdd(p0 + sb, yl * (w.wa * w.cwb));
                    if (a1 && b1)
                        atomicAdd(p0 + sa + sb, yl * (w.cwa * w.cwb));
                }
            }
        }

        // elsa's default CUDA adjoint (JosephsMethodCUDA with fast = true,
        // TraverseJosephsCUDA.cu:218-287): a voxel-driven backprojection, not the transpose of the
        // forward. For voxel centre c and view p: pixel = B_p (c - o_p) with B_p the leading
        // DIM x DIM block of the projection matrix and o_p = -Binv_p p4_p, divided by its last
        // coordinate; the sinogram is read through a layered texture (linear filtering, border
        // addressing) and the views are summed in order. The float operations are the reference
        // kernel's: its x coordinates come from 32 lanes per (y, z) row, lane t taking voxels
        // t + 32 s and advancing the first difference by adding 32 once per step s (voxels past
        // the last multiple of 32 computed directly), and its matrix-vector product
        // ((b0 r0 + b1 r1) + b2 r2, Matrix.cuh:12-32) is contracted as fma(b2, r2, fma(b0, r0,
        // b1 r1)). The layout is the reference's too, a row per 32 lanes, but with kRows rows per
        // block and the sums of kChunk steps in registers instead of shared memory.
        template <int DIM>
        __device__ __forceinline__ float fastSample(cudaTextureObject_t sino, const float* T,
                                                    float r0, float r1, float r2, int p)
        {
            if (DIM == 3) {
                const float q0 = __fmaf_rn(T[6], r2, __fmaf_rn(T[0], r0, __fmul_rn(T[3], r1)));
                const float q1 = __fmaf_rn(T[7], r2, __fmaf_rn(T[1], r0, __fmul_rn(T[4], r1)));
                const float q2 = __fmaf_rn(T[8], r2, __fmaf_rn(T[2], r0, __fmul_rn(T[5], r1)));
                return tex2DLayered<float>(sino, __fdiv_rn(q0, q2), __fdiv_rn(q1, q2), p);
            }
            const float q0 = __fmaf_rn(T[0], r0, __fmul_rn(T[2], r1));
            const float q1 = __fmaf_rn(T[1], r0, __fmul_rn(T[3], r1));
            return tex1DLayered<float>(sino, __fdiv_rn(q0, q1), p);
        }

        constexpr int kFastRows = 4;   // (y, z) rows per block of the fast adjoint
        constexpr int kFastChunk = 8;  // steps per lane summed in registers at once

        template <int DIM>
        __global__ void __launch_bounds__(32 * kFastRows)
            josephFastAdjointKernel(cudaTextureObject_t sino, const float* __restrict__ table,
                                    int np, VolumeShape vol, float* __restrict__ x)
        {
            constexpr int kT = DIM == 3 ? 12 : 6; // block (column-major) + origin
            extern __shared__ float tab[];        // kT floats per view
            for (int i = threadIdx.y * 32 + threadIdx.x; i < kT * np; i += 32 * kFastRows)
                tab[i] = table[i];
            __syncthreads();
            const int lane = threadIdx.x;
            const int row = blockIdx.x * kFastRows + threadIdx.y;
            const int nrows = vol.n[1] * (DIM == 3 ? vol.n[2] : 1);
            if (row >= nrows)
                return;
            // rows z fastest, as the reference's grid: neighbouring blocks then read neighbouring
            // detector rows of a view through the texture cache
            const int nz = DIM == 3 ? vol.n[2] : 1;
            const int zi = row % nz, yi = row / nz;
            const int nsteps = vol.n[0] / 32, rem = vol.n[0] - nsteps * 32;
            const float c1 = static_cast<float>(yi) + 0.5f;
            const float c2 = static_cast<float>(zi) + 0.5f;
            float* out = x + static_cast<int64_t>(vol.n[0]) * (yi + static_cast<int64_t>(vol.n[1]) * zi);
            const float c0 = static_cast<float>(lane) + 0.5f;
            for (int s0 = 0; s0 < nsteps; s0 += kFastChunk) {
                const int cnt = min(kFastChunk, nsteps - s0);
                float acc[kFastChunk];
#pragma unroll
                for (int k = 0; k < kFastChunk; ++k)
                    acc[k] = 0.0f;
                for (int p = 0; p < np; ++p) {
                    const float* T = tab + kT * p;
                    float r0 = __fsub_rn(c0, T[DIM * DIM]);
                    for (int s = 0; s < s0; ++s)
                        r0 = __fadd_rn(r0, 32.0f);
                    const float r1 = __fsub_rn(c1, T[DIM * DIM + 1]);
                    const float r2 = DIM == 3 ? __fsub_rn(c2, T[11]) : 0.0f;
#pragma unroll
                    for (int k = 0; k < kFastChunk; ++k) {
                        if (k < cnt)
                            acc[k] = __fadd_rn(acc[k], fastSample<DIM>(sino, T, r0, r1, r2, p));
                        r0 = __fadd_rn(r0, 32.0f);
                    }
                }
#pragma unroll
                for (int k = 0; k < kFastChunk; ++k)
                    if (k < cnt)
                        out[lane + 32 * (s0 + k)] = acc[k];
            }
            if (lane < rem) {
                const int xi = nsteps * 32 + lane;
                const float cr = static_cast<float>(xi) + 0.5f;
                float acc = 0.0f;
                for (int p = 0; p < np; ++p) {
                    const float* T = tab + kT * p;
                    const float r0 = __fsub_rn(cr, T[DIM * DIM]);
                    const float r1 = __fsub_rn(c1, T[DIM * DIM + 1]);
                    const float r2 = DIM == 3 ? __fsub_rn(c2, T[11]) : 0.0f;
                    acc = __fadd_rn(acc, fastSample<DIM>(sino, T, r0, r1, r2, p));
                }
                out[xi] = acc;
            }
        }

        // Detector window of every (brick, view): projection of the brick grown by one voxel,
        // plus one pixel of margin. Falls back to the whole detector when a corner lies behind
        // the source.
        // Number of entries of the ascending table t[0..n) that are < x (le: <= x).
        __device__ __forceinline__ int countBelow(const float* __restrict__ t, int n, float x,
                                                  bool le)
        {
            int lo = 0, hi = n;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (le ? (t[mid] <= x) : (t[mid] < x))
                    lo = mid + 1;
                else
                    hi = mid;
            }
            return lo;
        }

        // grow > 0 (tight mode, flat detectors): the window holds exactly the pixels whose
        // centres lie in the projection of the brick grown by `grow` voxels on every side, plus
        // `pixMargin` pixels (the float rays deviate from the exact pixel-centre rays by far less
        // than both). A Joseph sample on driving plane k touches the brick only if its position
        // lies within half a voxel of the brick in both non-driving axes (taps floor(p - 0.5)
        // and floor(p - 0.5) + 1), so grow = 0.5 plus the accumulated-position slack suffices.
        // grow = 0: the conservative window (brick grown by one voxel, one pixel of margin).
        __global__ void josephWindowKernel(const float* __restrict__ poses, VolumeShape vol,
                                           DetectorShape det, int3 brick, int3 nBricks,
                                           CurvedMap cm, float grow, float pixMargin,
                                           RayWindow* __restrict__ out)
        {
            const int nb = nBricks.x * nBricks.y * nBricks.z;
            const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            if (t >= static_cast<int64_t>(nb) * det.np)
                return;
            const int bi = static_cast<int>(t % nb);
            const int p = static_cast<int>(t / nb);
            const float* P = poses + static_cast<int64_t>(p) * 40;
            const int bxi = bi % nBricks.x, byi = (bi / nBricks.x) % nBricks.y,
                      bzi = bi / (nBricks.x * nBricks.y);
            const bool tight = grow > 0.0f && !cm.planarU;
            const float g = tight ? grow : 1.0f;
            const float lo0 = static_cast<float>(bxi * brick.x) - g;
            const float lo1 = static_cast<float>(byi * brick.y) - g;
            const float lo2 = static_cast<float>(bzi * brick.z) - g;
            const float hi0 = static_cast<float>(bxi * brick.x + brick.x) + g;
            const float hi1 = static_cast<float>(byi * brick.y + brick.y) + g;
            const float hi2 = static_cast<float>(bzi * brick.z + brick.z) + g;
            float umin = 1e30f, umax = -1e30f, vmin = 1e30f, vmax = -1e30f;
            bool behind = false;
            const int corners = vol.dim == 3 ? 8 : 4;
            for (int c = 0; c < corners; ++c) {
                const float X = (c & 1) ? hi0 : lo0;
                const float Y = (c & 2) ? hi1 : lo1;
                if (vol.dim == 3) {
                    const float Z = (c & 4) ? hi2 : lo2;
                    const float h0 = P[0] * X + P[1] * Y + P[2] * Z + P[3];
                    const float h1 = P[4] * X + P[5] * Y + P[6] * Z + P[7];
                    const float h2 = P[8] * X + P[9] * Y + P[10] * Z + P[11];
                    if (!(h2 > 1e-6f)) {
                        behind = true;
                        break;
                    }
                    const float u = h0 / h2, v = h1 / h2;
                    umin = fminf(umin, u), umax = fmaxf(umax, u);
                    vmin = fminf(vmin, v), vmax = fmaxf(vmax, v);
                } else {
                    const float h0 = P[0] * X + P[1] * Y + P[2];
                    const float h1 = P[3] * X + P[4] * Y + P[5];
                    if (!(h1 > 1e-6f)) {
                        behind = true;
                        break;
                    }
                    const float u = h0 / h1;
                    umin = fminf(umin, u), umax = fmaxf(umax, u);
                    vmin = 0.0f, vmax = 0.0f;
                }
            }
            RayWindow w;
            if (behind) {
                w.u0 = 0, w.u1 = det.nu - 1, w.v0 = 0, w.v1 = det.nv - 1;
            } else if (cm.planarU) {
                // curved detector: the rays of pixel column u pass planar coordinate
                // planarU[u] (ascending), and rows are stretched by a factor in [fmin, fmax]
                // about the detector's centre row
                const int below = countBelow(cm.planarU, det.nu, umin, true);
                const int before = countBelow(cm.planarU, det.nu, umax, false);
                w.u0 = max(0, below - 2);
                w.u1 = min(det.nu - 1, before + 1);
                if (vol.dim == 3) {
                    const float cy = 0.5f * static_cast<float>(det.nv);
                    const float lo = cy + fminf((vmin - cy) / cm.fmin, (vmin - cy) / cm.fmax);
                    const float hi = cy + fmaxf((vmax - cy) / cm.fmin, (vmax - cy) / cm.fmax);
                    const float vLo = fmaxf(floorf(lo - 0.5f) - 1.0f, -1.0f);
                    const float vHi = fminf(ceilf(hi - 0.5f) + 1.0f, static_cast<float>(det.nv));
                    w.v0 = max(0, static_cast<int>(vLo));
                    w.v1 = min(det.nv - 1, static_cast<int>(vHi));
                } else {
                    w.v0 = 0, w.v1 = 0;
                }
            } else if (tight) {
                // pixels whose centres i + 0.5 lie in [umin - margin, umax + margin]
                const float uLo = fmaxf(ceilf(umin - 0.5f - pixMargin), -1.0f);
                const float uHi = fminf(floorf(umax - 0.5f + pixMargin), static_cast<float>(det.nu));
                w.u0 = max(0, static_cast<int>(uLo));
                w.u1 = min(det.nu - 1, static_cast<int>(uHi));
                if (vol.dim == 3) {
                    const float vLo = fmaxf(ceilf(vmin - 0.5f - pixMargin), -1.0f);
                    const float vHi =
                        fminf(floorf(vmax - 0.5f + pixMargin), static_cast<float>(det.nv));
                    w.v0 = max(0, static_cast<int>(vLo));
                    w.v1 = min(det.nv - 1, static_cast<int>(vHi));
                } else {
                    w.v0 = 0, w.v1 = 0;
                }
            } else {
                // pixel i has its centre at i + 0.5
                const float uLo = fmaxf(floorf(umin - 0.5f) - 1.0f, -1.0f);
                const float uHi = fminf(ceilf(umax - 0.5f) + 1.0f, static_cast<float>(det.nu));
                w.u0 = max(0, static_cast<int>(uLo));
                w.u1 = min(det.nu - 1, static_cast<int>(uHi));
                if (vol.dim == 3) {
                    const float vLo = fmaxf(floorf(vmin - 0.5f) - 1.0f, -1.0f);
                    const float vHi =
                        fminf(ceilf(vmax - 0.5f) + 1.0f, static_cast<float>(det.nv));
                    w.v0 = max(0, static_cast<int>(vLo));
                    w.v1 = min(det.nv - 1, static_cast<int>(vHi));
                } else {
                    w.v0 = 0, w.v1 = 0;
                }
            }
            out[t] = w;
        }

        // Check of the brick windows (test support, elsa_projector_info key 8): every tap of
        // every sample must lie in a brick whose window for the ray's view contains the ray.
        // Counts the taps that violate this.
        __global__ void josephWindowCheckKernel(const JosephRay* __restrict__ rays,
                                                const RayWindow* __restrict__ windows,
                                                VolumeShape vol, DetectorShape det, int3 brick,
                                                int3 nBricks, int onlyAxis,
                                                unsigned long long* __restrict__ misses)
        {
            const int64_t nrays = static_cast<int64_t>(det.nu) * det.nv * det.np;
            const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            if (r >= nrays)
                return;
            const JosephRay R = rays[r];
            if (R.n == 0 || (onlyAxis >= 0 && (R.meta & 3) != onlyAxis))
                return;
            const int u = static_cast<int>(r % det.nu);
            const int v = static_cast<int>((r / det.nu) % det.nv);
            const int p = static_cast<int>(r / (static_cast<int64_t>(det.nu) * det.nv));
            const int nb = nBricks.x * nBricks.y * nBricks.z;
            const int g = R.meta & 3;
            const int dir = (R.meta & 4) ? -1 : 1;
            int a, b;
            nonDrivingAxes(g, a, b);
            const int bext[3] = {brick.x, brick.y, brick.z};
            float pa = R.pa, pb = R.pb;
            int k = R.k0;
            unsigned long long bad = 0;
            int lastBrick = -1;
            for (int j = 0; j < R.n; ++j, k += dir, pa = __fadd_rn(pa, R.sa),
                     pb = __fadd_rn(pb, R.sb)) {
                const int ia = static_cast<int>(floorf(__fsub_rn(pa, 0.5f)));
                const int ib = static_cast<int>(floorf(__fsub_rn(pb, 0.5f)));
                for (int t = 0; t < (vol.dim == 3 ? 4 : 2); ++t) {
                    int c[3];
                    c[g] = k;
                    c[a] = ia + (t & 1);
                    if (vol.dim == 3)
                        c[b] = ib + (t >> 1);
                    else
                        c[2] = 0;
                    bool in = true;
                    for (int i = 0; i < vol.dim; ++i)
                        in = in && c[i] >= 0 && c[i] < vol.n[i];
                    if (!in)
                        continue;
                    const int bi = c[0] / bext[0] + nBricks.x *
                                   (c[1] / bext[1] + nBricks.y * (vol.dim == 3 ? c[2] / bext[2] : 0));
                    if (bi == lastBrick)
                        continue;
                    const RayWindow w = windows[static_cast<int64_t>(p) * nb + bi];
                    if (u < w.u0 || u > w.u1 || v < w.v0 || v > w.v1)
                        ++bad;
                    else
                        lastBrick = bi;
                }
            }
            if (bad)
                atomicAdd(misses, bad);
        }

        // Approximate non-driving position of ray R on driving plane k (pos0 + j*step). It
        // differs from the accumulated position by at most n/2 ulp, which the separation margin
        // below absorbs.
        __device__ __forceinline__ float planePos(const JosephRay& R, int k, bool second)
        {
            const int dir = (R.meta & 4) ? -1 : 1;
            const float fj = static_cast<float>((k - R.k0) * dir);
            return second ? fmaf(fj, R.sb, R.pb) : fmaf(fj, R.sa, R.pa);
        }

        // True when rays R and S (same driving axis) stay more than two voxels apart in one
        // non-driving coordinate over their common planes, so their bilinear taps are disjoint.
        __device__ bool separated(const JosephRay& R, const JosephRay& S, int dim)
        {
            const int dr = (R.meta & 4) ? -1 : 1, ds = (S.meta & 4) ? -1 : 1;
            const int r0 = R.k0, r1 = R.k0 + (R.n - 1) * dr;
            const int s0 = S.k0, s1 = S.k0 + (S.n - 1) * ds;
            const int lo = max(min(r0, r1), min(s0, s1));
            const int hi = min(max(r0, r1), max(s0, s1));
            if (lo > hi)
                return true;
            const float margin = 2.05f;
            const float da0 = planePos(R, lo, false) - planePos(S, lo, false);
            const float da1 = planePos(R, hi, false) - planePos(S, hi, false);
            if ((da0 > margin && da1 > margin) || (da0 < -margin && da1 < -margin))
                return true;
            if (dim == 3) {
                const float db0 = planePos(R, lo, true) - planePos(S, lo, true);
                const float db1 = planePos(R, hi, true) - planePos(S, hi, true);
                if ((db0 > margin && db1 > margin) || (db0 < -margin && db1 < -margin))
                    return true;
            }
            return false;
        }

        // Records the driving axes present per view and, per candidate class spacing m, whether
        // two same-class neighbours could share a bilinear tap.
        __global__ void josephClassCheckKernel(const JosephRay* __restrict__ rays,
                                               DetectorShape det, int dim,
                                               unsigned* __restrict__ viewAxes,
                                               unsigned* __restrict__ badSpacing,
                                               unsigned long long* __restrict__ samples)
        {
            const int64_t nrays = static_cast<int64_t>(det.nu) * det.nv * det.np;
            const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            if (r >= nrays)
                return;
            const JosephRay R = rays[r];
            if (R.n == 0)
                return;
            const int u = static_cast<int>(r % det.nu);
            const int v = static_cast<int>((r / det.nu) % det.nv);
            const int p = static_cast<int>(r / (static_cast<int64_t>(det.nu) * det.nv));
            atomicOr(viewAxes + p, 1u << (R.meta & 3));
            atomicAdd(samples, static_cast<unsigned long long>(R.n));
            unsigned bad = 0;
            for (int m = kMinClass; m <= kMaxClass; ++m) {
                // pairs that the adjoint may process concurrently: same row m apart, and rows m
                // apart with any offset inside a 32-ray segment (plus one)
                const int noffs = dim == 3 ? 2 + 65 : 1;
                for (int o = 0; o < noffs; ++o) {
                    const int du = o == 0 ? m : (o == 1 ? 33 : o - 2 - 32);
                    const int dv = o < 2 ? 0 : m;
                    const int u2 = u + du, v2 = v + dv;
                    if (u2 < 0 || u2 >= det.nu || v2 < 0 || v2 >= det.nv)
                        continue;
                    const JosephRay S = rays[u2 + static_cast<int64_t>(det.nu) *
                                                       (v2 + static_cast<int64_t>(det.nv) * p)];
                    if (S.n == 0 || (S.meta & 3) != (R.meta & 3))
                        continue;
                    if (!separated(R, S, dim))
                        bad |= 1u << m;
                }
            }
            if (bad)
                atomicOr(badSpacing, bad);
        }

        // Exact accumulated position of every ray at its first sample in each driving-axis slab
        // of `depth` planes. Slab-major layout: row floor(k/depth) + 1, column = ray index, so a
        // warp of neighbouring rays reads one contiguous run.
        __global__ void josephCheckpointKernel(const JosephRay* __restrict__ rays, int64_t nrays,
                                               int depth, int slabRows,
                                               float2* __restrict__ checkpoints)
        {
            const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            if (r >= nrays)
                return;
            const JosephRay R = rays[r];
            if (R.n == 0)
                return;
            const int dir = (R.meta & 4) ? -1 : 1;
            float pa = R.pa, pb = R.pb;
            int k = R.k0, slab = floorDiv(R.k0, depth) - dir;
            for (int j = 0; j < R.n; ++j, k += dir) {
                const int s = floorDiv(k, depth);
                if (s != slab) {
                    slab = s;
                    // rows 0 .. slabRows-1 cover k in [-depth, (slabRows-1)*depth); the host
                    // sizes slabRows for every sample of an N-plane volume
                    if (s + 1 >= 0 && s + 1 < slabRows)
                        checkpoints[(s + 1) * nrays + r] = make_float2(pa, pb);
                }
                pa = __fadd_rn(pa, R.sa);
                pb = __fadd_rn(pb, R.sb);
            }
        }

        // Sample range [jLo, jHi] of ray R inside driving planes [kLo, kHi]; false if empty.
        __device__ __forceinline__ bool sampleRange(const JosephRay& R, int kLo, int kHi, int& jLo,
                                                    int& jHi)
        {
            const int dir = (R.meta & 4) ? -1 : 1;
            if (dir > 0) {
                jLo = max(0, kLo - R.k0);
                jHi = min(R.n - 1, kHi - R.k0);
            } else {
                jLo = max(0, R.k0 - kHi);
                jHi = min(R.n - 1, R.k0 - kLo);
            }
            return jLo <= jHi;
        }

        // Strides of the shared-memory brick (x fastest; the plane stride is padded by one word
        // so that neighbouring rays stepping along z or x hit different banks).
        template <int DIM, int BX, int BY>
        struct BrickLayout {
            static constexpr int kRow = DIM == 3 ? BX : BX + 1;
            static constexpr int kPlane = DIM == 3 ? BX * BY + 1 : kRow * BY;
        };

        // Axis roles for driving axis G: stride/extent of G and of the non-driving axes a < b.
        template <int DIM, int G, int BX, int BY, int BZ>
        struct AxisRoles {
            using L = BrickLayout<DIM, BX, BY>;
            static constexpr int strG = G == 0 ? 1 : (G == 1 ? L::kRow : L::kPlane);
            static constexpr int extG = G == 0 ? BX : (G == 1 ? BY : BZ);
            static constexpr int strA = G == 0 ? L::kRow : 1;
            static constexpr int extA = G == 0 ? BY : BX;
            static constexpr int strB = DIM == 2 ? 0 : (G == 2 ? L::kRow : L::kPlane);
            static constexpr int extB = DIM == 2 ? 1 : (G == 2 ? BY : BZ);
        };

        // Add to the brick word at local lane-axis column L, row-axis row O (if inside).
        template <int EXT_L, int EXT_O, int STR_L, int STR_O>
        __device__ __forceinline__ void addTap(float* plane, int L, int O, float v)
        {
            if (static_cast<unsigned>(L) < static_cast<unsigned>(EXT_L) &&
                static_cast<unsigned>(O) < static_cast<unsigned>(EXT_O)) {
                float* q = plane + L * STR_L + O * STR_O;
                *q = *q + v;
            }
        }

        // One warp splats 32 neighbouring rays (u = uSeg0 + lane) of detector row v through the
        // brick, plane by plane in ray order. Lanes spread along the "lane axis" (a, or b when
        // LB); taps landing in the same column are merged across neighbouring lanes, then the
        // first and the second column of every lane's bilinear footprint are written in two
        // separate phases, so no two lanes touch the same word at the same time. When the merge
        // precondition fails (two neighbours on one column but different rows, or three on one
        // column) the plane falls back to m phases of lanes m apart, which the class check proves
        // disjoint.
        template <int DIM, int G, bool LB, int BX, int BY, int BZ, int CPD>
        __device__ __forceinline__ void splatRowSegment(
            float* acc, const JosephRay* __restrict__ rays, const float2* __restrict__ cps,
            int64_t nrays, const float* __restrict__ y, const DetectorShape& det, int p, int v,
            int uSeg0, int u1, int m, int orgG, int orgA, int orgB)
        {
            using AR = AxisRoles<DIM, G, BX, BY, BZ>;
            constexpr int EXT_L = LB ? AR::extB : AR::extA;
            constexpr int EXT_O = LB ? AR::extA : AR::extB;
            constexpr int STR_L = LB ? AR::strB : AR::strA;
            constexpr int STR_O = LB ? AR::strA : AR::strB;
            const int lane = threadIdx.x & 31;
            const int u = uSeg0 + lane;
            const int kLo = orgG, kHi = orgG + AR::extG - 1;
            const int64_t r =
                u + static_cast<int64_t>(det.nu) * (v + static_cast<int64_t>(det.nv) * p);
            JosephRay R{};
            bool act = u <= u1;
            if (act)
                R = rays[r];
            act = act && R.n > 0 && (R.meta & 3) == G;
            int jLo = 0, jHi = -1;
            if (act)
                act = sampleRange(R, kLo, kHi, jLo, jHi);
            const int dir = (R.meta & 4) ? -1 : 1;
            float pa = 0.0f, pb = 0.0f, yl = 0.0f;
            if (act) {
                const int kFirst = R.k0 + jLo * dir;
                const float2 cp = __ldg(cps + (floorDiv(kFirst, CPD) + 1) * nrays + r);
                pa = cp.x, pb = cp.y;
                yl = __ldg(y + r) * R.len;
            }
            for (int dsel = 1; dsel >= -1; dsel -= 2) {
                const bool part = act && dir == dsel;
                if (!__any_sync(0xffffffffu, part))
                    continue;
                // plane offsets t in ray order: k = kLo + t (dir > 0) or kHi - t (dir < 0)
                const int kFirst = R.k0 + jLo * dir;
                const int t0 = part ? (dsel > 0 ? kFirst - kLo : kHi - kFirst) : (1 << 20);
                const int t1 = part ? t0 + (jHi - jLo) : -1;
                int tMin = t0, tMax = t1;
                for (int o = 16; o > 0; o >>= 1) {
                    tMin = min(tMin, __shfl_xor_sync(0xffffffffu, tMin, o));
                    tMax = max(tMax, __shfl_xor_sync(0xffffffffu, tMax, o));
                }
                for (int t = tMin; t <= tMax; ++t) {
                    const bool on = part && t >= t0 && t <= t1;
                    const int k = dsel > 0 ? kLo + t : kHi - t;
                    float* plane = acc + (k - orgG) * AR::strG;
                    int L = 0, O = 0;
                    float A = 0.0f, B = 0.0f, C = 0.0f, D = 0.0f;
                    if (on) {
                        Weights w;
                        tapWeights(pa, pb, w);
                        const int la = w.ia - orgA, lb = w.ib - orgB;
                        L = LB ? lb : la;
                        O = DIM == 2 ? 0 : (LB ? la : lb);
                        const float wl0 = LB ? w.wb : w.wa, wl1 = LB ? w.cwb : w.cwa;
                        const float wo0 = LB ? w.wa : w.wb, wo1 = LB ? w.cwa : w.cwb;
                        if (DIM == 2) {
                            A = yl * wl0;
                            B = yl * wl1;
                        } else {
                            A = yl * (wl0 * wo0);
                            B = yl * (wl1 * wo0);
                            C = yl * (wl0 * wo1);
                            D = yl * (wl1 * wo1);
                        }
                        pa = __fadd_rn(pa, R.sa);
                        pb = __fadd_rn(pb, R.sb);
                    }
                    // neighbour state packed in one word: bit 0 active, bits 1.. column + 2^20
                    const int packed = on ? (((L + (1 << 20)) << 1) | 1) : 0;
                    const int prev = __shfl_up_sync(0xffffffffu, packed, 1);
                    const int prev2 = __shfl_up_sync(0xffffffffu, packed, 2);
                    const bool pOn = lane > 0 && (prev & 1);
                    const int pL = (prev >> 1) - (1 << 20);
                    const bool p2On = lane > 1 && (prev2 & 1);
                    const int p2L = (prev2 >> 1) - (1 << 20);
                    const bool second = on && pOn && pL == L; // second ray on this column
                    // columns must be monotone along the active lanes and hold at most two rays
                    const bool inc = __any_sync(0xffffffffu, on && pOn && pL < L);
                    const bool dec = __any_sync(0xffffffffu, on && pOn && pL > L);
                    const bool triple = __any_sync(0xffffffffu, second && p2On && p2L == L);
                    if (!(inc && dec) && !triple) {
                        // first rays of distinct columns, then second rays: within one phase
                        // all writers sit on distinct columns
#pragma unroll
                        for (int ph = 0; ph < 4; ++ph) {
                            const bool mine = on && (second == (ph >= 2));
                            const int col = L + (ph & 1);
                            if (mine) {
                                addTap<EXT_L, EXT_O, STR_L, STR_O>(plane, col, O, (ph & 1) ? B : A);
                                if (DIM == 3)
                                    addTap<EXT_L, EXT_O, STR_L, STR_O>(plane, col, O + 1,
                                                                       (ph & 1) ? D : C);
                            }
                            __syncwarp();
                        }
                    } else {
                        for (int ph = 0; ph < m; ++ph) {
                            if (on && lane % m == ph) {
                                addTap<EXT_L, EXT_O, STR_L, STR_O>(plane, L, O, A);
                                addTap<EXT_L, EXT_O, STR_L, STR_O>(plane, L + 1, O, B);
                                if (DIM == 3) {
                                    addTap<EXT_L, EXT_O, STR_L, STR_O>(plane, L, O + 1, C);
                                    addTap<EXT_L, EXT_O, STR_L, STR_O>(plane, L + 1, O + 1, D);
                                }
                            }
                            __syncwarp();
                        }
                    }
                }
            }
        }

        // All row segments of one (view, driving axis G) for a brick. Warps take (row, 32-ray
        // segment) units; units that run concurrently are rows at least m apart or segments
        // separated by a whole segment, so their taps are disjoint. Phases end with barriers.
        template <int DIM, int G, bool LB, int BX, int BY, int BZ, int CPD, int NW>
        __device__ __forceinline__ void splatView(float* acc, const RayWindow& w, int p,
                                                  const JosephRay* __restrict__ rays,
                                                  const float2* __restrict__ cps, int64_t nrays,
                                                  const float* __restrict__ y,
                                                  const DetectorShape& det, int m, int org0,
                                                  int org1, int org2)
        {
            const int orgG = G == 0 ? org0 : (G == 1 ? org1 : org2);
            const int orgA = G == 0 ? org1 : org0;
            const int orgB = DIM == 2 ? 0 : (G == 2 ? org1 : org2);
            const int warp = threadIdx.x >> 5;
            const int nseg = (w.u1 - w.u0) / 32 + 1;
            const int rowPhases = DIM == 3 ? m : 1;
            for (int pr = 0; pr < rowPhases; ++pr) {
                const int vFirst = w.v0 + pr;
                const int nRows = DIM == 3 ? (vFirst <= w.v1 ? (w.v1 - vFirst) / m + 1 : 0) : 1;
                for (int ps = 0; ps < 2 && ps < nseg; ++ps) {
                    const int nSegs = (nseg - ps + 1) / 2;
                    const int units = nRows * nSegs;
                    for (int unit = warp; unit < units; unit += NW) {
                        const int row = unit / nSegs, seg = unit - row * nSegs;
                        const int v = DIM == 3 ? vFirst + row * m : 0;
                        splatRowSegment<DIM, G, LB, BX, BY, BZ, CPD>(
                            acc, rays, cps, nrays, y, det, p, v, w.u0 + 32 * (ps + 2 * seg),
                            w.u1, m, orgG, orgA, orgB);
                    }
                    __syncthreads();
                }
            }
        }

        // One CTA per brick of BX x BY x BZ voxels (BZ = 1 in 2D), NW warps. The brick
        // accumulates every view in a fixed order and is written once.
        template <int DIM, int BX, int BY, int BZ, int CPD, int NW>
        __global__ void __launch_bounds__(NW * 32)
            josephAdjointKernel(const JosephRay* __restrict__ rays,
                                const float2* __restrict__ checkpoints, int64_t nrays,
                                const float* __restrict__ y,
                                const RayWindow* __restrict__ windows,
                                const unsigned* __restrict__ viewAxes, VolumeShape vol,
                                DetectorShape det, int m, int3 nBricks, int viewsPerChunk,
                                float* __restrict__ x)
        {
            // blockIdx.y selects a chunk of views; with several chunks each CTA writes its
            // partial brick to x + chunk * nvox and a second pass sums the chunks in order
            extern __shared__ float smem[];
            using L = BrickLayout<DIM, BX, BY>;
            constexpr int NT = NW * 32;
            constexpr int kWords = L::kPlane * BZ;
            float* acc = smem;
            RayWindow* win = reinterpret_cast<RayWindow*>(smem + ((kWords + 3) & ~3));
            unsigned* axes = reinterpret_cast<unsigned*>(win + det.np);
            const int bi = blockIdx.x;
            const int org0 = (bi % nBricks.x) * BX, org1 = ((bi / nBricks.x) % nBricks.y) * BY,
                      org2 = (bi / (nBricks.x * nBricks.y)) * BZ;
            const int nb = nBricks.x * nBricks.y * nBricks.z;
            const int pBegin = blockIdx.y * viewsPerChunk;
            const int pEnd = min(det.np, pBegin + viewsPerChunk);
            for (int i = threadIdx.x; i < kWords; i += NT)
                acc[i] = 0.0f;
            for (int p = pBegin + threadIdx.x; p < pEnd; p += NT) {
                const RayWindow w = windows[static_cast<int64_t>(p) * nb + bi];
                win[p] = w;
                axes[p] = (w.u0 > w.u1 || w.v0 > w.v1) ? 0u : viewAxes[p];
            }
            __syncthreads();
            const int64_t nvox = static_cast<int64_t>(vol.n[0]) * vol.n[1] * vol.n[2];
            float* out = x + blockIdx.y * nvox;
            for (int p = pBegin; p < pEnd; ++p) {
                const unsigned ax = axes[p];
                if (!(ax & 7u))
                    continue;
                const RayWindow w = win[p];
                // bit g: rays drive along g; bit 4+g: their lanes spread along axis b
#define ELSA_SPLAT(G_)                                                                            \
    if (ax & (1u << G_)) {                                                                        \
        if (ax & (16u << G_))                                                                     \
            splatView<DIM, G_, true, BX, BY, BZ, CPD, NW>(acc, w, p, rays, checkpoints, nrays, y, \
                                                          det, m, org0, org1, org2);              \
        else                                                                                      \
            splatView<DIM, G_, false, BX, BY, BZ, CPD, NW>(acc, w, p, rays, checkpoints, nrays,   \
                                                           y, det, m, org0, org1, org2);          \
    }
                ELSA_SPLAT(0)
                ELSA_SPLAT(1)
                if (DIM == 3) {
                    ELSA_SPLAT((DIM == 3 ? 2 : 1))
                }
#undef ELSA_SPLAT
            }
            for (int i = threadIdx.x; i < BX * BY * BZ; i += NT) {
                const int lx = i % BX, ly = (i / BX) % BY, lz = i / (BX * BY);
                const int gx = org0 + lx, gy = org1 + ly, gz = org2 + lz;
                if (gx < vol.n[0] && gy < vol.n[1] && gz < vol.n[2])
                    out[gx + static_cast<int64_t>(vol.n[0]) *
                                 (gy + static_cast<int64_t>(vol.n[1]) * gz)] =
                        acc[lz * L::kPlane + ly * L::kRow + lx];
            }
        }

        // x[v] = sum over chunks c = 0, 1, ... of partial[c][v], in chunk order
        __global__ void sumChunksKernel(const float* __restrict__ partial, int chunks,
                                        int64_t nvox, float* __restrict__ x)
        {
            const int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            if (v >= nvox)
                return;
            float s = partial[v];
            for (int c = 1; c < chunks; ++c)
                s = s + partial[c * nvox + v];
            x[v] = s;
        }

        // sumChunksKernel for many volumes: blockIdx.y selects (partials, count, nvox, out)
        struct SumChunksEntry {
            const float* partial;
            int chunks;
            int64_t nvox;
            float* x;
        };
        __global__ void sumChunksManyKernel(const SumChunksEntry* __restrict__ e)
        {
            const SumChunksEntry E = e[blockIdx.y];
            for (int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
                 v < E.nvox; v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
                float s = E.partial[v];
                for (int c = 1; c < E.chunks; ++c)
                    s = s + E.partial[c * E.nvox + v];
                E.x[v] = s;
            }
        }

#ifndef ELSA_ADJ2D_CTAS_PER_SM
#define ELSA_ADJ2D_CTAS_PER_SM 16
#endif
        constexpr int kAdjoint2dCtasPerSm = ELSA_ADJ2D_CTAS_PER_SM;
#ifndef ELSA_ADJ3D_WARPS_PER_SM
#define ELSA_ADJ3D_WARPS_PER_SM 22
#endif
        constexpr int kAdjoint3dWarpsPerSm = ELSA_ADJ3D_WARPS_PER_SM;
        constexpr int kMinAdjointChunks = 32;                // default floor of the view chunks
        constexpr int64_t kChunkMemory = int64_t(1) << 31;   // default partial-volume budget
        constexpr int64_t kBatchPartialMemory = int64_t(8) << 30; // batched adjoints: up to 8 GiB

        template <int DIM, int BX, int BY, int BZ, int CPD, int NW>
        struct AdjointConfig {
            using L = BrickLayout<DIM, BX, BY>;
            static constexpr size_t kAccBytes = sizeof(float) * ((L::kPlane * BZ + 3) & ~3);
            static constexpr int kThreads = NW * 32;
            static constexpr int kCheckpointDepth = CPD;
            static_assert(BX % CPD == 0 && BY % CPD == 0 && (DIM == 2 || BZ % CPD == 0),
                          "brick edges must be multiples of the checkpoint depth");
            static int3 brick() { return make_int3(BX, BY, BZ); }
            // accumulator + per-view windows and axis masks
            static size_t smemBytes(int np)
            {
                return kAccBytes + (sizeof(RayWindow) + sizeof(unsigned)) * np;
            }
            // The dynamic shared-memory limit is an attribute of the kernel on the device, shared
            // by every projector: it only ever grows, so a projector with fewer views created
            // later leaves room for the earlier ones.
            static void prepare(int np)
            {
                static std::mutex mu;
                std::lock_guard<std::mutex> lock(mu);
                cudaFuncAttributes attr{};
                ELSA_CUDA(cudaFuncGetAttributes(&attr,
                                                josephAdjointKernel<DIM, BX, BY, BZ, CPD, NW>));
                const int need = static_cast<int>(smemBytes(np));
                if (need > attr.maxDynamicSharedSizeBytes)
                    ELSA_CUDA(cudaFuncSetAttribute(josephAdjointKernel<DIM, BX, BY, BZ, CPD, NW>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   need));
            }
            // Views per chunk so that bricks x chunks fills about kAdjoint2dCtasPerSm CTAs per SM
            // (16 measured best among 1-16 at 128^2 x 180 views and 512^2 x 720 views). The
            // partial volumes then hold fewer than 2 x 16 x 148 tiles of 64 x 64 floats (78 MB).
            static int chunks(int nbricks, int np)
            {
                const int want = (kAdjoint2dCtasPerSm * 148 + nbricks - 1) / nbricks;
                return want < 1 ? 1 : (want > np ? np : want);
            }
            // nc view chunks; partial: scratch of nc volumes (unused with one chunk)
            static void launch(int nbricks, int nc, cudaStream_t s, const JosephRay* rays,
                               const float2* cps, int64_t nrays, const float* y,
                               const RayWindow* win, const unsigned* axes, VolumeShape vol,
                               DetectorShape det, int m, int3 nb, float* x, float* partial)
            {
                const int per = (det.np + nc - 1) / nc;
                const int used = (det.np + per - 1) / per;
                const dim3 grid(static_cast<unsigned>(nbricks), static_cast<unsigned>(used));
                josephAdjointKernel<DIM, BX, BY, BZ, CPD, NW>
                    <<<grid, kThreads, smemBytes(det.np), s>>>(rays, cps, nrays, y, win, axes,
                                                               vol, det, m, nb, per,
                                                               used > 1 ? partial : x);
                if (used > 1)
                    launchSumChunks(partial, used,
                                    static_cast<int64_t>(vol.n[0]) * vol.n[1] * vol.n[2], x, s);
            }
        };

        // ---------------------------------------------------------------------------------------
        // 3D adjoint on axis bricks. The rays of one view all step along about the same axis G, so
        // the volume is cut, per driving axis present, into bricks that are TD planes deep along G
        // and TA x TB voxels across (a < b the other two axes). A ray crossing such a brick keeps
        // most of its TD samples inside it (a 16^3 brick loses half of the samples of oblique rays
        // to its sides), and the window of a brick, the pixels whose centres lie in the projection
        // of the brick grown by about half a voxel, holds few rays that miss it. One warp owns a
        // brick in shared memory for a chunk of views and splats the window's rays class by class:
        // rays of one class are more than two voxels apart, so no two lanes add to one word at
        // once and the brick needs no atomics. A tap outside the brick is predicated off (the
        // neighbouring brick owns it); with ELSA_AXIS_HALO 2 the brick instead carries a two-voxel
        // halo into which tap indices are clamped, and the halo is not written out.
        // ---------------------------------------------------------------------------------------
#ifndef ELSA_AXIS_HALO
// halo of the axis bricks: 0, taps outside the brick predicated off (256^3: 35.9 ms); 2, taps
// clamped into a two-voxel halo (38.9 ms with 8-deep bricks, whose halo costs occupancy)
#define ELSA_AXIS_HALO 0
#endif
        constexpr int kAxisHalo = ELSA_AXIS_HALO;
        static_assert(kAxisHalo == 0 || kAxisHalo == 2, "halo of 0 or 2 voxels");

        // Shared-memory brick of TD planes (along G) of TV rows x TW columns. Columns run along
        // the non-driving axis over which the rays of a detector row spread (the warp's lanes
        // spread along it, so stride 1 there keeps their taps in different banks), rows along the
        // other one; both carry the halo.
#ifndef ELSA_ADJ_PACKED
#define ELSA_ADJ_PACKED 1 // the (a, b) pairs on the packed two-wide FP32 instructions (256^3:
                          // 32.92 -> 32.17 ms, the same adjoint bit for bit)
#endif
#ifndef ELSA_AXIS_PLANE_ODD
#define ELSA_AXIS_PLANE_ODD 0 // 1: pad the plane stride to 1 modulo 32 (256^3: 35.8 ms, 0: 33.5 ms)
#endif
#ifndef ELSA_AXIS_ROWPAD
#define ELSA_AXIS_ROWPAD (ELSA_AXIS_HALO == 0 ? 1 : 0) // extra words per row (bank spread)
#endif
        template <int TD, int TW, int TV>
        struct AxisBrick {
            // words per row (stride 1 axis)
            static constexpr int kRow = TW + 2 * kAxisHalo + ELSA_AXIS_ROWPAD;
            static constexpr int kRows = TV + 2 * kAxisHalo; // rows per plane
            static constexpr int kPlaneMin = kRow * kRows;
            // plane stride unpadded (smaller bricks, more of them resident per SM), or congruent
            // to 1 modulo 32 with ELSA_AXIS_PLANE_ODD 1 (lanes one plane apart in other banks)
            static constexpr int kPlane =
                ELSA_AXIS_PLANE_ODD ? kPlaneMin + ((33 - kPlaneMin % 32) % 32) : kPlaneMin;
            static constexpr int kWords = kPlane * TD;
        };

        // Axis roles of an axis brick: non-driving axes a < b of G; UB: the columns run along b
        // (else along a). Edges and word strides along a and b.
        template <int TD, bool UB, int TW, int TV>
        struct AxisRolesAB {
            using L = AxisBrick<TD, TW, TV>;
            static constexpr int EA = UB ? TV : TW, EB = UB ? TW : TV;
            static constexpr int SA = UB ? L::kRow : 1, SB = UB ? 1 : L::kRow;
            static constexpr int kOrigin = kAxisHalo * (SA + SB); // word of (a, b) = (0, 0)
        };

        // Word of the bilinear footprint of position (pa, pb) on `plane` (the brick word of
        // a = b = 0 on that plane) and the reference's weights (JosephsMethod.cpp:37-52); tap
        // indices outside the brick are clamped into the halo.
        template <int EA, int EB, int SA, int SB>
        __device__ __forceinline__ float* axisTap(float* plane, float pa, float pb, int orgA,
                                                  int orgB, float& wa, float& cwa, float& wb,
                                                  float& cwb)
        {
            const float fa = floorf(__fsub_rn(pa, 0.5f));
            const float fb = floorf(__fsub_rn(pb, 0.5f));
            cwa = __fsub_rn(__fsub_rn(pa, fa), 0.5f);
            cwb = __fsub_rn(__fsub_rn(pb, fb), 0.5f);
            wa = __fsub_rn(1.0f, cwa);
            wb = __fsub_rn(1.0f, cwb);
            const int la = min(max(static_cast<int>(fa) - orgA, -kAxisHalo), EA);
            const int lb = min(max(static_cast<int>(fb) - orgB, -kAxisHalo), EB);
            return plane + la * SA + lb * SB;
        }

        // Without a halo: the word offset of the footprint on its plane and a mask of the taps
        // inside the brick (bit t: tap (a + (t & 1), b + (t >> 1))).
        template <int EA, int EB, int SA, int SB>
        __device__ __forceinline__ int axisTapMasked(float pa, float pb, int orgA, int orgB,
                                                     float& wa, float& cwa, float& wb, float& cwb,
                                                     unsigned& mask)
        {
            // (floorSmall here, instead of floorf and a conversion: 256^3 33.3 ms against 32.9)
            const float fa = floorf(__fsub_rn(pa, 0.5f));
            const float fb = floorf(__fsub_rn(pb, 0.5f));
            const int ia = static_cast<int>(fa), ib = static_cast<int>(fb);
            cwa = __fsub_rn(__fsub_rn(pa, fa), 0.5f);
            cwb = __fsub_rn(__fsub_rn(pb, fb), 0.5f);
            wa = __fsub_rn(1.0f, cwa);
            wb = __fsub_rn(1.0f, cwb);
            const int la = ia - orgA, lb = ib - orgB;
            const bool a0 = static_cast<unsigned>(la) < static_cast<unsigned>(EA);
            const bool a1 = static_cast<unsigned>(la + 1) < static_cast<unsigned>(EA);
            const bool b0 = static_cast<unsigned>(lb) < static_cast<unsigned>(EB);
            const bool b1 = static_cast<unsigned>(lb + 1) < static_cast<unsigned>(EB);
            mask = (a0 && b0 ? 1u : 0u) | (a1 && b0 ? 2u : 0u) | (a0 && b1 ? 4u : 0u) |
                   (a1 && b1 ? 8u : 0u);
            return la * SA + lb * SB;
        }

        // Samples jLo..jHi of ray R (position cp at sample jLo, on brick plane t0) into the brick.
        // Software-pipelined: the footprint of sample j+1 (always on another plane) is read before
        // the sums of sample j are written back.
        template <int TD, bool UB, int TW, int TV>
        __device__ __forceinline__ void axisSplat(float* acc, const JosephRay& R, float yl,
                                                  float2 cp, int jLo, int jHi, int t0, int orgA,
                                                  int orgB)
        {
            using L = AxisBrick<TD, TW, TV>;
            using AR = AxisRolesAB<TD, UB, TW, TV>;
            constexpr int SA = AR::SA, SB = AR::SB;
#if ELSA_ADJ_PACKED
            if constexpr (kAxisHalo == 0) {
                // (a, b) pairs on the packed two-wide FP32 instructions: the same roundings
                const int dPlane = ((R.meta & 4) ? -1 : 1) * L::kPlane;
                const float2 h = make_float2(0.5f, 0.5f), one = make_float2(1.0f, 1.0f);
                const float2 s2 = make_float2(R.sa, R.sb), yy = make_float2(yl, yl);
                int plane = t0 * L::kPlane;
                float2 p2 = cp;
                auto tap = [&](int pl, float2& w, float2& cw, unsigned& mk) {
                    int ia, ib;
                    const float2 fl = floorSmall2(sub2(p2, h), ia, ib);
                    cw = sub2(sub2(p2, fl), h);
                    w = sub2(one, cw);
                    const int la = ia - orgA, lb = ib - orgB;
                    const bool a0 = static_cast<unsigned>(la) < static_cast<unsigned>(AR::EA);
                    const bool a1 = static_cast<unsigned>(la + 1) < static_cast<unsigned>(AR::EA);
                    const bool b0 = static_cast<unsigned>(lb) < static_cast<unsigned>(AR::EB);
                    const bool b1 = static_cast<unsigned>(lb + 1) < static_cast<unsigned>(AR::EB);
                    mk = (a0 && b0 ? 1u : 0u) | (a1 && b0 ? 2u : 0u) | (a0 && b1 ? 4u : 0u) |
                         (a1 && b1 ? 8u : 0u);
                    return pl + la * SA + lb * SB;
                };
                float2 w, cw;
                unsigned mk;
                int o = tap(plane, w, cw, mk);
                float2 v01 = make_float2((mk & 1u) ? acc[o] : 0.0f, (mk & 2u) ? acc[o + SA] : 0.0f);
                float2 v23 = make_float2((mk & 4u) ? acc[o + SB] : 0.0f,
                                         (mk & 8u) ? acc[o + SA + SB] : 0.0f);
                float2 yac = mul2(yy, make_float2(w.x, cw.x)); // (ya, yc)
                float wb = w.y, cwb = cw.y;
#pragma unroll kSplatUnroll
                for (int j = jLo; j < jHi; ++j) {
                    plane += dPlane;
                    p2 = add2(p2, s2);
                    float2 w2, cw2;
                    unsigned mk2;
                    const int o2 = tap(plane, w2, cw2, mk2);
                    const float2 n01 = make_float2((mk2 & 1u) ? acc[o2] : 0.0f,
                                                   (mk2 & 2u) ? acc[o2 + SA] : 0.0f);
                    const float2 n23 = make_float2((mk2 & 4u) ? acc[o2 + SB] : 0.0f,
                                                   (mk2 & 8u) ? acc[o2 + SA + SB] : 0.0f);
                    const float2 r01 = fma2(yac, make_float2(wb, wb), v01);
                    const float2 r23 = fma2(yac, make_float2(cwb, cwb), v23);
                    if (mk & 1u)
                        acc[o] = r01.x;
                    if (mk & 2u)
                        acc[o + SA] = r01.y;
                    if (mk & 4u)
                        acc[o + SB] = r23.x;
                    if (mk & 8u)
                        acc[o + SA + SB] = r23.y;
                    o = o2, mk = mk2;
                    v01 = n01, v23 = n23;
                    yac = mul2(yy, make_float2(w2.x, cw2.x));
                    wb = w2.y, cwb = cw2.y;
                }
                const float2 r01 = fma2(yac, make_float2(wb, wb), v01);
                const float2 r23 = fma2(yac, make_float2(cwb, cwb), v23);
                if (mk & 1u)
                    acc[o] = r01.x;
                if (mk & 2u)
                    acc[o + SA] = r01.y;
                if (mk & 4u)
                    acc[o + SB] = r23.x;
                if (mk & 8u)
                    acc[o + SA + SB] = r23.y;
                return;
            }
#endif
            if constexpr (kAxisHalo == 0) {
                const int dPlane = ((R.meta & 4) ? -1 : 1) * L::kPlane;
                int plane = t0 * L::kPlane;
                float pa = cp.x, pb = cp.y;
                float wa, cwa, wb, cwb;
                unsigned mk;
                int o = plane + axisTapMasked<AR::EA, AR::EB, SA, SB>(pa, pb, orgA, orgB, wa, cwa,
                                                                       wb, cwb, mk);
                float v0 = (mk & 1u) ? acc[o] : 0.0f, v1 = (mk & 2u) ? acc[o + SA] : 0.0f;
                float v2 = (mk & 4u) ? acc[o + SB] : 0.0f, v3 = (mk & 8u) ? acc[o + SA + SB] : 0.0f;
                float ya = yl * wa, yc = yl * cwa;
#pragma unroll kSplatUnroll
                for (int j = jLo; j < jHi; ++j) {
                    plane += dPlane;
                    pa = __fadd_rn(pa, R.sa);
                    pb = __fadd_rn(pb, R.sb);
                    float wa2, cwa2, wb2, cwb2;
                    unsigned mk2;
                    const int o2 = plane + axisTapMasked<AR::EA, AR::EB, SA, SB>(
                                               pa, pb, orgA, orgB, wa2, cwa2, wb2, cwb2, mk2);
                    const float n0 = (mk2 & 1u) ? acc[o2] : 0.0f;
                    const float n1 = (mk2 & 2u) ? acc[o2 + SA] : 0.0f;
                    const float n2 = (mk2 & 4u) ? acc[o2 + SB] : 0.0f;
                    const float n3 = (mk2 & 8u) ? acc[o2 + SA + SB] : 0.0f;
                    if (mk & 1u)
                        acc[o] = v0 + ya * wb;
                    if (mk & 2u)
                        acc[o + SA] = v1 + yc * wb;
                    if (mk & 4u)
                        acc[o + SB] = v2 + ya * cwb;
                    if (mk & 8u)
                        acc[o + SA + SB] = v3 + yc * cwb;
                    o = o2, mk = mk2;
                    v0 = n0, v1 = n1, v2 = n2, v3 = n3;
                    ya = yl * wa2, yc = yl * cwa2;
                    wb = wb2, cwb = cwb2;
                }
                if (mk & 1u)
                    acc[o] = v0 + ya * wb;
                if (mk & 2u)
                    acc[o + SA] = v1 + yc * wb;
                if (mk & 4u)
                    acc[o + SB] = v2 + ya * cwb;
                if (mk & 8u)
                    acc[o + SA + SB] = v3 + yc * cwb;
                return;
            }
            const int dPlane = ((R.meta & 4) ? -1 : 1) * L::kPlane;
            float* plane = acc + AR::kOrigin + t0 * L::kPlane;
            float pa = cp.x, pb = cp.y;
            float wa, cwa, wb, cwb;
            float* q = axisTap<AR::EA, AR::EB, SA, SB>(plane, pa, pb, orgA, orgB, wa, cwa, wb, cwb);
            float v0 = q[0], v1 = q[SA], v2 = q[SB], v3 = q[SA + SB];
            float ya = yl * wa, yc = yl * cwa;
#pragma unroll kSplatUnroll
            for (int j = jLo; j < jHi; ++j) {
                plane += dPlane;
                pa = __fadd_rn(pa, R.sa);
                pb = __fadd_rn(pb, R.sb);
                float wa2, cwa2, wb2, cwb2;
                float* q2 = axisTap<AR::EA, AR::EB, SA, SB>(plane, pa, pb, orgA, orgB, wa2, cwa2,
                                                           wb2, cwb2);
                const float n0 = q2[0], n1 = q2[SA], n2 = q2[SB], n3 = q2[SA + SB];
                q[0] = v0 + ya * wb;
                q[SA] = v1 + yc * wb;
                q[SB] = v2 + ya * cwb;
                q[SA + SB] = v3 + yc * cwb;
                q = q2;
                v0 = n0, v1 = n1, v2 = n2, v3 = n3;
                ya = yl * wa2, yc = yl * cwa2;
                wb = wb2, cwb = cwb2;
            }
            q[0] = v0 + ya * wb;
            q[SA] = v1 + yc * wb;
            q[SB] = v2 + ya * cwb;
            q[SA + SB] = v3 + yc * cwb;
        }

        // One view for an axis brick of grid G: m x m ray classes separated by __syncwarp; lane i
        // takes class rays i, i + 32, ... (u fastest within the class grid).
        template <int G, int TD, bool UB, int TW, int TV, int CPD>
        __device__ __forceinline__ void axisView(float* acc, const RayWindow& w, int p, int m,
                                                 int cpdShift, const JosephRay* __restrict__ rays,
                                                 const float2* __restrict__ cps, int64_t nrays,
                                                 const float* __restrict__ y,
                                                 const DetectorShape& det, int orgG, int orgA,
                                                 int orgB)
        {
            // Checkpoint slabs of CPD planes, or of 2^cpdShift planes when CPD is 0 (the
            // deeper slabs that save memory). A brick that does not start at its ray's first
            // sample in the slab catches up from the checkpoint by exact additions.
            const int kLo = orgG, kHi = orgG + TD - 1;
            const int shift = CPD > 0 ? 0 : cpdShift;
            const int slabLo = CPD > 0 ? (orgG / CPD) * CPD : (orgG >> shift) << shift;
            const int slabHi = slabLo + (CPD > 0 ? CPD : 1 << shift) - 1;
            const bool catchUp = CPD > 0 ? TD < CPD : (1 << shift) > TD;
            const int64_t cpRow =
                static_cast<int64_t>((CPD > 0 ? orgG / CPD : orgG >> shift) + 1) * nrays;
            const int lane = threadIdx.x & 31;
            const int64_t viewBase = static_cast<int64_t>(det.nu) * det.nv * p;
            for (int ov = 0; ov < m; ++ov) {
                const int vStart = w.v0 + ov;
                const int nvc = vStart <= w.v1 ? (w.v1 - vStart) / m + 1 : 0;
                for (int ou = 0; ou < m; ++ou) {
                    const int uStart = w.u0 + ou;
                    const int nuc = uStart <= w.u1 ? (w.u1 - uStart) / m + 1 : 0;
                    const int total = nuc * nvc;
                    const float invNuc = nuc > 0 ? 1.0f / static_cast<float>(nuc) : 0.0f;
                    constexpr int kBatch = ELSA_ADJ_BATCH;
                    for (int base = lane; base < total; base += 32 * kBatch) {
                        JosephRay Rb[kBatch];
                        float2 cpb[kBatch];
                        float yb[kBatch];
#pragma unroll
                        for (int q = 0; q < kBatch; ++q) {
                            const int i = base + 32 * q;
                            Rb[q].n = 0;
                            if (i < total) {
                                // i / nuc by a float reciprocal: exact for i < 2^20, nuc < 2^11
                                const int iv =
                                    static_cast<int>((static_cast<float>(i) + 0.5f) * invNuc);
                                const int iu = i - iv * nuc;
                                const int64_t r = viewBase + (uStart + iu * m) +
                                                  static_cast<int64_t>(det.nu) * (vStart + iv * m);
                                Rb[q] = rays[r];
                                cpb[q] = __ldg(cps + cpRow + r);
                                yb[q] = __ldg(y + r);
                            }
                        }
#pragma unroll
                        for (int q = 0; q < kBatch; ++q) {
                            const JosephRay& R = Rb[q];
                            if (R.n == 0 || (R.meta & 3) != G)
                                continue;
                            int jLo, jHi;
                            if (!sampleRange(R, kLo, kHi, jLo, jHi))
                                continue;
                            // the checkpoint holds the position at the ray's first sample in
                            // the slab; a brick thinner than the slab advances it to its own
                            // planes
                            float2 cp = cpb[q];
                            if (catchUp) {
                                int jS0, jS1;
                                sampleRange(R, slabLo, slabHi, jS0, jS1);
                                for (int j = jS0; j < jLo; ++j) {
                                    cp.x = __fadd_rn(cp.x, R.sa);
                                    cp.y = __fadd_rn(cp.y, R.sb);
                                }
                            }
                            const int dir = (R.meta & 4) ? -1 : 1;
                            const int t0 = R.k0 + jLo * dir - orgG;
                            axisSplat<TD, UB, TW, TV>(acc, R, yb[q] * R.len, cp, jLo, jHi, t0,
                                                      orgA, orgB);
                        }
                    }
                    __syncwarp();
                }
            }
        }

        // Brick edges of grid G in volume axis order (x, y, z).
        template <int G, int TD, bool UB, int TW, int TV>
        __host__ __device__ constexpr int axisBrickEdge(int axis)
        {
            return axis == G ? TD : (axis == (G == 0 ? 1 : 0) ? (UB ? TV : TW) : (UB ? TW : TV));
        }

        // Shape of the axis bricks (depth along the driving axis, columns, rows) and the
        // checkpoint slab depth of the 3D operator.
        constexpr int kAxisTD = ELSA_AXIS_TD, kAxisTW = ELSA_AXIS_TW, kAxisTV = ELSA_AXIS_TV;
        constexpr int kAxisCheckpointDepth = 16; // the smallest checkpoint slab of the 3D adjoint
        static_assert(kAxisCheckpointDepth % kAxisTD == 0,
                      "axis bricks are a whole fraction of a checkpoint slab deep");

        // What one axis-brick adjoint launch works on: the operator's tables, the sinogram y,
        // the grid's windows and (chunk, partial volume) entries, and where partial volumes go.
        struct AxisJob {
            const JosephRay* rays;
            const float2* checkpoints;
            int64_t nrays;
            const float* y;
            const RayWindow* windows; // this grid's windows, [view][brick]
            const unsigned* viewAxes;
            const int2* chunks; // this grid's entries (chunk, partial volume)
            int entries;
            int viewsPerChunk;
            VolumeShape vol;
            DetectorShape det;
            int m;
            int cpdShift; // checkpoint slabs of 2^cpdShift planes
            int3 nBricks;
            float* out;       // partial volume k at out + k * nvox (x itself for one partial)
            int64_t itemBase; // batched launches: first block of this job
        };

        // One warp: brick bi of grid G, chunk entry e (views [chunks[e].x * per, ...)), written
        // to the entry's partial volume.
        template <int G, int TD, bool UB, int TW, int TV, int CPD>
        __device__ __forceinline__ void axisBrickWork(const AxisJob& J, int bi, int e, float* acc)
        {
            using L = AxisBrick<TD, TW, TV>;
            using AR = AxisRolesAB<TD, UB, TW, TV>;
            constexpr int EX = axisBrickEdge<G, TD, UB, TW, TV>(0);
            constexpr int EY = axisBrickEdge<G, TD, UB, TW, TV>(1);
            constexpr int EZ = axisBrickEdge<G, TD, UB, TW, TV>(2);
            const int lane = threadIdx.x;
            const int3 nBricks = J.nBricks;
            const int org[3] = {(bi % nBricks.x) * EX, ((bi / nBricks.x) % nBricks.y) * EY,
                                (bi / (nBricks.x * nBricks.y)) * EZ};
            int a, b;
            nonDrivingAxes(G, a, b);
            const int orgG = org[G], orgA = org[a], orgB = org[b];
            const int nb = nBricks.x * nBricks.y * nBricks.z;
            for (int i = lane; i < L::kWords; i += 32)
                acc[i] = 0.0f;
            __syncwarp();
            const int2 entry = J.chunks[e];
            const int pBegin = entry.x * J.viewsPerChunk;
            const int pEnd = min(J.det.np, pBegin + J.viewsPerChunk);
            for (int p = pBegin; p < pEnd; ++p) {
                if (!(J.viewAxes[p] & (1u << G)))
                    continue;
                const RayWindow w = J.windows[static_cast<int64_t>(p) * nb + bi];
                if (w.u0 > w.u1 || w.v0 > w.v1)
                    continue;
                axisView<G, TD, UB, TW, TV, CPD>(acc, w, p, J.m, J.cpdShift, J.rays,
                                                 J.checkpoints, J.nrays,
                                                 J.y, J.det, orgG, orgA, orgB);
            }
            __syncwarp();
            const VolumeShape& vol = J.vol;
            const int64_t nvox = static_cast<int64_t>(vol.n[0]) * vol.n[1] * vol.n[2];
            float* dst = J.out + static_cast<int64_t>(entry.y) * nvox;
            for (int i = lane; i < TD * TW * TV; i += 32) {
                // i runs x fastest over the brick's voxels
                const int lx = i % EX, ly = (i / EX) % EY, lz = i / (EX * EY);
                const int gx = org[0] + lx, gy = org[1] + ly, gz = org[2] + lz;
                if (gx < vol.n[0] && gy < vol.n[1] && gz < vol.n[2]) {
                    const int l[3] = {lx, ly, lz};
                    dst[gx + static_cast<int64_t>(vol.n[0]) *
                                 (gy + static_cast<int64_t>(vol.n[1]) * gz)] =
                        acc[AR::kOrigin + l[G] * L::kPlane + l[a] * AR::SA + l[b] * AR::SB];
                }
            }
        }

        // One warp per axis brick of grid G (blockIdx.x) and chunk entry (entryBase +
        // blockIdx.y); blockIdx.z: batch element (sinogram y + b yStride, partial volumes
        // out + b outStride).
        template <int G, int TD, bool UB, int TW, int TV, int CPD>
        __global__ void __launch_bounds__(32, ELSA_ADJ_MIN_BLOCKS)
            josephAdjointAxisKernel(AxisJob J, int entryBase, int64_t yStride, int64_t outStride)
        {
            __shared__ float acc[AxisBrick<TD, TW, TV>::kWords];
            J.y += blockIdx.z * yStride;
            J.out += blockIdx.z * outStride;
            axisBrickWork<G, TD, UB, TW, TV, CPD>(J, blockIdx.x, entryBase + blockIdx.y, acc);
        }

        // Many operators in one launch (batched solves): block k belongs to the job whose
        // [itemBase, itemBase + bricks x entries) holds k; within it, brick k % bricks and entry
        // k / bricks, exactly the work of that operator's own launch.
        template <int G, int TD, bool UB, int TW, int TV, int CPD>
        __global__ void __launch_bounds__(32, ELSA_ADJ_MIN_BLOCKS)
            josephAdjointAxisManyKernel(const AxisJob* __restrict__ jobs, int njobs)
        {
            __shared__ float acc[AxisBrick<TD, TW, TV>::kWords];
            const int64_t k = blockIdx.x;
            int lo = 0, hi = njobs - 1; // last job with itemBase <= k
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (jobs[mid].itemBase <= k)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            const AxisJob J = jobs[lo];
            const int nb = J.nBricks.x * J.nBricks.y * J.nBricks.z;
            const int64_t local = k - J.itemBase;
            axisBrickWork<G, TD, UB, TW, TV, CPD>(J, static_cast<int>(local % nb),
                                                  static_cast<int>(local / nb), acc);
        }

        using Adjoint2d = AdjointConfig<2, 64, 64, 1, 64, 8>;

        class JosephProjector final : public Projector
        {
        public:
            // fast: elsa's unmatched `fast` adjoint (JosephsMethodCUDA.h:60-67) instead of the
            // matched one
            JosephProjector(const VolumeShape& vol, const DetectorShape& det,
                            const std::vector<PoseRecord>& poses, const CurvedDetector& curved,
                            bool fast)
                : Projector(0, vol, det, poses), curved_(vol.dim, det, curved), fast_(fast)
            {
                const int64_t nrays = rangeSize_;
                ELSA_CUDA(cudaMalloc(&dRays_, sizeof(JosephRay) * nrays));
                const int threads = 256;
                const unsigned blocks = static_cast<unsigned>((nrays + threads - 1) / threads);
                josephSetupKernel<<<blocks, threads>>>(dPoses_, vol_, det_, curved_.planar(),
                                                       dRays_);
                ELSA_LAUNCH_CHECK("josephSetupKernel");

                // per-view axis masks, then (at +np) the bad-spacing mask and a 64-bit counter
                const size_t axesWords = static_cast<size_t>(det_.np) + 4;
                ELSA_CUDA(cudaMalloc(&dViewAxes_, sizeof(unsigned) * axesWords));
                ELSA_CUDA(cudaMemset(dViewAxes_, 0, sizeof(unsigned) * axesWords));
                unsigned* dBad = dViewAxes_ + det_.np;
                auto* dCount = reinterpret_cast<unsigned long long*>(
                    dViewAxes_ + ((det_.np + 2) & ~1));
                josephClassCheckKernel<<<blocks, threads>>>(dRays_, det_, vol_.dim, dViewAxes_,
                                                            dBad, dCount);
                ELSA_LAUNCH_CHECK("josephClassCheckKernel");
                unsigned bad = 0;
                unsigned long long count = 0;
                ELSA_CUDA(cudaMemcpy(&bad, dBad, sizeof(unsigned), cudaMemcpyDeviceToHost));
                ELSA_CUDA(cudaMemcpy(&count, dCount, sizeof(count), cudaMemcpyDeviceToHost));
                sampleCount_ = static_cast<int64_t>(count);
                laneAxisBits();
                classSpacing_ = 0;
                for (int m = kMinClass; m <= kMaxClass; ++m)
                    if (!((bad >> m) & 1u)) {
                        classSpacing_ = m;
                        break;
                    }
                if (fast_) {
                    buildFastAdjoint();
                    if (vol_.dim == 3) {
                        std::vector<float> hp(poses_.size() * kPoseFloats);
                        std::memcpy(hp.data(), poses_.data(), sizeof(float) * hp.size());
                        tma_ = std::make_unique<JosephForwardTma>(vol_, det_, hp, dRays_);
                    }
                    ELSA_CUDA(cudaDeviceSynchronize());
                    curved_.release();
                    return;
                }
                if (classSpacing_ == 0)
                    throw Error(ELSA_ERROR_NOT_SUPPORTED,
                                "JosephsMethod: neighbouring detector rays pass within two voxels "
                                "of each other even eight pixels apart; the atomic-free adjoint "
                                "needs a coarser detector");

                int cpd;
                if (vol_.dim == 3) {
                    cpd = defaultCheckpointDepth();
                } else {
                    brick_ = Adjoint2d::brick();
                    cpd = Adjoint2d::kCheckpointDepth;
                    Adjoint2d::prepare(det_.np);
                }
                buildCheckpoints(cpd);

                if (vol_.dim == 3) {
                    buildAxisGrids();
                } else {
                    nBricks_ = make_int3((vol_.n[0] + brick_.x - 1) / brick_.x,
                                         (vol_.n[1] + brick_.y - 1) / brick_.y,
                                         (vol_.n[2] + brick_.z - 1) / brick_.z);
                    const int64_t nwin =
                        static_cast<int64_t>(nBricks_.x) * nBricks_.y * nBricks_.z * det_.np;
                    ELSA_CUDA(cudaMalloc(&dWindows_, sizeof(RayWindow) * nwin));
                    josephWindowKernel<<<static_cast<unsigned>((nwin + 255) / 256), 256>>>(
                        dPoses_, vol_, det_, brick_, nBricks_, curved_.map(), windowGrow(vol_),
                        kWindowPixelMargin, dWindows_);
                    ELSA_LAUNCH_CHECK("josephWindowKernel");
                }
                setKnob(kKnobAdjointChunks, defaultChunks());
                if (vol_.dim == 3) {
                    std::vector<float> hp(poses_.size() * kPoseFloats);
                    std::memcpy(hp.data(), poses_.data(), sizeof(float) * hp.size());
                    tma_ = std::make_unique<JosephForwardTma>(vol_, det_, hp, dRays_);
                }
                ELSA_CUDA(cudaDeviceSynchronize());
                curved_.release(); // rays and windows are built
            }

            // Per view and driving axis g: set bit 4+g of the view's axis word when neighbouring
            // pixels of a detector row spread along the second non-driving axis b on the planes
            // of g (centre pixel and its right neighbour).
            void laneAxisBits()
            {
                std::vector<unsigned> axes(det_.np);
                ELSA_CUDA(cudaMemcpy(axes.data(), dViewAxes_, sizeof(unsigned) * det_.np,
                                     cudaMemcpyDeviceToHost));
                for (int p = 0; p < det_.np; ++p) {
                    const float* P = poses_[p].v + kPoseOffPinv;
                    const int d = vol_.dim;
                    const float uc = det_.nu / 2 + 0.5f, vc = det_.nv / 2 + 0.5f;
                    float D[3] = {0, 0, 0}, E[3] = {0, 0, 0};
                    for (int i = 0; i < d; ++i) {
                        if (d == 3) {
                            D[i] = P[i * 3] * uc + P[i * 3 + 1] * vc + P[i * 3 + 2];
                            E[i] = P[i * 3] * (uc + 1.0f) + P[i * 3 + 1] * vc + P[i * 3 + 2];
                        } else {
                            D[i] = P[i * 2] * uc + P[i * 2 + 1];
                            E[i] = P[i * 2] * (uc + 1.0f) + P[i * 2 + 1];
                        }
                    }
                    if (d == 3) {
                        for (int g = 0; g < 3; ++g) {
                            int a, b;
                            nonDrivingAxes(g, a, b);
                            if (std::fabs(D[g]) == 0.0f || std::fabs(E[g]) == 0.0f)
                                continue;
                            const float da =
                                std::fabs(E[a] / std::fabs(E[g]) - D[a] / std::fabs(D[g]));
                            const float db =
                                std::fabs(E[b] / std::fabs(E[g]) - D[b] / std::fabs(D[g]));
                            if (db > da)
                                axes[p] |= 16u << g;
                        }
                    }
                }
                ELSA_CUDA(cudaMemcpy(dViewAxes_, axes.data(), sizeof(unsigned) * det_.np,
                                     cudaMemcpyHostToDevice));
            }

            // The fast adjoint's per-view table (leading block of P, column-major, and the ray
            // origin -Binv p4 as JosephsMethodCUDA.cpp:80-84 computes it, in float, k-sums in
            // order) and the layered sinogram array it reads through a texture.
            void buildFastAdjoint()
            {
                const int d = vol_.dim;
                const int kT = d == 3 ? 12 : 6;
                std::vector<float> table(static_cast<size_t>(kT) * det_.np);
                for (int p = 0; p < det_.np; ++p) {
                    const float* P = poses_[p].v;
                    const float* Pinv = poses_[p].v + kPoseOffPinv;
                    float* T = table.data() + static_cast<size_t>(kT) * p;
                    for (int c = 0; c < d; ++c)
                        for (int r = 0; r < d; ++r)
                            T[d * c + r] = P[(d + 1) * r + c];
                    for (int r = 0; r < d; ++r) {
                        float s = 0.0f;
                        for (int c = 0; c < d; ++c)
                            s += Pinv[d * r + c] * P[(d + 1) * c + d];
                        T[d * d + r] = -s;
                    }
                }
                // the kernel keeps the table in shared memory; the limit attribute only grows, as
                // for the brick-owner adjoints (shared by every projector of the process)
                const int need = static_cast<int>(sizeof(float) * table.size());
                if (need > 227 * 1024)
                    throw Error(ELSA_ERROR_NOT_SUPPORTED,
                                "JosephsMethodCUDA: too many poses for the fast adjoint");
                {
                    static std::mutex mu;
                    std::lock_guard<std::mutex> lock(mu);
                    cudaFuncAttributes attr{};
                    const void* fn = d == 3 ? reinterpret_cast<const void*>(
                                                  josephFastAdjointKernel<3>)
                                            : reinterpret_cast<const void*>(
                                                  josephFastAdjointKernel<2>);
                    ELSA_CUDA(cudaFuncGetAttributes(&attr, fn));
                    if (need > attr.maxDynamicSharedSizeBytes)
                        ELSA_CUDA(cudaFuncSetAttribute(
                            fn, cudaFuncAttributeMaxDynamicSharedMemorySize, need));
                }
                fastTable_ = std::make_unique<DeviceBuffer>(sizeof(float) * table.size());
                ELSA_CUDA(cudaMemcpy(fastTable_->as<float>(), table.data(),
                                     sizeof(float) * table.size(), cudaMemcpyHostToDevice));
                cudaDeviceProp prop{};
                ELSA_CUDA(cudaGetDeviceProperties(&prop, device_));
                const int* lim = d == 3 ? prop.maxTexture2DLayered : prop.maxTexture1DLayered;
                if (det_.nu > lim[0] || (d == 3 && det_.nv > lim[1]) || det_.np > lim[d - 1])
                    throw Error(ELSA_ERROR_NOT_SUPPORTED,
                                "JosephsMethodCUDA: the fast adjoint's layered texture cannot "
                                "hold this detector (size or number of poses)");
                const cudaChannelFormatDesc fd =
                    cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat);
                const cudaExtent ext =
                    make_cudaExtent(det_.nu, d == 3 ? det_.nv : 0, det_.np);
                ELSA_CUDA(cudaMalloc3DArray(&fastArray_, &fd, ext, cudaArrayLayered));
                cudaResourceDesc res;
                std::memset(&res, 0, sizeof(res));
                res.resType = cudaResourceTypeArray;
                res.res.array.array = fastArray_;
                cudaTextureDesc tex;
                std::memset(&tex, 0, sizeof(tex));
                tex.addressMode[0] = tex.addressMode[1] = tex.addressMode[2] =
                    cudaAddressModeBorder;
                tex.filterMode = cudaFilterModeLinear;
                tex.readMode = cudaReadModeElementType;
                tex.normalizedCoords = 0;
                ELSA_CUDA(cudaCreateTextureObject(&fastTex_, &res, &tex, nullptr));
            }

            ~JosephProjector() override
            {
                if (fastTex_)
                    cudaDestroyTextureObject(fastTex_);
                if (fastArray_)
                    cudaFreeArray(fastArray_);
                cudaFree(dRays_);
                cudaFree(dViewAxes_);
                cudaFree(dWindows_);
                cudaFree(dCheckpoints_);
            }

            void forward(const float* x, float* y, cudaStream_t s) override
            {
                const int64_t nrays = rangeSize_;
                const unsigned blocks =
                    static_cast<unsigned>((nrays + forwardThreads_ - 1) / forwardThreads_);
                if (tma_)
                    tma_->forward(x, y, s);
                else if (vol_.dim == 3)
                    josephForwardKernel<3><<<blocks, forwardThreads_, 0, s>>>(dRays_, nrays, x,
                                                                                vol_, y);
                else
                    josephForwardKernel<2><<<blocks, forwardThreads_, 0, s>>>(dRays_, nrays, x,
                                                                                vol_, y);
                ELSA_LAUNCH_CHECK("josephForwardKernel");
            }

            void adjoint(const float* y, float* x, cudaStream_t s) override
            {
                if (fast_) {
                    // the sinogram into the layered array (JosephsMethodCUDA.cpp:234-240 copies
                    // the host data there on every call)
                    const int d = vol_.dim;
                    cudaMemcpy3DParms prm = {};
                    prm.srcPtr = make_cudaPitchedPtr(const_cast<float*>(y), sizeof(float) * det_.nu,
                                                     det_.nu, d == 3 ? det_.nv : 1);
                    prm.dstArray = fastArray_;
                    prm.extent = make_cudaExtent(det_.nu, d == 3 ? det_.nv : 1, det_.np);
                    prm.kind = cudaMemcpyDeviceToDevice;
                    ELSA_CUDA(cudaMemcpy3DAsync(&prm, s));
                    const int64_t rows =
                        static_cast<int64_t>(vol_.n[1]) * (d == 3 ? vol_.n[2] : 1);
                    const dim3 grid(static_cast<unsigned>((rows + kFastRows - 1) / kFastRows));
                    const dim3 block(32, kFastRows);
                    const size_t smem = sizeof(float) * (d == 3 ? 12 : 6) * det_.np;
                    if (d == 3)
                        josephFastAdjointKernel<3><<<grid, block, smem, s>>>(
                            fastTex_, fastTable_->as<float>(), det_.np, vol_, x);
                    else
                        josephFastAdjointKernel<2><<<grid, block, smem, s>>>(
                            fastTex_, fastTable_->as<float>(), det_.np, vol_, x);
                    ELSA_LAUNCH_CHECK("josephFastAdjointKernel");
                    return;
                }
                if (scatter_) {
                    const int64_t nrays = rangeSize_;
                    const unsigned blocks =
                        static_cast<unsigned>((nrays + kForwardThreads - 1) / kForwardThreads);
                    ELSA_CUDA(cudaMemsetAsync(x, 0, sizeof(float) * domainSize_, s));
                    if (vol_.dim == 3)
                        josephScatterKernel<3><<<blocks, kForwardThreads, 0, s>>>(dRays_, nrays, y,
                                                                                 vol_, x);
                    else
                        josephScatterKernel<2><<<blocks, kForwardThreads, 0, s>>>(dRays_, nrays, y,
                                                                                 vol_, x);
                    ELSA_LAUNCH_CHECK("josephScatterKernel");
                    return;
                }
                if (vol_.dim == 3) {
                    const int used = usedChunks();
                    float* out = axisPartials_ > 1 ? partial_->as<float>() : x;
                    launchAxisChunks(0, used, y, out, s);
                    if (axisPartials_ > 1)
                        launchSumChunks(partial_->as<float>(), axisPartials_, domainSize_, x, s);
                    return;
                }
                const int nb = nBricks_.x * nBricks_.y * nBricks_.z;
                float* partial = partial_ ? partial_->as<float>() : nullptr;
                Adjoint2d::launch(nb, adjointChunks_, s, dRays_, dCheckpoints_, rangeSize_, y,
                                  dWindows_, dViewAxes_, vol_, det_, classSpacing_, nBricks_, x,
                                  partial);
                ELSA_LAUNCH_CHECK("josephAdjointKernel");
            }

            // Batched applies (3D matched operator): one launch per kernel for all volumes,
            // sharing the ray tables; every batch element is computed exactly as by a single
            // apply (same kernels, chunks and summation order).
            void forwardBatch(const float* x, int64_t xs, float* y, int64_t ys, int batch,
                              cudaStream_t s) override
            {
                if (!tma_) {
                    Projector::forwardBatch(x, xs, y, ys, batch, s);
                    return;
                }
                tma_->forwardBatch(x, xs, y, ys, batch, s);
            }
            void adjointBatch(const float* y, int64_t ys, float* x, int64_t xs, int batch,
                              cudaStream_t s) override
            {
                if (batch <= 0)
                    return;
                if (fast_ || scatter_ || vol_.dim != 3) {
                    Projector::adjointBatch(y, ys, x, xs, batch, s);
                    return;
                }
                const int used = usedChunks();
                if (axisPartials_ <= 1) {
                    launchAxisChunks(0, used, y, x, s, batch, ys, xs);
                    return;
                }
                // partial volumes for as many batch elements as fit in kBatchPartialMemory
                const int64_t perElem = static_cast<int64_t>(axisPartials_) * domainSize_;
                const int fit = static_cast<int>(std::max<int64_t>(
                    1, std::min<int64_t>(batch, kBatchPartialMemory / (4 * perElem))));
                const size_t need = sizeof(float) * static_cast<size_t>(perElem) * fit;
                if (partial_->bytes() < need) {
                    ELSA_CUDA(cudaStreamSynchronize(s)); // no launch in flight reads the old one
                    ELSA_CUDA(cudaDeviceSynchronize());
                    partial_.reset();
                    partial_ = std::make_unique<DeviceBuffer>(need);
                }
                for (int b0 = 0; b0 < batch; b0 += fit) {
                    const int nb = std::min(fit, batch - b0);
                    launchAxisChunks(0, used, y + b0 * ys, partial_->as<float>(), s, nb, ys,
                                     perElem);
                    for (int b = 0; b < nb; ++b)
                        launchSumChunks(partial_->as<float>() + b * perElem, axisPartials_,
                                        domainSize_, x + (b0 + b) * xs, s);
                }
            }

            // Host-buffer pipelining: kHostGroups groups of views for the TMA forward; for the
            // chunked 3D brick-owner adjoint, groups of whole view chunks. Only the copy of the
            // forward's last group and of the adjoint's first group are not overlapped with a
            // kernel, so those groups are small: the forward's groups hold 30/30/30/10 % of
            // the views, the adjoint's first group one view chunk and the rest thirds.
            static constexpr int kHostGroups = 4;
            int forwardGroups() const override
            {
                return tma_ && det_.np >= 10 ? kHostGroups : 0;
            }
            std::pair<int, int> forwardGroupViews(int g, int G) const override
            {
                static constexpr int kEnd[kHostGroups + 1] = {0, 30, 60, 90, 100};
                (void)G;
                return {static_cast<int>(static_cast<int64_t>(det_.np) * kEnd[g] / 100),
                        static_cast<int>(static_cast<int64_t>(det_.np) * kEnd[g + 1] / 100)};
            }
            // first chunk of adjoint group g (g = 0 .. kHostGroups)
            int groupChunk(int g) const
            {
                const int used = usedChunks();
                if (g == 0)
                    return 0;
                return 1 + static_cast<int>(static_cast<int64_t>(used - 1) * (g - 1) /
                                            (kHostGroups - 1));
            }
            void prepareForward(const float* x, cudaStream_t s) override { tma_->prepare(x, s); }
            void forwardGroup(const float* x, float* y, int g, int G, cudaStream_t s) override
            {
                const auto v = forwardGroupViews(g, G);
                tma_->forwardViews(x, y, v.first, v.second, s);
            }
            int usedChunks() const
            {
                const int per = (det_.np + adjointChunks_ - 1) / adjointChunks_;
                return (det_.np + per - 1) / per;
            }
            int adjointGroups() const override
            {
                if (fast_ || scatter_ || vol_.dim != 3 || axisPartials_ <= 1)
                    return 0;
                return usedChunks() >= kHostGroups ? kHostGroups : 0;
            }
            std::pair<int, int> adjointGroupViews(int g, int G) const override
            {
                (void)G;
                const int per = (det_.np + adjointChunks_ - 1) / adjointChunks_;
                return {std::min(det_.np, groupChunk(g) * per),
                        std::min(det_.np, groupChunk(g + 1) * per)};
            }
            void adjointGroup(const float* y, int g, int G, cudaStream_t s) override
            {
                (void)G;
                launchAxisChunks(groupChunk(g), groupChunk(g + 1), y, partial_->as<float>(), s);
            }
            void adjointFinish(float* x, cudaStream_t s) override
            {
                launchSumChunks(partial_->as<float>(), axisPartials_, domainSize_, x, s);
            }

            std::vector<int> knobCandidates(int knob) const override
            {
                if (fast_ && knob != kKnobForwardThreads)
                    return {}; // the fast adjoint has no adjoint knobs
                if (knob == kKnobAdjointChunks) {
                    // partial volumes limited to 4 GiB
                    const int64_t byMemory =
                        std::max<int64_t>(1, (int64_t(1) << 32) / (4 * domainSize_));
                    const int limit = static_cast<int>(
                        std::min<int64_t>(std::min<int64_t>(det_.np, 256), byMemory));
                    return chunkCandidates(limit, std::min(limit, defaultChunks()));
                }
                if (knob == kKnobForwardThreads && !tma_)
                    return {64, 128, 256, 512};
                if (knob == kKnobAdjointScatter)
                    return {0, 1};
                if (knob == kKnobCheckpointDepth && vol_.dim == 3) {
                    // depths whose table takes at most an eighth of the device's memory, and
                    // the current one
                    size_t freeBytes = 0, totalBytes = 0;
                    ELSA_CUDA(cudaMemGetInfo(&freeBytes, &totalBytes));
                    const int maxDim = std::max(vol_.n[0], std::max(vol_.n[1], vol_.n[2]));
                    std::vector<int> c;
                    for (int cpd = kAxisCheckpointDepth; cpd <= 128; cpd *= 2)
                        if (cpd == (1 << cpdShift_) ||
                            8.0 * static_cast<double>(rangeSize_) * (maxDim / cpd + 3) <=
                                static_cast<double>(totalBytes) / 8.0)
                            c.push_back(cpd);
                    return c;
                }
                return {};
            }

            int knob(int knob) const override
            {
                if (knob == kKnobCheckpointDepth)
                    return vol_.dim == 3 && !fast_ ? 1 << cpdShift_ : -1;
                if (knob == kKnobAdjointChunks)
                    return adjointChunks_;
                if (knob == kKnobForwardThreads)
                    return tma_ ? -1 : forwardThreads_;
                if (knob == kKnobAdjointScatter)
                    return scatter_;
                return -1;
            }

            void setKnob(int knob, int value) override
            {
                const std::vector<int> c = knobCandidates(knob);
                if (knob == kKnobAdjointChunks && value == defaultChunks()) {
                    // the default is always allowed, also past the tuning limits
                } else if (std::find(c.begin(), c.end(), value) == c.end()) {
                    throw Error(ELSA_ERROR_INVALID_ARGUMENT,
                                "JosephsMethod: value " + std::to_string(value) +
                                    " is not a candidate of knob " + std::to_string(knob));
                }
                if (batchRefs_.load() > 0 && knob != kKnobForwardThreads)
                    throw Error(ELSA_ERROR_INVALID_ARGUMENT,
                                "JosephsMethod: a batched solver holds this operator's adjoint "
                                "tables; destroy it before changing an adjoint knob");
                if (knob == kKnobForwardThreads) {
                    forwardThreads_ = value;
                    return;
                }
                if (knob == kKnobAdjointScatter) {
                    scatter_ = value;
                    return;
                }
                if (knob == kKnobCheckpointDepth) {
                    buildCheckpoints(value);
                    return;
                }
                adjointChunks_ = value;
                const int volumes = vol_.dim == 3 ? buildAxisEntries() : value;
                const size_t need = sizeof(float) * static_cast<size_t>(domainSize_) *
                                    static_cast<size_t>(volumes);
                if (volumes <= 1)
                    partial_.reset();
                else if (!partial_ || partial_->bytes() < need) {
                    partial_.reset();
                    partial_ = std::make_unique<DeviceBuffer>(need);
                }
            }

            // Checkpoint slab depth of the 3D adjoint by default: the smallest of 16, 32, 64, 128
            // planes whose table (8 bytes per ray and slab) takes at most an eighth of the
            // device's memory (256^3 / 360 x 384^2: 16 planes, 8.1 GB; 512^3 / 720 x 768^2: 128
            // planes, 15 GB instead of 119 GB). Deeper slabs cost catch-up additions from the
            // slab's checkpoint to a brick's first plane; the results are the same.
            int defaultCheckpointDepth() const
            {
                size_t freeBytes = 0, totalBytes = 0;
                ELSA_CUDA(cudaMemGetInfo(&freeBytes, &totalBytes));
                const int maxDim = std::max(vol_.n[0], std::max(vol_.n[1], vol_.n[2]));
                int cpd = kAxisCheckpointDepth;
                while (cpd < 128 && 8.0 * static_cast<double>(rangeSize_) * (maxDim / cpd + 3) >
                                        static_cast<double>(totalBytes) / 8.0)
                    cpd *= 2;
                return cpd;
            }

            // (Re)builds the slab checkpoints for slabs of cpd planes.
            void buildCheckpoints(int cpd)
            {
                if (dCheckpoints_ != nullptr) {
                    ELSA_CUDA(cudaDeviceSynchronize()); // no adjoint may still read the table
                    ELSA_CUDA(cudaFree(dCheckpoints_));
                    dCheckpoints_ = nullptr;
                }
                int shift = 0;
                while ((1 << shift) < cpd)
                    ++shift;
                cpdShift_ = shift;
                const int maxDim = std::max(vol_.n[0], std::max(vol_.n[1], vol_.n[2]));
                const int64_t nrays = rangeSize_;
                cpStride_ = maxDim / cpd + 3;
                ELSA_CUDA(cudaMalloc(&dCheckpoints_, sizeof(float2) * nrays * cpStride_));
                const unsigned blocks = static_cast<unsigned>((nrays + 255) / 256);
                josephCheckpointKernel<<<blocks, 256>>>(dRays_, nrays, cpd, cpStride_,
                                                        dCheckpoints_);
                ELSA_LAUNCH_CHECK("josephCheckpointKernel");
            }

            bool setWaitTest(long long cycles, bool withhold) override
            {
                if (!tma_)
                    return false;
                tma_->setWaitTest(cycles, withhold);
                return true;
            }

            int64_t info(int key) const override
            {
                switch (key) {
                case 0:
                    return classSpacing_;
                case 1: // bricks of the matched adjoint (3D: over the axis grids)
                    if (vol_.dim == 3) {
                        int64_t n = 0;
                        for (const AxisGrid& g : grids_)
                            if (g.present)
                                n += static_cast<int64_t>(g.nb.x) * g.nb.y * g.nb.z;
                        return n;
                    }
                    return nBricks_.x * nBricks_.y * nBricks_.z;
                case 2:
                    return sampleCount_;
                case 3: // error word of the TMA forward (synchronizes)
                    return tma_ ? static_cast<int64_t>(tma_->errorWord()) : 0;
                case 4: // parts per million of detector tiles on the gather fallback
                    return tma_ ? static_cast<int64_t>(tma_->fallbackFraction() * 1e6) : -1;
                case 6: // kernel launches per forward call
                    return tma_ ? tma_->launchesPerForward() : 1;
                case 7: // kernel launches per adjoint call (3D: one per axis grid; with
                        // several partial volumes: + the chunk sum)
                    if (fast_ || scatter_)
                        return 1;
                    if (vol_.dim == 3) {
                        int n = 0;
                        for (const AxisGrid& g : grids_)
                            n += g.present && g.entryEnd > g.entryBegin ? 1 : 0;
                        return n + (axisPartials_ > 1 ? 1 : 0);
                    }
                    return adjointChunks_ > 1 ? 2 : 1;
                case 8: // taps outside the windows of their bricks (test support; synchronizes)
                    return windowMisses();
                default:
                    return -1;
                }
            }

        private:
            int64_t windowMisses() const
            {
                if (fast_ || (vol_.dim == 2 && !dWindows_))
                    return -1;
                DeviceBuffer count(sizeof(unsigned long long));
                ELSA_CUDA(cudaMemset(count.as<unsigned long long>(), 0, sizeof(unsigned long long)));
                const int64_t nrays = rangeSize_;
                const unsigned blocks = static_cast<unsigned>((nrays + 255) / 256);
                if (vol_.dim == 3) {
                    for (int g = 0; g < 3; ++g)
                        if (grids_[g].present)
                            josephWindowCheckKernel<<<blocks, 256>>>(
                                dRays_, grids_[g].windows->as<RayWindow>(), vol_, det_,
                                grids_[g].edge, grids_[g].nb, g, count.as<unsigned long long>());
                } else {
                    josephWindowCheckKernel<<<blocks, 256>>>(dRays_, dWindows_, vol_, det_,
                                                             brick_, nBricks_, -1,
                                                             count.as<unsigned long long>());
                }
                ELSA_LAUNCH_CHECK("josephWindowCheckKernel");
                unsigned long long h = 0;
                ELSA_CUDA(cudaMemcpy(&h, count.as<unsigned long long>(), sizeof(h),
                                     cudaMemcpyDeviceToHost));
                return static_cast<int64_t>(h);
            }

            bool fast_ = false; // elsa's unmatched fast adjoint
            cudaArray_t fastArray_ = nullptr;
            cudaTextureObject_t fastTex_ = 0;
            std::unique_ptr<DeviceBuffer> fastTable_;
            int scatter_ = 0; // 1: atomic scatter adjoint (2D: 512^2 / 720 views 1.74 ms
                              // against 2.00; 3D 256^3 / 360 views 92 ms against 54.8)
            JosephRay* dRays_ = nullptr;
            unsigned* dViewAxes_ = nullptr;
            RayWindow* dWindows_ = nullptr;
            float2* dCheckpoints_ = nullptr;
            int cpStride_ = 0;
            int cpdShift_ = 4; // checkpoint slabs of 2^cpdShift_ planes (3D)

        public:
            // batched adjoint plans holding pointers into this operator's tables
            mutable std::atomic<int> batchRefs_{0};

        private:
            int classSpacing_ = 0;
            int64_t sampleCount_ = 0;
            std::unique_ptr<JosephForwardTma> tma_;
            CurvedTables curved_; // curved detector coordinates while the rays are set up
            std::unique_ptr<DeviceBuffer> partial_; // adjoint: per view-chunk partial volumes
            int adjointChunks_ = 1;                 // view chunks of the adjoint
            int forwardThreads_ = kForwardThreads;  // rays per block of the gather forward

            // View chunks of the adjoint: enough for bricks x chunks to fill the GPU (see the
            // launch configs) and at least kMinAdjointChunks, within kChunkMemory of partial
            // volumes. Finer chunks also balance bricks of uneven work: at 256^3 / 360 views
            // the adjoint takes 63.4 ms with 1 chunk, 55.5 with 8 and 54.8 with 16-32.
            int defaultChunks() const
            {
                int fill;
                if (vol_.dim == 2) {
                    fill = Adjoint2d::chunks(nBricks_.x * nBricks_.y * nBricks_.z, det_.np);
                } else {
                    // bricks x chunks of the smallest present grid reach kAdjoint3dWarpsPerSm
                    // one-warp CTAs per SM (each grid sees about its share of the views)
                    int64_t nb = 0;
                    for (const AxisGrid& g : grids_)
                        if (g.present)
                            nb = std::max<int64_t>(nb, static_cast<int64_t>(g.nb.x) * g.nb.y *
                                                           g.nb.z);
                    const int64_t want = (kAdjoint3dWarpsPerSm * 148 + nb - 1) / std::max<int64_t>(nb, 1);
                    fill = static_cast<int>(std::min<int64_t>(det_.np, std::max<int64_t>(1, want)));
                }
                // partial volumes within kChunkMemory: the 3D adjoint writes one per (chunk,
                // axis grid) pair, so leave room for the chunks whose views drive along two axes
                const int64_t cap = std::max<int64_t>(1, kChunkMemory / (4 * domainSize_));
                const int64_t capChunks = vol_.dim == 3 ? std::max<int64_t>(1, cap * 7 / 8) : cap;
                return static_cast<int>(std::min<int64_t>(
                    std::min<int64_t>(det_.np, capChunks), std::max(fill, kMinAdjointChunks)));
            }

            // ---- 3D matched adjoint on axis bricks ----

            struct AxisGrid {
                bool present = false;
                bool ub = false;   // columns (the wide, stride-1 edge) along b instead of a
                int3 edge{}, nb{}; // brick edges and brick counts in volume axis order
                std::unique_ptr<DeviceBuffer> windows; // [view][brick]
                int entryBegin = 0, entryEnd = 0;      // this grid's (chunk, partial) entries
            };
            AxisGrid grids_[3];
            std::vector<unsigned> viewAxesHost_;
            std::vector<int2> entries_;                 // (chunk, partial volume), grid-major
            std::unique_ptr<DeviceBuffer> dEntries_;
            int axisPartials_ = 0;                      // partial volumes of the 3D adjoint

            static int3 axisEdge(int g, bool ub)
            {
                int a, b;
                nonDrivingAxes(g, a, b);
                int e[3];
                e[g] = kAxisTD;
                e[a] = ub ? kAxisTV : kAxisTW;
                e[b] = ub ? kAxisTW : kAxisTV;
                return make_int3(e[0], e[1], e[2]);
            }

            // Brick grids and windows for every driving axis of the geometry.
            void buildAxisGrids()
            {
                viewAxesHost_.resize(det_.np);
                ELSA_CUDA(cudaMemcpy(viewAxesHost_.data(), dViewAxes_, sizeof(unsigned) * det_.np,
                                     cudaMemcpyDeviceToHost));
                for (int g = 0; g < 3; ++g) {
                    AxisGrid& G = grids_[g];
                    G.present = std::any_of(viewAxesHost_.begin(), viewAxesHost_.end(),
                                            [g](unsigned a) { return (a >> g) & 1u; });
                    if (!G.present)
                        continue;
                    // columns along the axis over which a detector row's rays spread, by a vote
                    // of the views driving along g (bit 4+g of a view's axis word: along b)
                    int alongB = 0, votes = 0;
                    for (unsigned w : viewAxesHost_)
                        if ((w >> g) & 1u) {
                            ++votes;
                            alongB += (w >> (4 + g)) & 1u;
                        }
                    G.ub = 2 * alongB > votes;
                    G.edge = axisEdge(g, G.ub);
                    G.nb = make_int3((vol_.n[0] + G.edge.x - 1) / G.edge.x,
                                     (vol_.n[1] + G.edge.y - 1) / G.edge.y,
                                     (vol_.n[2] + G.edge.z - 1) / G.edge.z);
                    const int64_t nwin = static_cast<int64_t>(G.nb.x) * G.nb.y * G.nb.z * det_.np;
                    G.windows = std::make_unique<DeviceBuffer>(sizeof(RayWindow) * nwin);
                    josephWindowKernel<<<static_cast<unsigned>((nwin + 255) / 256), 256>>>(
                        dPoses_, vol_, det_, G.edge, G.nb, curved_.map(), windowGrow(vol_),
                        kWindowPixelMargin, G.windows->as<RayWindow>());
                    ELSA_LAUNCH_CHECK("josephWindowKernel");
                }
            }

            // (chunk, partial volume) entries of every grid for adjointChunks_ view chunks: chunk
            // c covers views [c per, (c + 1) per); a grid takes the chunks holding a view that
            // drives along its axis. Partial volumes are numbered by (chunk, axis), the order in
            // which the chunk sum adds them. Returns the number of partial volumes.
            int buildAxisEntries()
            {
                const int per = (det_.np + adjointChunks_ - 1) / adjointChunks_;
                const int used = (det_.np + per - 1) / per;
                std::vector<std::vector<int2>> byGrid(3);
                int next = 0;
                for (int c = 0; c < used; ++c) {
                    for (int g = 0; g < 3; ++g) {
                        if (!grids_[g].present)
                            continue;
                        bool any = false;
                        for (int p = c * per; p < std::min(det_.np, (c + 1) * per) && !any; ++p)
                            any = (viewAxesHost_[p] >> g) & 1u;
                        if (any)
                            byGrid[g].push_back(make_int2(c, next++));
                    }
                }
                entries_.clear();
                for (int g = 0; g < 3; ++g) {
                    grids_[g].entryBegin = static_cast<int>(entries_.size());
                    entries_.insert(entries_.end(), byGrid[g].begin(), byGrid[g].end());
                    grids_[g].entryEnd = static_cast<int>(entries_.size());
                }
                if (next == 1) // one partial: the kernel writes x itself
                    for (auto& e : entries_)
                        e.y = 0;
                dEntries_ = std::make_unique<DeviceBuffer>(sizeof(int2) * std::max<size_t>(1, entries_.size()));
                if (!entries_.empty())
                    ELSA_CUDA(cudaMemcpy(dEntries_->as<int2>(), entries_.data(),
                                         sizeof(int2) * entries_.size(), cudaMemcpyHostToDevice));
                axisPartials_ = next;
                return next;
            }

        public:
            // This operator's share of a batched adjoint (planJosephAdjointMany): its axis-brick
            // jobs keyed by (grid, column axis), and its chunk sum (chunks <= 1: none).
            bool batchable() const
            {
                return vol_.dim == 3 && !fast_ && !scatter_ && dCheckpoints_ != nullptr;
            }
            void appendAxisJobs(const float* y, float* x, std::vector<AxisJob> (&jobs)[6],
                                std::vector<SumChunksEntry>& sums) const
            {
                float* out = axisPartials_ > 1 ? partial_->as<float>() : x;
                for (int g = 0; g < 3; ++g) {
                    const AxisGrid& G = grids_[g];
                    if (!G.present || G.entryEnd <= G.entryBegin)
                        continue;
                    jobs[2 * g + (G.ub ? 1 : 0)].push_back(axisJob(g, y, out));
                }
                if (axisPartials_ > 1)
                    sums.push_back(SumChunksEntry{partial_->as<float>(), axisPartials_,
                                                  domainSize_, x});
            }

        private:
            // The axis-brick job of grid g on sinogram y into out (entries indexed from the grid's
            // first entry; itemBase left to batched callers).
            AxisJob axisJob(int g, const float* y, float* out) const
            {
                const AxisGrid& G = grids_[g];
                AxisJob J{};
                J.rays = dRays_;
                J.checkpoints = dCheckpoints_;
                J.nrays = rangeSize_;
                J.y = y;
                J.windows = G.windows->as<RayWindow>();
                J.viewAxes = dViewAxes_;
                J.chunks = dEntries_->as<int2>() + G.entryBegin;
                J.entries = G.entryEnd - G.entryBegin;
                J.viewsPerChunk = (det_.np + adjointChunks_ - 1) / adjointChunks_;
                J.vol = vol_;
                J.det = det_;
                J.m = classSpacing_;
                J.cpdShift = cpdShift_;
                J.nBricks = G.nb;
                J.out = out;
                J.itemBase = 0;
                return J;
            }

            // The axis-brick kernels for view chunks [c0, c1), writing their partial volumes into
            // out (x itself when there is a single partial volume); `batch` sinograms
            // y + b yStride into out + b outStride.
            void launchAxisChunks(int c0, int c1, const float* y, float* out, cudaStream_t s,
                                  int batch = 1, int64_t yStride = 0, int64_t outStride = 0)
            {
                for (int g = 0; g < 3; ++g) {
                    const AxisGrid& G = grids_[g];
                    if (!G.present)
                        continue;
                    int e0 = G.entryBegin, e1 = G.entryBegin;
                    for (int e = G.entryBegin; e < G.entryEnd; ++e) {
                        if (entries_[e].x < c0)
                            e0 = e + 1;
                        if (entries_[e].x < c1)
                            e1 = e + 1;
                    }
                    if (e1 <= e0)
                        continue;
                    const dim3 grid(static_cast<unsigned>(G.nb.x * G.nb.y * G.nb.z),
                                    static_cast<unsigned>(e1 - e0), static_cast<unsigned>(batch));
                    const AxisJob J = axisJob(g, y, out);
                    // slabs of kAxisCheckpointDepth planes: the depth fixed at compile time;
                    // deeper ones (CPD 0): read from the job
                    const bool deep = (1 << cpdShift_) != kAxisCheckpointDepth;
#define ELSA_AXIS_LAUNCH(G_, UB_)                                                                \
    do {                                                                                         \
        if (deep)                                                                                \
            josephAdjointAxisKernel<G_, kAxisTD, UB_, kAxisTW, kAxisTV, 0>                       \
                <<<grid, 32, 0, s>>>(J, e0 - G.entryBegin, yStride, outStride);                  \
        else                                                                                     \
            josephAdjointAxisKernel<G_, kAxisTD, UB_, kAxisTW, kAxisTV, kAxisCheckpointDepth>     \
                <<<grid, 32, 0, s>>>(J, e0 - G.entryBegin, yStride, outStride);                  \
    } while (0)
                    if (g == 0) {
                        if (G.ub)
                            ELSA_AXIS_LAUNCH(0, true);
                        else
                            ELSA_AXIS_LAUNCH(0, false);
                    } else if (g == 1) {
                        if (G.ub)
                            ELSA_AXIS_LAUNCH(1, true);
                        else
                            ELSA_AXIS_LAUNCH(1, false);
                    } else {
                        if (G.ub)
                            ELSA_AXIS_LAUNCH(2, true);
                        else
                            ELSA_AXIS_LAUNCH(2, false);
                    }
#undef ELSA_AXIS_LAUNCH
                    ELSA_LAUNCH_CHECK("josephAdjointAxisKernel");
                }
            }

            int3 brick_{}, nBricks_{};
        };
    } // namespace

    void launchBrickWindows(const float* poses, const VolumeShape& vol, const DetectorShape& det,
                            int3 brick, int3 nBricks, RayWindow* out, cudaStream_t s,
                            CurvedMap cm, float grow, float pixMargin)
    {
        const int64_t nwin = static_cast<int64_t>(nBricks.x) * nBricks.y * nBricks.z * det.np;
        if (nwin == 0)
            return;
        josephWindowKernel<<<static_cast<unsigned>((nwin + 255) / 256), 256, 0, s>>>(
            poses, vol, det, brick, nBricks, cm, grow, pixMargin, out);
        ELSA_LAUNCH_CHECK("josephWindowKernel");
    }

    void launchSumChunks(const float* partial, int chunks, int64_t nvox, float* x,
                         cudaStream_t s)
    {
        if (nvox == 0)
            return;
        sumChunksKernel<<<static_cast<unsigned>((nvox + 255) / 256), 256, 0, s>>>(partial, chunks,
                                                                                  nvox, x);
        ELSA_LAUNCH_CHECK("sumChunksKernel");
    }

    class AdjointManyPlan
    {
    public:
        std::unique_ptr<DeviceBuffer> jobs[6]; // per (grid, column axis)
        int64_t items[6] = {0, 0, 0, 0, 0, 0};
        int counts[6] = {0, 0, 0, 0, 0, 0};
        std::unique_ptr<DeviceBuffer> sums;
        int sumCount = 0;
        int64_t maxVox = 0;
        bool deep = false; // some instance uses checkpoint slabs deeper than kAxisCheckpointDepth
        // operators whose tables the jobs point into: their adjoint knobs stay fixed meanwhile
        std::vector<const JosephProjector*> holds;
        ~AdjointManyPlan()
        {
            for (const JosephProjector* J : holds)
                --J->batchRefs_;
        }
    };

    std::shared_ptr<AdjointManyPlan> planJosephAdjointMany(const std::vector<Projector*>& ops,
                                                           const std::vector<const float*>& ys,
                                                           const std::vector<float*>& xs)
    {
        if (ops.size() != ys.size() || ops.size() != xs.size())
            throw Error(ELSA_ERROR_INVALID_ARGUMENT, "planJosephAdjointMany: size mismatch");
        std::vector<AxisJob> jobs[6];
        std::vector<SumChunksEntry> sums;
        auto plan = std::make_shared<AdjointManyPlan>();
        for (size_t i = 0; i < ops.size(); ++i) {
            const auto* J = dynamic_cast<const JosephProjector*>(ops[i]);
            if (!J || !J->batchable())
                throw Error(ELSA_ERROR_NOT_SUPPORTED,
                            "batched adjoints take 3D Joseph operators with the matched "
                            "brick-owner adjoint only");
            J->appendAxisJobs(ys[i], xs[i], jobs, sums);
            ++J->batchRefs_;
            plan->holds.push_back(J);
            plan->maxVox = std::max(plan->maxVox, J->domainSize());
            plan->deep = plan->deep || J->knob(kKnobCheckpointDepth) != kAxisCheckpointDepth;
        }
        for (int k = 0; k < 6; ++k) {
            int64_t base = 0;
            for (AxisJob& j : jobs[k]) {
                j.itemBase = base;
                base += static_cast<int64_t>(j.nBricks.x) * j.nBricks.y * j.nBricks.z * j.entries;
            }
            if (base >= (int64_t(1) << 31))
                throw Error(ELSA_ERROR_NOT_SUPPORTED, "planJosephAdjointMany: too many bricks");
            plan->items[k] = base;
            plan->counts[k] = static_cast<int>(jobs[k].size());
            if (!jobs[k].empty()) {
                plan->jobs[k] = std::make_unique<DeviceBuffer>(sizeof(AxisJob) * jobs[k].size());
                ELSA_CUDA(cudaMemcpy(plan->jobs[k]->as<AxisJob>(), jobs[k].data(),
                                     sizeof(AxisJob) * jobs[k].size(), cudaMemcpyHostToDevice));
            }
        }
        plan->sumCount = static_cast<int>(sums.size());
        if (!sums.empty()) {
            plan->sums = std::make_unique<DeviceBuffer>(sizeof(SumChunksEntry) * sums.size());
            ELSA_CUDA(cudaMemcpy(plan->sums->as<SumChunksEntry>(), sums.data(),
                                 sizeof(SumChunksEntry) * sums.size(), cudaMemcpyHostToDevice));
        }
        return plan;
    }

    void runJosephAdjointMany(const AdjointManyPlan& plan, cudaStream_t s)
    {
        constexpr int TD = kAxisTD, TW = kAxisTW, TV = kAxisTV, CPD = kAxisCheckpointDepth;
        for (int k = 0; k < 6; ++k) {
            if (plan.items[k] == 0)
                continue;
            const unsigned grid = static_cast<unsigned>(plan.items[k]);
            const AxisJob* jobs = plan.jobs[k]->as<AxisJob>();
            const int n = plan.counts[k];
#define ELSA_AXIS_MANY(G_, UB_)                                                                   \
    do {                                                                                         \
        if (plan.deep)                                                                           \
            josephAdjointAxisManyKernel<G_, TD, UB_, TW, TV, 0><<<grid, 32, 0, s>>>(jobs, n);    \
        else                                                                                     \
            josephAdjointAxisManyKernel<G_, TD, UB_, TW, TV, CPD><<<grid, 32, 0, s>>>(jobs, n);  \
    } while (0)
            switch (k) {
            case 0: ELSA_AXIS_MANY(0, false); break;
            case 1: ELSA_AXIS_MANY(0, true); break;
            case 2: ELSA_AXIS_MANY(1, false); break;
            case 3: ELSA_AXIS_MANY(1, true); break;
            case 4: ELSA_AXIS_MANY(2, false); break;
            default: ELSA_AXIS_MANY(2, true); break;
            }
#undef ELSA_AXIS_MANY
            ELSA_LAUNCH_CHECK("josephAdjointAxisManyKernel");
        }
        if (plan.sumCount > 0) {
            const int64_t blocks = std::min<int64_t>((plan.maxVox + 255) / 256, 148 * 8);
            sumChunksManyKernel<<<dim3(static_cast<unsigned>(blocks),
                                       static_cast<unsigned>(plan.sumCount)),
                                  256, 0, s>>>(plan.sums->as<SumChunksEntry>());
            ELSA_LAUNCH_CHECK("sumChunksManyKernel");
        }
    }

    std::unique_ptr<Projector> makeJosephProjector(const VolumeShape& vol,
                                                   const DetectorShape& det,
                                                   const std::vector<PoseRecord>& poses,
                                                   const CurvedDetector& curved, bool fast)
    {
        return std::make_unique<JosephProjector>(vol, det, poses, curved, fast);
    }
} // namespace elsa_b200
