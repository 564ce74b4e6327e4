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
// Adjoint: atomic-free and deterministic. Each CTA owns one brick of the volume in shared memory
// for all views. For every view it visits the rays of the brick's detector window one
// conflict-free class at a time: rays whose pixel indices are congruent modulo m stay more than
// two voxels apart on every plane (m is validated per geometry at construction), so their
// bilinear taps never overlap and the threads update shared memory without atomics. Each thread
// walks one ray through the brick; classes are separated by barriers. Every voxel receives its
// contributions in a fixed order, with exactly the positions and weights of the forward kernel.
#include "joseph_tma.cuh"
#include "projector.hpp"
#include "raysetup.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace elsa_b200
{
    namespace
    {
        constexpr int kForwardThreads = 256;
        constexpr int kMinClass = 2;
        constexpr int kMaxClass = 8;

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
        __global__ void __launch_bounds__(kForwardThreads)
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

        // Detector window of every (brick, view): projection of the brick grown by one voxel,
        // plus one pixel of margin. Falls back to the whole detector when a corner lies behind
        // the source.
        __global__ void josephWindowKernel(const float* __restrict__ poses, VolumeShape vol,
                                           DetectorShape det, int3 brick, int3 nBricks,
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
            const float lo0 = static_cast<float>(bxi * brick.x - 1);
            const float lo1 = static_cast<float>(byi * brick.y - 1);
            const float lo2 = static_cast<float>(bzi * brick.z - 1);
            const float hi0 = static_cast<float>(bxi * brick.x + brick.x + 1);
            const float hi1 = static_cast<float>(byi * brick.y + brick.y + 1);
            const float hi2 = static_cast<float>(bzi * brick.z + brick.z + 1);
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
                const int noffs = dim == 3 ? 4 : 1;
                for (int o = 0; o < noffs; ++o) {
                    const int du = (o == 1) ? 0 : m;
                    const int dv = (o == 0) ? 0 : (o == 3 ? -m : m);
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
        // of `depth` planes (slab index floor(k/depth), visited in ray order).
        __global__ void josephCheckpointKernel(const JosephRay* __restrict__ rays, int64_t nrays,
                                               int depth, int stride,
                                               float2* __restrict__ checkpoints)
        {
            const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            if (r >= nrays)
                return;
            const JosephRay R = rays[r];
            if (R.n == 0)
                return;
            const int dir = (R.meta & 4) ? -1 : 1;
            const int first = floorDiv(R.k0, depth);
            float2* out = checkpoints + r * stride;
            float pa = R.pa, pb = R.pb;
            int k = R.k0, slab = first - dir;
            for (int j = 0; j < R.n; ++j, k += dir) {
                const int s = floorDiv(k, depth);
                if (s != slab) {
                    slab = s;
                    const int idx = (s - first) * dir;
                    if (idx < stride) // always true: the host sizes stride for N + 1 samples
                        out[idx] = make_float2(pa, pb);
                }
                pa = __fadd_rn(pa, R.sa);
                pb = __fadd_rn(pb, R.sb);
            }
        }

        struct PassGeom {
            int extG, extA, extB;
            int orgG, orgA, orgB;
            int strG, strA, strB;
        };

        // Walk ray r (one thread) through the brick and add its bilinear splats to the
        // shared-memory accumulator. Positions start from the slab checkpoint at the ray's first
        // sample inside the brick and are accumulated exactly as in the forward kernel.
        template <int DIM, int CPD>
        __device__ __forceinline__ void splatRay(float* acc, const JosephRay& R, float yl,
                                                 const float2* __restrict__ cps,
                                                 const PassGeom& pg)
        {
            const int dir = (R.meta & 4) ? -1 : 1;
            const int kLo = pg.orgG, kHi = pg.orgG + pg.extG - 1;
            int jLo, jHi;
            if (dir > 0) {
                jLo = max(0, kLo - R.k0);
                jHi = min(R.n - 1, kHi - R.k0);
            } else {
                jLo = max(0, R.k0 - kHi);
                jHi = min(R.n - 1, R.k0 - kLo);
            }
            if (jLo > jHi)
                return;
            int k = R.k0 + jLo * dir;
            const int first = floorDiv(R.k0, CPD);
            const float2 cp = cps[(floorDiv(k, CPD) - first) * dir];
            float pa = cp.x, pb = cp.y;
            float* plane = acc + (k - pg.orgG) * pg.strG;
            const int dPlane = dir * pg.strG;
            for (int j = jLo; j <= jHi; ++j, plane += dPlane, pa = __fadd_rn(pa, R.sa),
                     pb = __fadd_rn(pb, R.sb)) {
                Weights w;
                tapWeights(pa, pb, w);
                const int ia = w.ia - pg.orgA;
                const bool a0 = static_cast<unsigned>(ia) < static_cast<unsigned>(pg.extA);
                const bool a1 = static_cast<unsigned>(ia + 1) < static_cast<unsigned>(pg.extA);
                if (DIM == 2) {
                    if (a0)
                        plane[ia * pg.strA] += yl * w.wa;
                    if (a1)
                        plane[(ia + 1) * pg.strA] += yl * w.cwa;
                } else {
                    const int ib = w.ib - pg.orgB;
                    const bool b0 = static_cast<unsigned>(ib) < static_cast<unsigned>(pg.extB);
                    const bool b1 = static_cast<unsigned>(ib + 1) < static_cast<unsigned>(pg.extB);
                    float* q = plane + ia * pg.strA + ib * pg.strB;
                    if (a0 && b0)
                        q[0] += yl * (w.wa * w.wb);
                    if (a1 && b0)
                        q[pg.strA] += yl * (w.cwa * w.wb);
                    if (a0 && b1)
                        q[pg.strB] += yl * (w.wa * w.cwb);
                    if (a1 && b1)
                        q[pg.strA + pg.strB] += yl * (w.cwa * w.cwb);
                }
            }
        }

        // One CTA per brick of BX x BY x BZ voxels (BZ = 1 in 2D). The z stride is padded by one
        // word (2D: the y stride) so that threads on neighbouring rays hit distinct banks.
        template <int DIM, int BX, int BY, int BZ, int CPD, int NT>
        __global__ void __launch_bounds__(NT)
            josephAdjointKernel(const JosephRay* __restrict__ rays,
                                const float2* __restrict__ checkpoints, int cpStride,
                                const float* __restrict__ y,
                                const RayWindow* __restrict__ windows,
                                const unsigned* __restrict__ viewAxes, VolumeShape vol,
                                DetectorShape det, int m, int3 nBricks, float* __restrict__ x)
        {
            extern __shared__ float acc[];
            constexpr int kRow = DIM == 3 ? BX : BX + 1;
            constexpr int kPlane = DIM == 3 ? BX * BY + 1 : kRow * BY;
            constexpr int kWords = kPlane * BZ;
            for (int i = threadIdx.x; i < kWords; i += blockDim.x)
                acc[i] = 0.0f;
            const int bi = blockIdx.x;
            const int org0 = (bi % nBricks.x) * BX, org1 = ((bi / nBricks.x) % nBricks.y) * BY,
                      org2 = (bi / (nBricks.x * nBricks.y)) * BZ;
            const int nb = nBricks.x * nBricks.y * nBricks.z;
            __syncthreads();
            for (int p = 0; p < det.np; ++p) {
                const RayWindow w = windows[static_cast<int64_t>(p) * nb + bi];
                if (w.u0 > w.u1 || w.v0 > w.v1)
                    continue;
                const unsigned axes = viewAxes[p];
                for (int g = 0; g < DIM; ++g) {
                    if (!((axes >> g) & 1u))
                        continue;
                    // axis g is driving; (a, b) are the remaining axes in increasing order
                    PassGeom pg;
                    if (g == 0) {
                        pg.extG = BX, pg.orgG = org0, pg.strG = 1;
                        pg.extA = BY, pg.orgA = org1, pg.strA = kRow;
                        pg.extB = BZ, pg.orgB = org2, pg.strB = kPlane;
                    } else if (g == 1) {
                        pg.extG = BY, pg.orgG = org1, pg.strG = kRow;
                        pg.extA = BX, pg.orgA = org0, pg.strA = 1;
                        pg.extB = BZ, pg.orgB = org2, pg.strB = kPlane;
                    } else {
                        pg.extG = BZ, pg.orgG = org2, pg.strG = kPlane;
                        pg.extA = BX, pg.orgA = org0, pg.strA = 1;
                        pg.extB = BY, pg.orgB = org1, pg.strB = kRow;
                    }
                    if (DIM == 2)
                        pg.extB = 1, pg.orgB = 0, pg.strB = 0;
                    const int mv = DIM == 3 ? m : 1;
                    for (int cv = 0; cv < mv; ++cv) {
                        const int vStart = w.v0 + ((cv - w.v0 % m) % m + m) % m;
                        const int nvc =
                            DIM == 3 ? (vStart <= w.v1 ? (w.v1 - vStart) / m + 1 : 0) : 1;
                        for (int cu = 0; cu < m; ++cu) {
                            const int uStart = w.u0 + ((cu - w.u0 % m) % m + m) % m;
                            const int nuc = uStart <= w.u1 ? (w.u1 - uStart) / m + 1 : 0;
                            const int total = nuc * nvc;
                            for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
                                const int u = uStart + (idx % nuc) * m;
                                const int v = DIM == 3 ? vStart + (idx / nuc) * m : 0;
                                const int64_t r = u + static_cast<int64_t>(det.nu) *
                                                          (v + static_cast<int64_t>(det.nv) * p);
                                const JosephRay R = rays[r];
                                if (R.n == 0 || (R.meta & 3) != g)
                                    continue;
                                splatRay<DIM, CPD>(acc, R, __ldg(y + r) * R.len,
                                                   checkpoints + r * cpStride, pg);
                            }
                            __syncthreads();
                        }
                    }
                }
            }
            for (int i = threadIdx.x; i < BX * BY * BZ; i += blockDim.x) {
                const int lx = i % BX, ly = (i / BX) % BY, lz = i / (BX * BY);
                const int gx = org0 + lx, gy = org1 + ly, gz = org2 + lz;
                if (gx < vol.n[0] && gy < vol.n[1] && gz < vol.n[2])
                    x[gx + static_cast<int64_t>(vol.n[0]) *
                               (gy + static_cast<int64_t>(vol.n[1]) * gz)] =
                        acc[lz * kPlane + ly * kRow + lx];
            }
        }

        template <int DIM, int BX, int BY, int BZ, int CPD, int NT>
        struct AdjointConfig {
            static constexpr int kRow = DIM == 3 ? BX : BX + 1;
            static constexpr int kPlane = DIM == 3 ? BX * BY + 1 : kRow * BY;
            static constexpr size_t kSmem = sizeof(float) * kPlane * BZ;
            static constexpr int kThreads = NT;
            static constexpr int kCheckpointDepth = CPD;
            static_assert(BX % CPD == 0 && BY % CPD == 0 && (DIM == 2 || BZ % CPD == 0),
                          "brick edges must be multiples of the checkpoint depth");
            static int3 brick() { return make_int3(BX, BY, BZ); }
            static void prepare()
            {
                ELSA_CUDA(cudaFuncSetAttribute(josephAdjointKernel<DIM, BX, BY, BZ, CPD, NT>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               static_cast<int>(kSmem)));
            }
            static void launch(int nbricks, cudaStream_t s, const JosephRay* rays,
                               const float2* cps, int cpStride, const float* y,
                               const RayWindow* win, const unsigned* axes, VolumeShape vol,
                               DetectorShape det, int m, int3 nb, float* x)
            {
                josephAdjointKernel<DIM, BX, BY, BZ, CPD, NT><<<nbricks, kThreads, kSmem, s>>>(
                    rays, cps, cpStride, y, win, axes, vol, det, m, nb, x);
            }
        };

        using Adjoint3d = AdjointConfig<3, 16, 32, 16, 16, 128>;
        using Adjoint2d = AdjointConfig<2, 64, 64, 1, 64, 256>;

        class JosephProjector final : public Projector
        {
        public:
            JosephProjector(const VolumeShape& vol, const DetectorShape& det,
                            const std::vector<PoseRecord>& poses)
                : Projector(0, vol, det, poses)
            {
                const int64_t nrays = rangeSize_;
                ELSA_CUDA(cudaMalloc(&dRays_, sizeof(JosephRay) * nrays));
                const int threads = 256;
                const unsigned blocks = static_cast<unsigned>((nrays + threads - 1) / threads);
                josephSetupKernel<<<blocks, threads>>>(dPoses_, vol_, det_, dRays_);
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
                classSpacing_ = 0;
                for (int m = kMinClass; m <= kMaxClass; ++m)
                    if (!((bad >> m) & 1u)) {
                        classSpacing_ = m;
                        break;
                    }
                if (classSpacing_ == 0)
                    throw Error(ELSA_ERROR_NOT_SUPPORTED,
                                "JosephsMethod: neighbouring detector rays pass within two voxels "
                                "of each other even eight pixels apart; the atomic-free adjoint "
                                "needs a coarser detector");

                int cpd;
                if (vol_.dim == 3) {
                    brick_ = Adjoint3d::brick();
                    cpd = Adjoint3d::kCheckpointDepth;
                    Adjoint3d::prepare();
                } else {
                    brick_ = Adjoint2d::brick();
                    cpd = Adjoint2d::kCheckpointDepth;
                    Adjoint2d::prepare();
                }
                const int maxDim = std::max(vol_.n[0], std::max(vol_.n[1], vol_.n[2]));
                cpStride_ = maxDim / cpd + 3;
                ELSA_CUDA(cudaMalloc(&dCheckpoints_, sizeof(float2) * nrays * cpStride_));
                josephCheckpointKernel<<<blocks, threads>>>(dRays_, nrays, cpd, cpStride_,
                                                            dCheckpoints_);
                ELSA_LAUNCH_CHECK("josephCheckpointKernel");

                nBricks_ = make_int3((vol_.n[0] + brick_.x - 1) / brick_.x,
                                     (vol_.n[1] + brick_.y - 1) / brick_.y,
                                     (vol_.n[2] + brick_.z - 1) / brick_.z);
                const int64_t nwin =
                    static_cast<int64_t>(nBricks_.x) * nBricks_.y * nBricks_.z * det_.np;
                ELSA_CUDA(cudaMalloc(&dWindows_, sizeof(RayWindow) * nwin));
                josephWindowKernel<<<static_cast<unsigned>((nwin + 255) / 256), 256>>>(
                    dPoses_, vol_, det_, brick_, nBricks_, dWindows_);
                ELSA_LAUNCH_CHECK("josephWindowKernel");
                if (vol_.dim == 3) {
                    std::vector<float> hp(poses_.size() * kPoseFloats);
                    std::memcpy(hp.data(), poses_.data(), sizeof(float) * hp.size());
                    tma_ = std::make_unique<JosephForwardTma>(vol_, det_, hp, dRays_);
                }
                ELSA_CUDA(cudaDeviceSynchronize());
            }

            ~JosephProjector() override
            {
                cudaFree(dRays_);
                cudaFree(dViewAxes_);
                cudaFree(dWindows_);
                cudaFree(dCheckpoints_);
            }

            void forward(const float* x, float* y, cudaStream_t s) override
            {
                const int64_t nrays = rangeSize_;
                const unsigned blocks =
                    static_cast<unsigned>((nrays + kForwardThreads - 1) / kForwardThreads);
                if (tma_)
                    tma_->forward(x, y, s);
                else if (vol_.dim == 3)
                    josephForwardKernel<3><<<blocks, kForwardThreads, 0, s>>>(dRays_, nrays, x,
                                                                                vol_, y);
                else
                    josephForwardKernel<2><<<blocks, kForwardThreads, 0, s>>>(dRays_, nrays, x,
                                                                                vol_, y);
                ELSA_LAUNCH_CHECK("josephForwardKernel");
            }

            void adjoint(const float* y, float* x, cudaStream_t s) override
            {
                const int nb = nBricks_.x * nBricks_.y * nBricks_.z;
                if (vol_.dim == 3)
                    Adjoint3d::launch(nb, s, dRays_, dCheckpoints_, cpStride_, y, dWindows_,
                                      dViewAxes_, vol_, det_, classSpacing_, nBricks_, x);
                else
                    Adjoint2d::launch(nb, s, dRays_, dCheckpoints_, cpStride_, y, dWindows_,
                                      dViewAxes_, vol_, det_, classSpacing_, nBricks_, x);
                ELSA_LAUNCH_CHECK("josephAdjointKernel");
            }

            int64_t info(int key) const override
            {
                switch (key) {
                case 0:
                    return classSpacing_;
                case 1:
                    return nBricks_.x * nBricks_.y * nBricks_.z;
                case 2:
                    return sampleCount_;
                case 3: // error word of the TMA forward (synchronizes)
                    return tma_ ? static_cast<int64_t>(tma_->errorWord()) : 0;
                case 4: // parts per million of detector tiles on the gather fallback
                    return tma_ ? static_cast<int64_t>(tma_->fallbackFraction() * 1e6) : -1;
                default:
                    return -1;
                }
            }

        private:
            JosephRay* dRays_ = nullptr;
            unsigned* dViewAxes_ = nullptr;
            RayWindow* dWindows_ = nullptr;
            float2* dCheckpoints_ = nullptr;
            int cpStride_ = 0;
            int classSpacing_ = 0;
            int64_t sampleCount_ = 0;
            std::unique_ptr<JosephForwardTma> tma_;
            int3 brick_{}, nBricks_{};
        };
    } // namespace

    std::unique_ptr<Projector> makeJosephProjector(const VolumeShape& vol,
                                                   const DetectorShape& det,
                                                   const std::vector<PoseRecord>& poses)
    {
        return std::make_unique<JosephProjector>(vol, det, poses);
    }
} // namespace elsa_b200
