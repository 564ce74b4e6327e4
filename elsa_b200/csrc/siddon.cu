// Siddon's method (exact intersection lengths) for sm_100a.
//
// Reference semantics: projectors/SiddonsMethod.cpp:76-124 with projectors/TraverseAABB.cpp:6-184
// (elsa's CPU path, the parity target). A ray visits the voxels it crosses in order; each visit
// advances every axis whose next boundary parameter T is minimal, and the voxel's weight is the
// parameter difference tExit - tEntry:
//   forward  y[r] = sum_visits x[voxel] * (tExit - tEntry)
//   adjoint  x[v] = sum_r sum_{visits of v} y[r] * (tExit - tEntry)
// T advances by repeated float addition (T += tDelta), so both kernels replay the reference's
// float operations one by one (no contraction): the visited voxels and weights are bit-identical
// to the CPU traversal.
//
// Forward: one thread per ray, voxels gathered through the read-only cache.
//
// Adjoint, two kernels (launch knob kKnobAdjointScatter). The scatter kernel replays each ray
// like the forward, one thread per ray, and adds y * weight to every visited voxel with a
// fire-and-forget atomic: the reference's own scheme, with an addition order that varies from run
// to run. The brick-owner kernel is atomic-free and deterministic:
// on the brick-owner scheme of the Joseph adjoint. One
// warp owns a 16^3 brick in shared memory for all views. Rays are cut into slabs of 16 voxels
// along their axis g of largest |direction|; per (ray, slab) a checkpoint holds the traversal
// state (T of every axis, entry parameter, voxel) at the ray's first visit inside the slab,
// computed once per geometry. For each view the warp takes the rays of the brick's detector
// window class by class (pixel indices congruent modulo m, m validated per geometry so that
// same-class rays with the same g stay more than two voxels apart laterally on every slice);
// each lane replays one ray's visits inside the slab from its checkpoint and adds the weights of
// the visits that fall inside the brick. Same-class rays therefore never touch the same voxel,
// and every voxel sums its contributions in a fixed order.
#include "projector.hpp"
#include "raysetup.cuh"
#include "solvers.hpp"

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cstring>

namespace elsa_b200
{
    namespace
    {
        constexpr int kForwardThreads = 128;    // default rays per block of the forward
        constexpr int kScatterThreads = 256;    // rays per block of the scatter adjoint
        constexpr int kMaxForwardThreads = 512; // largest block the autotuner may choose
        constexpr int kAdjointWarpsPerSm = 22;  // view-chunk target of the warp-brick adjoint
        constexpr int kMinAdjointChunks = 32;   // default floor of the view chunks
        constexpr int64_t kChunkMemory = int64_t(1) << 31; // default partial-volume budget
        constexpr int kSlab = 16; // brick edge = checkpoint slab depth
        constexpr float kWindowSlack = 0.1f;       // voxels around a brick in its ray window
        constexpr float kWindowPixelMargin = 0.05f; // pixels around the projected brick
        constexpr int kMinClass = 2;
        constexpr int kMaxClass = 8;
        constexpr int kActive = 256;

        __device__ __forceinline__ int floorDiv(int a, int b)
        {
            const int q = a / b;
            return (a % b != 0 && ((a < 0) != (b < 0))) ? q - 1 : q;
        }

        __device__ __forceinline__ int axisStep(int meta, int i)
        {
            return ((meta >> (5 + i)) & 1) ? 0 : (((meta >> (2 + i)) & 1) ? -1 : 1);
        }

        // One visit: the parameter where the ray leaves the current voxel, and which axes cross
        // (TraverseAABB.cpp:55-100: all axes whose T is minimal advance together).
        template <int DIM>
        __device__ __forceinline__ float nextCrossing(float T0, float T1, float T2, bool& m0,
                                                      bool& m1, bool& m2)
        {
            // an axis crosses when its T is the minimum (T0 <= T1 && T0 <= T2 and so on: the T
            // are never NaN, FLT_MAX for an axis the ray does not cross)
            const float tm = DIM == 3 ? fminf(T0, fminf(T1, T2)) : fminf(T0, T1);
            m0 = T0 == tm;
            m1 = T1 == tm;
            m2 = DIM == 3 && T2 == tm;
            return tm;
        }

        // Entry voxel in axis order from the record (g and the two other axes a < b).
        __device__ __forceinline__ void entryVoxel(int g, int kg, int ca, int cb, int& c0,
                                                   int& c1, int& c2)
        {
            c0 = g == 0 ? kg : ca;
            c1 = g == 1 ? kg : (g == 0 ? ca : cb);
            c2 = g == 2 ? kg : cb;
        }

        template <int DIM>
        __global__ void __launch_bounds__(kMaxForwardThreads)
            siddonForwardKernel(const SiddonRay* __restrict__ rays, int64_t nrays,
                                const float* __restrict__ x, VolumeShape vol, int binary,
                                float* __restrict__ y)
        {
            // binary: BinaryMethod (projectors/BinaryMethod.cpp:66-111), weight 1 per visit
            const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            if (r >= nrays)
                return;
            const SiddonRay R = rays[r];
            float acc = 0.0f;
            if (R.meta & kActive) {
                const int g = R.meta & 3;
                int c0, c1, c2;
                entryVoxel(g, R.kFirst, R.cur[0], R.cur[1], c0, c1, c2);
                const int s0 = axisStep(R.meta, 0), s1 = axisStep(R.meta, 1),
                          s2 = axisStep(R.meta, 2);
                const int nx = vol.n[0], ny = vol.n[1], nz = vol.n[2];
                const int64_t sy = nx, sz = static_cast<int64_t>(nx) * ny;
                int64_t idx = c0 + sy * c1 + (DIM == 3 ? sz * c2 : 0);
                float T0 = R.T[0], T1 = R.T[1], T2 = R.T[2];
                float tExit = 0.0f;
                const int maxVisits = nx + ny + (DIM == 3 ? nz : 0) + 3;
                for (int it = 0; it < maxVisits; ++it) {
                    const float tEntry = tExit;
                    bool m0, m1, m2;
                    tExit = nextCrossing<DIM>(T0, T1, T2, m0, m1, m2);
                    if (m0) {
                        c0 += s0;
                        T0 = __fadd_rn(T0, R.tDelta[0]);
                    }
                    if (m1) {
                        c1 += s1;
                        T1 = __fadd_rn(T1, R.tDelta[1]);
                    }
                    if (m2) {
                        c2 += s2;
                        T2 = __fadd_rn(T2, R.tDelta[2]);
                    }
                    const bool inside =
                        static_cast<unsigned>(c0) < static_cast<unsigned>(nx) &&
                        static_cast<unsigned>(c1) < static_cast<unsigned>(ny) &&
                        (DIM < 3 || static_cast<unsigned>(c2) < static_cast<unsigned>(nz));
                    const float w = binary ? 1.0f : __fsub_rn(tExit, tEntry);
                    acc = __fadd_rn(acc, __fmul_rn(__ldg(x + idx), w));
                    if (!inside)
                        break;
                    idx += (m0 ? s0 : 0) + (m1 ? s1 * sy : 0) + (m2 ? s2 * sz : 0);
                }
            }
            y[r] = acc;
        }

        // Adjoint by atomic scatter: the forward's visit loop, adding y[r] * weight to each
        // visited voxel (x zeroed beforehand). The atomics' return values are unused, so they
        // compile to reductions that do not wait for the memory system.
        template <int DIM>
        __global__ void __launch_bounds__(kScatterThreads)
            siddonScatterKernel(const SiddonRay* __restrict__ rays, int64_t nrays,
                                const float* __restrict__ y, VolumeShape vol, int binary,
                                float* __restrict__ x)
        {
            const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            if (r >= nrays)
                return;
            const float yr = __ldg(y + r);
            const SiddonRay R = rays[r];
            if (!(R.meta & kActive) || yr == 0.0f)
                return;
            const int g = R.meta & 3;
            int c0, c1, c2;
            entryVoxel(g, R.kFirst, R.cur[0], R.cur[1], c0, c1, c2);
            const int s0 = axisStep(R.meta, 0), s1 = axisStep(R.meta, 1), s2 = axisStep(R.meta, 2);
            const int nx = vol.n[0], ny = vol.n[1], nz = vol.n[2];
            const int64_t sy = nx, sz = static_cast<int64_t>(nx) * ny;
            int64_t idx = c0 + sy * c1 + (DIM == 3 ? sz * c2 : 0);
            float T0 = R.T[0], T1 = R.T[1], T2 = R.T[2];
            float tExit = 0.0f;
            const int maxVisits = nx + ny + (DIM == 3 ? nz : 0) + 3;
            for (int it = 0; it < maxVisits; ++it) {
                const float tEntry = tExit;
                bool m0, m1, m2;
                tExit = nextCrossing<DIM>(T0, T1, T2, m0, m1, m2);
                if (m0) {
                    c0 += s0;
                    T0 = __fadd_rn(T0, R.tDelta[0]);
                }
                if (m1) {
                    c1 += s1;
                    T1 = __fadd_rn(T1, R.tDelta[1]);
                }
                if (m2) {
                    c2 += s2;
                    T2 = __fadd_rn(T2, R.tDelta[2]);
                }
                const bool inside = static_cast<unsigned>(c0) < static_cast<unsigned>(nx) &&
                                    static_cast<unsigned>(c1) < static_cast<unsigned>(ny) &&
                                    (DIM < 3 || static_cast<unsigned>(c2) < static_cast<unsigned>(nz));
                const float w = binary ? 1.0f : __fsub_rn(tExit, tEntry);
                atomicAdd(x + idx, __fmul_rn(yr, w));
                if (!inside)
                    break;
                idx += (m0 ? s0 : 0) + (m1 ? s1 * sy : 0) + (m2 ? s2 * sz : 0);
            }
        }

        // Replays every ray once: writes the traversal state at the ray's first visit in each
        // slab of kSlab voxels along g (slab-major, row floor(k/kSlab) + 1, column = ray; skipped
        // when cpState is null), the last visited index along g and the visit count
        // (SiddonsMethod's sample count; skipped when visits is null).
        template <int DIM>
        __global__ void siddonCheckpointKernel(SiddonRay* __restrict__ rays, int64_t nrays,
                                               VolumeShape vol, int slabRows,
                                               float4* __restrict__ cpState,
                                               unsigned* __restrict__ cpVoxel,
                                               unsigned long long* __restrict__ visits)
        {
            const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            if (r >= nrays)
                return;
            SiddonRay R = rays[r];
            if (!(R.meta & kActive))
                return;
            const int g = R.meta & 3;
            int a, b;
            nonDrivingAxes(g, a, b);
            int c0, c1, c2;
            entryVoxel(g, R.kFirst, R.cur[0], R.cur[1], c0, c1, c2);
            const int s0 = axisStep(R.meta, 0), s1 = axisStep(R.meta, 1), s2 = axisStep(R.meta, 2);
            const int nx = vol.n[0], ny = vol.n[1], nz = vol.n[2];
            float T0 = R.T[0], T1 = R.T[1], T2 = R.T[2];
            float tExit = 0.0f;
            int slab = INT_MIN, count = 0, kLast = R.kFirst;
            const int maxVisits = nx + ny + (DIM == 3 ? nz : 0) + 3;
            for (int it = 0; it < maxVisits; ++it) {
                const float tEntry = tExit;
                const int cg = g == 0 ? c0 : (g == 1 ? c1 : c2);
                const int s = floorDiv(cg, kSlab);
                if (s != slab) {
                    slab = s;
                    if (cpState != nullptr && s + 1 >= 0 && s + 1 < slabRows) {
                        const int ca = a == 0 ? c0 : c1;
                        const int cb = DIM == 3 ? (b == 1 ? c1 : c2) : 0;
                        const int64_t at = static_cast<int64_t>(s + 1) * nrays + r;
                        cpState[at] = make_float4(T0, T1, T2, tEntry);
                        cpVoxel[at] =
                            static_cast<unsigned>(ca) | (static_cast<unsigned>(cb) << 16);
                    }
                }
                kLast = cg;
                ++count;
                bool m0, m1, m2;
                tExit = nextCrossing<DIM>(T0, T1, T2, m0, m1, m2);
                if (m0) {
                    c0 += s0;
                    T0 = __fadd_rn(T0, R.tDelta[0]);
                }
                if (m1) {
                    c1 += s1;
                    T1 = __fadd_rn(T1, R.tDelta[1]);
                }
                if (m2) {
                    c2 += s2;
                    T2 = __fadd_rn(T2, R.tDelta[2]);
                }
                const bool inside =
                    static_cast<unsigned>(c0) < static_cast<unsigned>(nx) &&
                    static_cast<unsigned>(c1) < static_cast<unsigned>(ny) &&
                    (DIM < 3 || static_cast<unsigned>(c2) < static_cast<unsigned>(nz));
                if (!inside)
                    break;
            }
            R.kLast = kLast;
            R.crossings = count;
            rays[r] = R;
            if (visits != nullptr)
                atomicAdd(visits, static_cast<unsigned long long>(count));
        }

        // True when rays R and S (same axis g) stay more than two voxels apart in one lateral
        // coordinate over the slices of g that both visit.
        __device__ bool separated(const SiddonRay& R, const SiddonLine& LR, const SiddonRay& S,
                                  const SiddonLine& LS, int dim)
        {
            const int lo = max(min(R.kFirst, R.kLast), min(S.kFirst, S.kLast));
            const int hi = min(max(R.kFirst, R.kLast), max(S.kFirst, S.kLast));
            if (lo > hi)
                return true;
            const float margin = 2.05f;
            const float g0 = static_cast<float>(lo), g1 = static_cast<float>(hi + 1);
            const float da0 = fmaf(g0 - LR.g0, LR.sa, LR.a0) - fmaf(g0 - LS.g0, LS.sa, LS.a0);
            const float da1 = fmaf(g1 - LR.g0, LR.sa, LR.a0) - fmaf(g1 - LS.g0, LS.sa, LS.a0);
            if ((da0 > margin && da1 > margin) || (da0 < -margin && da1 < -margin))
                return true;
            if (dim == 3) {
                const float db0 = fmaf(g0 - LR.g0, LR.sb, LR.b0) - fmaf(g0 - LS.g0, LS.sb, LS.b0);
                const float db1 = fmaf(g1 - LR.g0, LR.sb, LR.b0) - fmaf(g1 - LS.g0, LS.sb, LS.b0);
                if ((db0 > margin && db1 > margin) || (db0 < -margin && db1 < -margin))
                    return true;
            }
            return false;
        }

        // Axes present per view and, per candidate class spacing m, whether two rays that the
        // adjoint may process concurrently could visit the same voxel. Neighbours checked: the
        // same detector row m pixels apart, and the next class row (m rows down) within +-32
        // pixels; rays further apart in a class are further apart on every slice (the pixel ->
        // slice-position map of a flat detector is monotone for rays sharing g).
        __global__ void siddonClassCheckKernel(const SiddonRay* __restrict__ rays,
                                               const SiddonLine* __restrict__ lines,
                                               DetectorShape det, int dim,
                                               unsigned* __restrict__ viewAxes,
                                               unsigned* __restrict__ badSpacing)
        {
            const int64_t nrays = static_cast<int64_t>(det.nu) * det.nv * det.np;
            const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            if (r >= nrays)
                return;
            const SiddonRay R = rays[r];
            if (!(R.meta & kActive))
                return;
            const SiddonLine LR = lines[r];
            const int u = static_cast<int>(r % det.nu);
            const int v = static_cast<int>((r / det.nu) % det.nv);
            const int p = static_cast<int>(r / (static_cast<int64_t>(det.nu) * det.nv));
            atomicOr(viewAxes + p, 1u << (R.meta & 3));
            unsigned bad = 0;
            for (int m = kMinClass; m <= kMaxClass; ++m) {
                const int noffs = dim == 3 ? 1 + 65 : 1;
                for (int o = 0; o < noffs; ++o) {
                    const int du = o == 0 ? m : o - 1 - 32;
                    const int dv = o == 0 ? 0 : m;
                    const int u2 = u + du, v2 = v + dv;
                    if (u2 < 0 || u2 >= det.nu || v2 < 0 || v2 >= det.nv)
                        continue;
                    const int64_t r2 =
                        u2 + static_cast<int64_t>(det.nu) * (v2 + static_cast<int64_t>(det.nv) * p);
                    const SiddonRay S = rays[r2];
                    if (!(S.meta & kActive) || (S.meta & 3) != (R.meta & 3))
                        continue;
                    if (!separated(R, LR, S, lines[r2], dim))
                        bad |= 1u << m;
                }
            }
            if (bad)
                atomicOr(badSpacing, bad);
        }

        // Shared-memory brick of one warp (x stride 1, row stride 17, plane stride = 1 mod 32).
        // Check of the brick windows (test support, elsa_projector_info key 8): every visited
        // voxel must lie in a brick whose window for the ray's view contains the ray. Counts the
        // visits that violate this.
        template <int DIM>
        __global__ void siddonWindowCheckKernel(const SiddonRay* __restrict__ rays,
                                                const RayWindow* __restrict__ windows,
                                                VolumeShape vol, DetectorShape det, int3 brick,
                                                int3 nBricks, int onlyAxis,
                                                unsigned long long* __restrict__ misses)
        {
            const int64_t nrays = static_cast<int64_t>(det.nu) * det.nv * det.np;
            const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            if (r >= nrays)
                return;
            const SiddonRay R = rays[r];
            if (!(R.meta & kActive) || (onlyAxis >= 0 && (R.meta & 3) != onlyAxis))
                return;
            const int u = static_cast<int>(r % det.nu);
            const int v = static_cast<int>((r / det.nu) % det.nv);
            const int p = static_cast<int>(r / (static_cast<int64_t>(det.nu) * det.nv));
            const int nb = nBricks.x * nBricks.y * nBricks.z;
            const int g = R.meta & 3;
            int c0, c1, c2;
            entryVoxel(g, R.kFirst, R.cur[0], R.cur[1], c0, c1, c2);
            const int s0 = axisStep(R.meta, 0), s1 = axisStep(R.meta, 1), s2 = axisStep(R.meta, 2);
            float T0 = R.T[0], T1 = R.T[1], T2 = R.T[2];
            const int maxVisits = vol.n[0] + vol.n[1] + (DIM == 3 ? vol.n[2] : 0) + 3;
            unsigned long long bad = 0;
            int lastBrick = -1;
            for (int it = 0; it < maxVisits; ++it) {
                const int o0 = c0, o1 = c1, o2 = DIM == 3 ? c2 : 0; // the voxel of this visit
                bool m0, m1, m2;
                nextCrossing<DIM>(T0, T1, T2, m0, m1, m2);
                if (m0) {
                    c0 += s0;
                    T0 = __fadd_rn(T0, R.tDelta[0]);
                }
                if (m1) {
                    c1 += s1;
                    T1 = __fadd_rn(T1, R.tDelta[1]);
                }
                if (m2) {
                    c2 += s2;
                    T2 = __fadd_rn(T2, R.tDelta[2]);
                }
                const int bi = o0 / brick.x + nBricks.x * (o1 / brick.y + nBricks.y * (o2 / brick.z));
                if (bi != lastBrick) {
                    const RayWindow w = windows[static_cast<int64_t>(p) * nb + bi];
                    if (u < w.u0 || u > w.u1 || v < w.v0 || v > w.v1)
                        ++bad;
                    else
                        lastBrick = bi;
                }
                const bool inside =
                    static_cast<unsigned>(c0) < static_cast<unsigned>(vol.n[0]) &&
                    static_cast<unsigned>(c1) < static_cast<unsigned>(vol.n[1]) &&
                    (DIM < 3 || static_cast<unsigned>(c2) < static_cast<unsigned>(vol.n[2]));
                if (!inside)
                    break;
            }
            if (bad)
                atomicAdd(misses, bad);
        }

        template <int DIM>
        struct SiddonBrick {
            static constexpr int kBz = DIM == 3 ? kSlab : 1;
            static constexpr int kRow = kSlab + 1;
            static constexpr int kPlaneMin = kRow * kSlab;
            static constexpr int kPlane = kPlaneMin + ((33 - kPlaneMin % 32) % 32);
            static constexpr int kWords = kPlane * kBz + 1; // + dummy word
        };

        // Replays the visits of one ray inside the slab [kLo, kLo + 15] along G from its
        // checkpoint and adds y * weight to the visited voxels of the brick (visits outside the
        // brick go to the dummy word).
        template <int DIM, int G>
        __device__ __forceinline__ void splatSegment(float* acc, float3 tDelta, int meta,
                                                     int kFirst, float4 cp, unsigned cpv, float yv,
                                                     int kLo, int org0, int org1, int org2,
                                                     const VolumeShape& vol, int binary)
        {
            using L = SiddonBrick<DIM>;
            const int dirG = ((meta >> (2 + G)) & 1) ? -1 : 1;
            const int kg = dirG > 0 ? max(kLo, kFirst) : min(kLo + kSlab - 1, kFirst);
            int c0, c1, c2;
            entryVoxel(G, kg, static_cast<int>(cpv & 0xffffu), static_cast<int>(cpv >> 16), c0,
                       c1, c2);
            const int s0 = axisStep(meta, 0), s1 = axisStep(meta, 1), s2 = axisStep(meta, 2);
            float T0 = cp.x, T1 = cp.y, T2 = cp.z;
            float tEntry = cp.w;
            float* dummy = acc + L::kWords - 1;
            for (int it = 0; it < 3 * kSlab + 3; ++it) {
                bool m0, m1, m2;
                const float tExit = nextCrossing<DIM>(T0, T1, T2, m0, m1, m2);
                const int l0 = c0 - org0, l1 = c1 - org1, l2 = DIM == 3 ? c2 - org2 : 0;
                const bool mine = static_cast<unsigned>(l0) < static_cast<unsigned>(kSlab) &&
                                  static_cast<unsigned>(l1) < static_cast<unsigned>(kSlab) &&
                                  static_cast<unsigned>(l2) < static_cast<unsigned>(L::kBz);
                float* adr = mine ? acc + l2 * L::kPlane + l1 * L::kRow + l0 : dummy;
                const float w = binary ? 1.0f : __fsub_rn(tExit, tEntry);
                *adr = __fadd_rn(*adr, __fmul_rn(yv, w));
                if (m0) {
                    c0 += s0;
                    T0 = __fadd_rn(T0, tDelta.x);
                }
                if (m1) {
                    c1 += s1;
                    T1 = __fadd_rn(T1, tDelta.y);
                }
                if (m2) {
                    c2 += s2;
                    T2 = __fadd_rn(T2, tDelta.z);
                }
                const bool inside =
                    static_cast<unsigned>(c0) < static_cast<unsigned>(vol.n[0]) &&
                    static_cast<unsigned>(c1) < static_cast<unsigned>(vol.n[1]) &&
                    (DIM < 3 || static_cast<unsigned>(c2) < static_cast<unsigned>(vol.n[2]));
                const int cg = G == 0 ? c0 : (G == 1 ? c1 : c2);
                if (!inside || cg < kLo || cg >= kLo + kSlab)
                    break;
                tEntry = tExit;
            }
        }

        // One (view, axis G) for a warp-owned brick: m x m ray classes separated by __syncwarp;
        // lane i takes class rays i, i + 32, ... (u fastest within the class grid).
        template <int DIM, int G>
        __device__ __forceinline__ void siddonView(float* acc, const RayWindow& w, int p, int m,
                                                   const SiddonRay* __restrict__ rays,
                                                   const float4* __restrict__ cpState,
                                                   const unsigned* __restrict__ cpVoxel,
                                                   int64_t nrays, const float* __restrict__ y,
                                                   const DetectorShape& det, int org0, int org1,
                                                   int org2, const VolumeShape& vol, int binary)
        {
            const int kLo = G == 0 ? org0 : (G == 1 ? org1 : org2);
            const int kHi = kLo + kSlab - 1;
            const int lane = threadIdx.x & 31;
            const int64_t viewBase = static_cast<int64_t>(det.nu) * det.nv * p;
            const int64_t cpRow = static_cast<int64_t>(kLo / kSlab + 1) * nrays;
            for (int ov = 0; ov < m; ++ov) {
                const int vStart = w.v0 + ov;
                const int nvc = vStart <= w.v1 ? (w.v1 - vStart) / m + 1 : 0;
                for (int ou = 0; ou < m; ++ou) {
                    const int uStart = w.u0 + ou;
                    const int nuc = uStart <= w.u1 ? (w.u1 - uStart) / m + 1 : 0;
                    const int total = nuc * nvc;
                    for (int i = lane; i < total; i += 32) {
                        const int iv = i / nuc;
                        const int iu = i - iv * nuc;
                        const int64_t r = viewBase + (uStart + iu * m) +
                                          static_cast<int64_t>(det.nu) * (vStart + iv * m);
                        const int4* rp = reinterpret_cast<const int4*>(rays + r);
                        const int4 q0 = __ldg(rp);     // tDelta[3], meta
                        const int4 q1 = __ldg(rp + 1); // kFirst, kLast, cur[2]
                        const int meta = q0.w;
                        if (!(meta & kActive) || (meta & 3) != G)
                            continue;
                        if (max(q1.x, q1.y) < kLo || min(q1.x, q1.y) > kHi)
                            continue;
                        const float3 td = make_float3(__int_as_float(q0.x), __int_as_float(q0.y),
                                                      __int_as_float(q0.z));
                        splatSegment<DIM, G>(acc, td, meta, q1.x, __ldg(cpState + cpRow + r),
                                             __ldg(cpVoxel + cpRow + r), __ldg(y + r), kLo, org0,
                                             org1, org2, vol, binary);
                    }
                    __syncwarp();
                }
            }
        }

        template <int DIM>
        __global__ void __launch_bounds__(32)
            siddonAdjointKernel(const SiddonRay* __restrict__ rays,
                                const float4* __restrict__ cpState,
                                const unsigned* __restrict__ cpVoxel, int64_t nrays,
                                const float* __restrict__ y,
                                const RayWindow* __restrict__ windows,
                                const unsigned* __restrict__ viewAxes, VolumeShape vol,
                                DetectorShape det, int m, int3 nBricks, int viewsPerChunk,
                                int binary, float* __restrict__ x)
        {
            // blockIdx.y selects a chunk of views; with several chunks the brick goes to
            // x + chunk * nvox and launchSumChunks adds the chunks in order
            using L = SiddonBrick<DIM>;
            __shared__ float acc[L::kWords];
            const int lane = threadIdx.x;
            const int bi = blockIdx.x;
            const int org0 = (bi % nBricks.x) * kSlab;
            const int org1 = ((bi / nBricks.x) % nBricks.y) * kSlab;
            const int org2 = (bi / (nBricks.x * nBricks.y)) * L::kBz;
            const int nb = nBricks.x * nBricks.y * nBricks.z;
            for (int i = lane; i < L::kWords; i += 32)
                acc[i] = 0.0f;
            __syncwarp();
            const int pBegin = blockIdx.y * viewsPerChunk;
            const int pEnd = min(det.np, pBegin + viewsPerChunk);
            for (int p = pBegin; p < pEnd; ++p) {
                const RayWindow w = windows[static_cast<int64_t>(p) * nb + bi];
                if (w.u0 > w.u1 || w.v0 > w.v1)
                    continue;
                const unsigned ax = viewAxes[p];
                if (ax & 1u)
                    siddonView<DIM, 0>(acc, w, p, m, rays, cpState, cpVoxel, nrays, y, det, org0,
                                       org1, org2, vol, binary);
                if (ax & 2u)
                    siddonView<DIM, 1>(acc, w, p, m, rays, cpState, cpVoxel, nrays, y, det, org0,
                                       org1, org2, vol, binary);
                if (DIM == 3 && (ax & 4u))
                    siddonView<DIM, DIM == 3 ? 2 : 0>(acc, w, p, m, rays, cpState, cpVoxel, nrays,
                                                      y, det, org0, org1, org2, vol, binary);
            }
            __syncwarp();
            const int64_t nvox = static_cast<int64_t>(vol.n[0]) * vol.n[1] * vol.n[2];
            float* out = x + blockIdx.y * nvox;
            for (int i = lane; i < kSlab * kSlab * L::kBz; i += 32) {
                const int lx = i % kSlab, ly = (i / kSlab) % kSlab, lz = i / (kSlab * kSlab);
                const int gx = org0 + lx, gy = org1 + ly, gz = org2 + lz;
                if (gx < vol.n[0] && gy < vol.n[1] && gz < vol.n[2])
                    out[gx + static_cast<int64_t>(vol.n[0]) *
                                 (gy + static_cast<int64_t>(vol.n[1]) * gz)] =
                        acc[lz * L::kPlane + ly * L::kRow + lx];
            }
        }

        // ---------------------------------------------------------------------------------------
        // 3D brick-owner adjoint on axis bricks: per driving axis G present, bricks one checkpoint
        // slab (kSlab planes) deep along G, kAxisTW voxels along the non-driving axis over which
        // the rays of a detector row spread (the columns: stride 1 in shared memory, the lanes
        // spread along it) and kAxisTV along the other. A ray crossing a brick keeps most of its
        // visits inside it, and a warp's taps fall into different banks. Visits outside the brick
        // across the rays are predicated off. As the 16^3 kernel: one warp per (brick, chunk
        // entry), the window's rays class by class, each lane replaying one ray's visits of the
        // slab from its checkpoint.
        // ---------------------------------------------------------------------------------------
#ifndef ELSA_SIDDON_AXIS_TV
#define ELSA_SIDDON_AXIS_TV 8 // rows of a Siddon axis brick
#endif
        constexpr int kAxisTW = 32, kAxisTV = ELSA_SIDDON_AXIS_TV;
#ifndef ELSA_SIDDON_AXIS_BATCH
#define ELSA_SIDDON_AXIS_BATCH 1 // class rays per lane whose records are fetched together
                                 // (256^3 / 360 views: 1: 44.6 ms, 2: 50.6, 3: 50.3; the
                                 // records of the next ray prefetched instead: 44.4 ms)
#endif
#ifndef ELSA_SIDDON_NOZERO
#define ELSA_SIDDON_NOZERO 1 // 256^3 owner: 39.5 ms, against 41.3 ms reading 0 into skipped words
#endif
#ifndef ELSA_SIDDON_PLANE_ODD
#define ELSA_SIDDON_PLANE_ODD 0 // 1: plane stride padded to 1 modulo 32
#endif
        constexpr int kSiddonAxisBatch = ELSA_SIDDON_AXIS_BATCH;

        struct SiddonAxisBrick {
            static constexpr int kRow = kAxisTW + 1; // columns (+1: rows land in other banks)
            static constexpr int kPlaneMin = kRow * kAxisTV;
            // unpadded planes keep the brick at 16.9 KB (12 resident per SM instead of 11)
            static constexpr int kPlane =
                ELSA_SIDDON_PLANE_ODD ? kPlaneMin + ((33 - kPlaneMin % 32) % 32) : kPlaneMin;
            static constexpr int kWords = kPlane * kSlab;
        };

        // Brick edges of grid G (UB: columns along b) in volume axis order.
        template <int G, bool UB>
        __host__ __device__ constexpr int siddonAxisEdge(int axis)
        {
            return axis == G ? kSlab
                             : (axis == (G == 0 ? 1 : 0) ? (UB ? kAxisTV : kAxisTW)
                                                         : (UB ? kAxisTW : kAxisTV));
        }

        struct SiddonAxisJob {
            const SiddonRay* rays;
            const float4* cpState;
            const unsigned* cpVoxel;
            int64_t nrays;
            const float* y;
            const RayWindow* windows;
            const unsigned* viewAxes;
            const int2* chunks;
            int viewsPerChunk;
            VolumeShape vol;
            DetectorShape det;
            int m;
            int3 nBricks;
            int binary;
            float* out;
        };

        // Replays the visits of one ray inside the slab [kLo, kLo + kSlab) along G from its
        // checkpoint and adds y * weight to the visits inside the axis brick.
        template <int G, bool UB>
        __device__ __forceinline__ void splatAxisSegment(float* acc, float3 tDelta, int meta,
                                                         int kFirst, float4 cp, unsigned cpv,
                                                         float yv, int kLo, int orgA, int orgB,
                                                         const VolumeShape& vol, int binary)
        {
            using L = SiddonAxisBrick;
            constexpr int EA = UB ? kAxisTV : kAxisTW, EB = UB ? kAxisTW : kAxisTV;
            constexpr int SA = UB ? L::kRow : 1, SB = UB ? 1 : L::kRow;
            int a, b;
            nonDrivingAxes(G, a, b);
            const int dirG = ((meta >> (2 + G)) & 1) ? -1 : 1;
            const int kg = dirG > 0 ? max(kLo, kFirst) : min(kLo + kSlab - 1, kFirst);
            int c0, c1, c2;
            entryVoxel(G, kg, static_cast<int>(cpv & 0xffffu), static_cast<int>(cpv >> 16), c0,
                       c1, c2);
            const int s0 = axisStep(meta, 0), s1 = axisStep(meta, 1), s2 = axisStep(meta, 2);
            float T0 = cp.x, T1 = cp.y, T2 = cp.z;
            float tEntry = cp.w;
            // the walk stays inside the volume and the slab: along G the two tests are one,
            // kLo <= cg < min(kLo + kSlab, n_G)
            const int nA = a == 0 ? vol.n[0] : (a == 1 ? vol.n[1] : vol.n[2]);
            const int nB = b == 1 ? vol.n[1] : vol.n[2];
            const int nG = G == 0 ? vol.n[0] : (G == 1 ? vol.n[1] : vol.n[2]);
            const unsigned spanG = static_cast<unsigned>(min(kLo + kSlab, nG) - kLo);
            // software-pipelined: the word of a visit is read before the sum of the previous
            // visit (always another voxel) is written back
            int prevOff = 0;
            float prevVal = 0.0f, prevW = 0.0f;
            bool prevIn = false;
            for (int it = 0; it < 3 * kSlab + 3; ++it) {
                bool m0, m1, m2;
                const float tExit = nextCrossing<3>(T0, T1, T2, m0, m1, m2);
                const int c[3] = {c0, c1, c2};
                const int lg = c[G] - kLo, la = c[a] - orgA, lb = c[b] - orgB;
                const bool in = static_cast<unsigned>(la) < static_cast<unsigned>(EA) &&
                                static_cast<unsigned>(lb) < static_cast<unsigned>(EB);
                const int off = lg * L::kPlane + la * SA + lb * SB;
#if ELSA_SIDDON_NOZERO
                float val; // read only where used: its store carries the same flag
                if (in)
                    val = acc[off];
#else
                const float val = in ? acc[off] : 0.0f;
#endif
                if (prevIn)
                    acc[prevOff] = __fadd_rn(prevVal, __fmul_rn(yv, prevW));
                prevOff = off, prevVal = val, prevIn = in;
                prevW = binary ? 1.0f : __fsub_rn(tExit, tEntry);
                if (m0) {
                    c0 += s0;
                    T0 = __fadd_rn(T0, tDelta.x);
                }
                if (m1) {
                    c1 += s1;
                    T1 = __fadd_rn(T1, tDelta.y);
                }
                if (m2) {
                    c2 += s2;
                    T2 = __fadd_rn(T2, tDelta.z);
                }
                const int cn[3] = {c0, c1, c2};
                if (static_cast<unsigned>(cn[a]) >= static_cast<unsigned>(nA) ||
                    static_cast<unsigned>(cn[b]) >= static_cast<unsigned>(nB) ||
                    static_cast<unsigned>(cn[G] - kLo) >= spanG)
                    break;
                tEntry = tExit;
            }
            if (prevIn)
                acc[prevOff] = __fadd_rn(prevVal, __fmul_rn(yv, prevW));
        }

        template <int G, bool UB>
        __global__ void __launch_bounds__(32)
            siddonAxisKernel(SiddonAxisJob J, int entryBase)
        {
            using L = SiddonAxisBrick;
            __shared__ float acc[L::kWords];
            constexpr int EX = siddonAxisEdge<G, UB>(0), EY = siddonAxisEdge<G, UB>(1),
                          EZ = siddonAxisEdge<G, UB>(2);
            constexpr int SA = UB ? L::kRow : 1, SB = UB ? 1 : L::kRow;
            const int lane = threadIdx.x;
            const int bi = blockIdx.x;
            const int3 nb3 = J.nBricks;
            const int org[3] = {(bi % nb3.x) * EX, ((bi / nb3.x) % nb3.y) * EY,
                                (bi / (nb3.x * nb3.y)) * EZ};
            int a, b;
            nonDrivingAxes(G, a, b);
            const int kLo = org[G], kHi = kLo + kSlab - 1;
            const int nb = nb3.x * nb3.y * nb3.z;
            for (int i = lane; i < L::kWords; i += 32)
                acc[i] = 0.0f;
            __syncwarp();
            const int2 entry = J.chunks[entryBase + blockIdx.y];
            const int pBegin = entry.x * J.viewsPerChunk;
            const int pEnd = min(J.det.np, pBegin + J.viewsPerChunk);
            const int64_t cpRow = static_cast<int64_t>(kLo / kSlab + 1) * J.nrays;
            const int m = J.m;
            for (int p = pBegin; p < pEnd; ++p) {
                if (!(J.viewAxes[p] & (1u << G)))
                    continue;
                const RayWindow w = J.windows[static_cast<int64_t>(p) * nb + bi];
                if (w.u0 > w.u1 || w.v0 > w.v1)
                    continue;
                const int64_t viewBase = static_cast<int64_t>(J.det.nu) * J.det.nv * p;
                for (int ov = 0; ov < m; ++ov) {
                    const int vStart = w.v0 + ov;
                    const int nvc = vStart <= w.v1 ? (w.v1 - vStart) / m + 1 : 0;
                    for (int ou = 0; ou < m; ++ou) {
                        const int uStart = w.u0 + ou;
                        const int nuc = uStart <= w.u1 ? (w.u1 - uStart) / m + 1 : 0;
                        const int total = nuc * nvc;
                        const float invNuc = nuc > 0 ? 1.0f / static_cast<float>(nuc) : 0.0f;
                        constexpr int kB = kSiddonAxisBatch;
                        for (int base = lane; base < total; base += 32 * kB) {
                            // the records of kB class rays first, then their visits in turn
                            int4 q0[kB], q1[kB];
                            float4 cps[kB];
                            unsigned cpvs[kB];
                            float ys[kB];
#pragma unroll
                            for (int q = 0; q < kB; ++q) {
                                const int i = base + 32 * q;
                                q0[q].w = 0;
                                if (i < total) {
                                    // i / nuc by a float reciprocal: exact for i < 2^20,
                                    // nuc < 2^11
                                    const int iv = static_cast<int>(
                                        (static_cast<float>(i) + 0.5f) * invNuc);
                                    const int iu = i - iv * nuc;
                                    const int64_t r =
                                        viewBase + (uStart + iu * m) +
                                        static_cast<int64_t>(J.det.nu) * (vStart + iv * m);
                                    const int4* rp = reinterpret_cast<const int4*>(J.rays + r);
                                    q0[q] = __ldg(rp);     // tDelta[3], meta
                                    q1[q] = __ldg(rp + 1); // kFirst, kLast, cur[2]
                                    cps[q] = __ldg(J.cpState + cpRow + r);
                                    cpvs[q] = __ldg(J.cpVoxel + cpRow + r);
                                    ys[q] = __ldg(J.y + r);
                                }
                            }
#pragma unroll
                            for (int q = 0; q < kB; ++q) {
                                const int meta = q0[q].w;
                                if (!(meta & kActive) || (meta & 3) != G)
                                    continue;
                                if (max(q1[q].x, q1[q].y) < kLo || min(q1[q].x, q1[q].y) > kHi)
                                    continue;
                                const float3 td = make_float3(__int_as_float(q0[q].x),
                                                              __int_as_float(q0[q].y),
                                                              __int_as_float(q0[q].z));
                                splatAxisSegment<G, UB>(acc, td, meta, q1[q].x, cps[q], cpvs[q],
                                                        ys[q], kLo, org[a], org[b], J.vol,
                                                        J.binary);
                            }
                        }
                        __syncwarp();
                    }
                }
            }
            __syncwarp();
            const VolumeShape& vol = J.vol;
            const int64_t nvox = static_cast<int64_t>(vol.n[0]) * vol.n[1] * vol.n[2];
            float* dst = J.out + static_cast<int64_t>(entry.y) * nvox;
            for (int i = lane; i < EX * EY * EZ; i += 32) {
                const int lx = i % EX, ly = (i / EX) % EY, lz = i / (EX * EY);
                const int gx = org[0] + lx, gy = org[1] + ly, gz = org[2] + lz;
                if (gx < vol.n[0] && gy < vol.n[1] && gz < vol.n[2]) {
                    const int l[3] = {lx, ly, lz};
                    dst[gx + static_cast<int64_t>(vol.n[0]) *
                                 (gy + static_cast<int64_t>(vol.n[1]) * gz)] =
                        acc[l[G] * L::kPlane + l[a] * SA + l[b] * SB];
                }
            }
        }

        class SiddonProjector final : public Projector
        {
        public:
            // binary: BinaryMethod (kind 6), the same visits with weight 1
            SiddonProjector(const VolumeShape& vol, const DetectorShape& det,
                            const std::vector<PoseRecord>& poses, bool binary,
                            const CurvedDetector& curved)
                : Projector(binary ? 6 : 1, vol, det, poses), binary_(binary ? 1 : 0),
                  curved_(curved)
            {
                CurvedTables tables(vol.dim, det, curved); // used while setting up
                const int maxDim = std::max(vol_.n[0], std::max(vol_.n[1], vol_.n[2]));
                if (maxDim >= 65536)
                    throw Error(ELSA_ERROR_NOT_SUPPORTED,
                                "SiddonsMethod: volume edges must be below 65536 voxels");
                const int64_t nrays = rangeSize_;
                const int threads = 256;
                const unsigned blocks = static_cast<unsigned>((nrays + threads - 1) / threads);
                rays_ = std::make_unique<DeviceBuffer>(sizeof(SiddonRay) * nrays);
                DeviceBuffer lines(sizeof(SiddonLine) * nrays);
                siddonSetupKernel<<<blocks, threads>>>(dPoses_, vol_, det_, tables.planar(),
                                                       rays_->as<SiddonRay>(),
                                                       lines.as<SiddonLine>());
                ELSA_LAUNCH_CHECK("siddonSetupKernel");

                cpRows_ = maxDim / kSlab + 3;
                // per-view axis masks, the bad-spacing mask and a 64-bit visit counter
                const size_t words = static_cast<size_t>(det_.np) + 4;
                viewAxes_ = std::make_unique<DeviceBuffer>(sizeof(unsigned) * words);
                unsigned* dAxes = viewAxes_->as<unsigned>();
                ELSA_CUDA(cudaMemset(dAxes, 0, sizeof(unsigned) * words));
                unsigned* dBad = dAxes + det_.np;
                auto* dCount =
                    reinterpret_cast<unsigned long long*>(dAxes + ((det_.np + 2) & ~1));
                // last visited slice and visit count of every ray; the checkpoints themselves are
                // written once the brick-owner adjoint is selected (buildOwner)
                if (vol_.dim == 3)
                    siddonCheckpointKernel<3><<<blocks, threads>>>(
                        rays_->as<SiddonRay>(), nrays, vol_, cpRows_, nullptr, nullptr, dCount);
                else
                    siddonCheckpointKernel<2><<<blocks, threads>>>(
                        rays_->as<SiddonRay>(), nrays, vol_, cpRows_, nullptr, nullptr, dCount);
                ELSA_LAUNCH_CHECK("siddonCheckpointKernel");
                siddonClassCheckKernel<<<blocks, threads>>>(rays_->as<SiddonRay>(),
                                                            lines.as<SiddonLine>(), det_,
                                                            vol_.dim, dAxes, dBad);
                ELSA_LAUNCH_CHECK("siddonClassCheckKernel");
                unsigned bad = 0;
                unsigned long long count = 0;
                ELSA_CUDA(cudaMemcpy(&bad, dBad, sizeof(unsigned), cudaMemcpyDeviceToHost));
                ELSA_CUDA(cudaMemcpy(&count, dCount, sizeof(count), cudaMemcpyDeviceToHost));
                visits_ = static_cast<int64_t>(count);
                // class spacing of the brick-owner adjoint; 0 when neighbouring detector rays pass
                // within two voxels of each other even eight pixels apart (only the scatter
                // adjoint is available then)
                for (int m = kMinClass; m <= kMaxClass; ++m)
                    if (!((bad >> m) & 1u)) {
                        classSpacing_ = m;
                        break;
                    }
                const int bz = vol_.dim == 3 ? kSlab : 1;
                nBricks_ = make_int3((vol_.n[0] + kSlab - 1) / kSlab,
                                     (vol_.n[1] + kSlab - 1) / kSlab, (vol_.n[2] + bz - 1) / bz);
                adjointChunks_ = defaultChunks();
                // The deterministic brick-owner adjoint is the default wherever it exists (a
                // valid class spacing) and its per-(ray, slab) checkpoints (20 B each: about
                // 20 GB at 256^3 / 360 x 384^2) take at most a quarter of the device's memory and
                // half of what is free; otherwise the atomic scatter.
                if (classSpacing_ > 0) {
                    size_t freeBytes = 0, totalBytes = 0;
                    ELSA_CUDA(cudaMemGetInfo(&freeBytes, &totalBytes));
                    const double need = 20.0 * static_cast<double>(nrays) * cpRows_;
                    if (need <= 0.25 * static_cast<double>(totalBytes) &&
                        need <= 0.5 * static_cast<double>(freeBytes))
                        setKnob(kKnobAdjointScatter, 0);
                }
                ELSA_CUDA(cudaDeviceSynchronize());
            }

            void forward(const float* x, float* y, cudaStream_t s) override
            {
                const int64_t nrays = rangeSize_;
                const unsigned blocks =
                    static_cast<unsigned>((nrays + forwardThreads_ - 1) / forwardThreads_);
                if (vol_.dim == 3)
                    siddonForwardKernel<3><<<blocks, forwardThreads_, 0, s>>>(
                        rays_->as<SiddonRay>(), nrays, x, vol_, binary_, y);
                else
                    siddonForwardKernel<2><<<blocks, forwardThreads_, 0, s>>>(
                        rays_->as<SiddonRay>(), nrays, x, vol_, binary_, y);
                ELSA_LAUNCH_CHECK("siddonForwardKernel");
            }

            void adjoint(const float* y, float* x, cudaStream_t s) override
            {
                if (scatter_) {
                    const int64_t nrays = rangeSize_;
                    const unsigned blocks =
                        static_cast<unsigned>((nrays + kScatterThreads - 1) / kScatterThreads);
                    ELSA_CUDA(cudaMemsetAsync(x, 0, sizeof(float) * domainSize_, s));
                    if (vol_.dim == 3)
                        siddonScatterKernel<3><<<blocks, kScatterThreads, 0, s>>>(
                            rays_->as<SiddonRay>(), nrays, y, vol_, binary_, x);
                    else
                        siddonScatterKernel<2><<<blocks, kScatterThreads, 0, s>>>(
                            rays_->as<SiddonRay>(), nrays, y, vol_, binary_, x);
                    ELSA_LAUNCH_CHECK("siddonScatterKernel");
                    return;
                }
                if (!cpState_)
                    throw Error(ELSA_ERROR_LOGIC, "SiddonsMethod: brick-owner adjoint not built");
                if (vol_.dim == 3) {
                    float* out = axisPartials_ > 1 ? partial_->as<float>() : x;
                    const int per = (det_.np + adjointChunks_ - 1) / adjointChunks_;
                    for (int g = 0; g < 3; ++g) {
                        const SiddonGrid& G = grids_[g];
                        if (!G.present || G.entryEnd <= G.entryBegin)
                            continue;
                        SiddonAxisJob J{};
                        J.rays = rays_->as<SiddonRay>();
                        J.cpState = cpState_->as<float4>();
                        J.cpVoxel = cpVoxel_->as<unsigned>();
                        J.nrays = rangeSize_;
                        J.y = y;
                        J.windows = G.windows->as<RayWindow>();
                        J.viewAxes = viewAxes_->as<unsigned>();
                        J.chunks = dEntries_->as<int2>() + G.entryBegin;
                        J.viewsPerChunk = per;
                        J.vol = vol_;
                        J.det = det_;
                        J.m = classSpacing_;
                        J.nBricks = G.nb;
                        J.binary = binary_;
                        J.out = out;
                        const dim3 grid(static_cast<unsigned>(G.nb.x * G.nb.y * G.nb.z),
                                        static_cast<unsigned>(G.entryEnd - G.entryBegin));
#define ELSA_SIDDON_AXIS(G_, UB_) siddonAxisKernel<G_, UB_><<<grid, 32, 0, s>>>(J, 0)
                        if (g == 0) {
                            if (G.ub)
                                ELSA_SIDDON_AXIS(0, true);
                            else
                                ELSA_SIDDON_AXIS(0, false);
                        } else if (g == 1) {
                            if (G.ub)
                                ELSA_SIDDON_AXIS(1, true);
                            else
                                ELSA_SIDDON_AXIS(1, false);
                        } else {
                            if (G.ub)
                                ELSA_SIDDON_AXIS(2, true);
                            else
                                ELSA_SIDDON_AXIS(2, false);
                        }
#undef ELSA_SIDDON_AXIS
                        ELSA_LAUNCH_CHECK("siddonAxisKernel");
                    }
                    if (axisPartials_ > 1)
                        launchSumChunks(partial_->as<float>(), axisPartials_, domainSize_, x, s);
                    return;
                }
                const int nb = nBricks_.x * nBricks_.y * nBricks_.z;
                const int per = (det_.np + adjointChunks_ - 1) / adjointChunks_;
                const int used = (det_.np + per - 1) / per;
                const dim3 grid(static_cast<unsigned>(nb), static_cast<unsigned>(used));
                float* out = used > 1 ? partial_->as<float>() : x;
                // 2D: square bricks (3D volumes take the axis bricks above)
                siddonAdjointKernel<2><<<grid, 32, 0, s>>>(
                    rays_->as<SiddonRay>(), cpState_->as<float4>(), cpVoxel_->as<unsigned>(),
                    rangeSize_, y, windows_->as<RayWindow>(), viewAxes_->as<unsigned>(), vol_,
                    det_, classSpacing_, nBricks_, per, binary_, out);
                ELSA_LAUNCH_CHECK("siddonAdjointKernel");
                if (used > 1)
                    launchSumChunks(partial_->as<float>(), used, domainSize_, x, s);
            }

            int64_t info(int key) const override
            {
                switch (key) {
                case 0:
                    return classSpacing_;
                case 1: // bricks of the brick-owner adjoint (3D: over the axis grids)
                    if (vol_.dim == 3) {
                        int64_t n = 0;
                        for (const SiddonGrid& g : grids_)
                            if (g.present)
                                n += static_cast<int64_t>(g.nb.x) * g.nb.y * g.nb.z;
                        return n;
                    }
                    return static_cast<int64_t>(nBricks_.x) * nBricks_.y * nBricks_.z;
                case 2:
                    return visits_;
                case 3:
                    return 0;
                case 6: // kernel launches per forward call
                    return 1;
                case 7: // kernel launches per adjoint call (brick owner in 3D: one per axis
                        // grid; with several partial volumes: + the chunk sum)
                    if (scatter_)
                        return 1;
                    if (vol_.dim == 3) {
                        int n = 0;
                        for (const SiddonGrid& g : grids_)
                            n += g.present && g.entryEnd > g.entryBegin ? 1 : 0;
                        return n + (axisPartials_ > 1 ? 1 : 0);
                    }
                    return adjointChunks_ > 1 ? 2 : 1;
                case 8: // visits outside the windows of their bricks (brick-owner adjoint only;
                        // test support; synchronizes)
                    return windowMisses();
                default:
                    return -1;
                }
            }

            int64_t windowMisses() const
            {
                if (!cpState_)
                    return -1;
                DeviceBuffer count(sizeof(unsigned long long));
                ELSA_CUDA(cudaMemset(count.as<unsigned long long>(), 0, sizeof(unsigned long long)));
                const int64_t nrays = rangeSize_;
                const unsigned blocks = static_cast<unsigned>((nrays + 255) / 256);
                const int bz = vol_.dim == 3 ? kSlab : 1;
                if (vol_.dim == 3)
                    for (int g = 0; g < 3; ++g) {
                        if (!grids_[g].present)
                            continue;
                        siddonWindowCheckKernel<3><<<blocks, 256>>>(
                            rays_->as<SiddonRay>(), grids_[g].windows->as<RayWindow>(), vol_,
                            det_, grids_[g].edge, grids_[g].nb, g,
                            count.as<unsigned long long>());
                    }
                else
                    siddonWindowCheckKernel<2><<<blocks, 256>>>(
                        rays_->as<SiddonRay>(), windows_->as<RayWindow>(), vol_, det_,
                        make_int3(kSlab, kSlab, bz), nBricks_, -1,
                        count.as<unsigned long long>());
                ELSA_LAUNCH_CHECK("siddonWindowCheckKernel");
                unsigned long long h = 0;
                ELSA_CUDA(cudaMemcpy(&h, count.as<unsigned long long>(), sizeof(h),
                                     cudaMemcpyDeviceToHost));
                return static_cast<int64_t>(h);
            }

            std::vector<int> knobCandidates(int knob) const override
            {
                if (knob == kKnobAdjointChunks) {
                    if (scatter_)
                        return {}; // chunks only exist in the brick-owner adjoint
                    // partial volumes limited to 4 GiB
                    const int64_t byMemory =
                        std::max<int64_t>(1, (int64_t(1) << 32) / (4 * domainSize_));
                    const int limit = static_cast<int>(
                        std::min<int64_t>(std::min<int64_t>(det_.np, 256), byMemory));
                    return chunkCandidates(limit, std::min(limit, defaultChunks()));
                }
                if (knob == kKnobForwardThreads)
                    return {64, 128, 256, 512};
                if (knob == kKnobAdjointScatter)
                    return classSpacing_ > 0 ? std::vector<int>{0, 1} : std::vector<int>{1};
                return {};
            }

            int knob(int knob) const override
            {
                if (knob == kKnobAdjointChunks)
                    return adjointChunks_;
                if (knob == kKnobForwardThreads)
                    return forwardThreads_;
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
                                "SiddonsMethod: value " + std::to_string(value) +
                                    " is not a candidate of knob " + std::to_string(knob));
                }
                if (knob == kKnobForwardThreads) {
                    forwardThreads_ = value;
                    return;
                }
                if (knob == kKnobAdjointScatter) {
                    if (value == 0)
                        buildOwner();
                    else
                        releaseOwner();
                    scatter_ = value;
                } else {
                    adjointChunks_ = value;
                }
                // the partial volumes exist only while the brick-owner adjoint uses chunks (3D:
                // one per (chunk, axis grid) pair)
                int volumes = adjointChunks_;
                if (!scatter_ && vol_.dim == 3)
                    volumes = buildAxisEntries();
                const size_t need = sizeof(float) * static_cast<size_t>(domainSize_) *
                                    static_cast<size_t>(volumes);
                if (scatter_ || volumes <= 1)
                    partial_.reset();
                else if (!partial_ || partial_->bytes() < need) {
                    partial_.reset();
                    partial_ = std::make_unique<DeviceBuffer>(need);
                }
            }

        private:
            // Per-(ray, slab) checkpoints (16 + 4 bytes per ray and slab: about 20 GB at
            // 256^3 / 360 x 384^2) and per-(brick, view) ray windows of the brick-owner adjoint,
            // built when that adjoint is selected and released when the scatter adjoint is.
            void buildOwner()
            {
                if (cpState_)
                    return;
                const int64_t nrays = rangeSize_;
                const int threads = 256;
                const unsigned blocks = static_cast<unsigned>((nrays + threads - 1) / threads);
                cpState_ = std::make_unique<DeviceBuffer>(sizeof(float4) * nrays * cpRows_);
                cpVoxel_ = std::make_unique<DeviceBuffer>(sizeof(unsigned) * nrays * cpRows_);
                if (vol_.dim == 3)
                    siddonCheckpointKernel<3><<<blocks, threads>>>(
                        rays_->as<SiddonRay>(), nrays, vol_, cpRows_, cpState_->as<float4>(),
                        cpVoxel_->as<unsigned>(), nullptr);
                else
                    siddonCheckpointKernel<2><<<blocks, threads>>>(
                        rays_->as<SiddonRay>(), nrays, vol_, cpRows_, cpState_->as<float4>(),
                        cpVoxel_->as<unsigned>(), nullptr);
                ELSA_LAUNCH_CHECK("siddonCheckpointKernel");
                CurvedTables tables(vol_.dim, det_, curved_);
                if (vol_.dim == 3) {
                    buildAxisGrids(tables.map());
                    ELSA_CUDA(cudaDeviceSynchronize());
                    return;
                }
                const int bz = vol_.dim == 3 ? kSlab : 1;
                const int64_t nwin =
                    static_cast<int64_t>(nBricks_.x) * nBricks_.y * nBricks_.z * det_.np;
                windows_ = std::make_unique<DeviceBuffer>(sizeof(RayWindow) * nwin);
                // Siddon visits exactly the voxels a ray crosses: the window is the projection
                // of the brick itself, grown by kWindowSlack for the rounding of the float rays
                launchBrickWindows(dPoses_, vol_, det_, make_int3(kSlab, kSlab, bz), nBricks_,
                                   windows_->as<RayWindow>(), nullptr, tables.map(),
                                   kWindowSlack, kWindowPixelMargin);
                ELSA_CUDA(cudaDeviceSynchronize());
            }

            void releaseOwner()
            {
                ELSA_CUDA(cudaDeviceSynchronize());
                cpState_.reset();
                cpVoxel_.reset();
                windows_.reset();
                for (SiddonGrid& g : grids_)
                    g = SiddonGrid{};
                dEntries_.reset();
                axisPartials_ = 0;
            }

            // ---- 3D brick-owner adjoint on axis bricks ----
            struct SiddonGrid {
                bool present = false;
                bool ub = false; // columns along b instead of a
                int3 edge{}, nb{};
                std::unique_ptr<DeviceBuffer> windows;
                int entryBegin = 0, entryEnd = 0;
            };
            SiddonGrid grids_[3];
            std::vector<unsigned> viewAxesHost_;
            std::vector<int2> entries_;
            std::unique_ptr<DeviceBuffer> dEntries_;
            int axisPartials_ = 0;

            // Per view and driving axis g: true when neighbouring pixels of the centre detector
            // row spread more along b than along a on the planes of g.
            bool rowAlongB(int p, int g) const
            {
                const float* P = poses_[p].v + kPoseOffPinv;
                const float uc = det_.nu / 2 + 0.5f, vc = det_.nv / 2 + 0.5f;
                float D[3], E[3];
                for (int i = 0; i < 3; ++i) {
                    D[i] = P[i * 3] * uc + P[i * 3 + 1] * vc + P[i * 3 + 2];
                    E[i] = P[i * 3] * (uc + 1.0f) + P[i * 3 + 1] * vc + P[i * 3 + 2];
                }
                int a, b;
                nonDrivingAxes(g, a, b);
                if (std::fabs(D[g]) == 0.0f || std::fabs(E[g]) == 0.0f)
                    return false;
                const float da = std::fabs(E[a] / std::fabs(E[g]) - D[a] / std::fabs(D[g]));
                const float db = std::fabs(E[b] / std::fabs(E[g]) - D[b] / std::fabs(D[g]));
                return db > da;
            }

            void buildAxisGrids(CurvedMap cm)
            {
                viewAxesHost_.resize(det_.np);
                ELSA_CUDA(cudaMemcpy(viewAxesHost_.data(), viewAxes_->as<unsigned>(),
                                     sizeof(unsigned) * det_.np, cudaMemcpyDeviceToHost));
                for (int g = 0; g < 3; ++g) {
                    SiddonGrid& G = grids_[g];
                    int votes = 0, alongB = 0;
                    for (int p = 0; p < det_.np; ++p)
                        if ((viewAxesHost_[p] >> g) & 1u) {
                            ++votes;
                            alongB += rowAlongB(p, g) ? 1 : 0;
                        }
                    G.present = votes > 0;
                    if (!G.present)
                        continue;
                    G.ub = 2 * alongB > votes;
                    int a, b;
                    nonDrivingAxes(g, a, b);
                    int e[3];
                    e[g] = kSlab;
                    e[a] = G.ub ? kAxisTV : kAxisTW;
                    e[b] = G.ub ? kAxisTW : kAxisTV;
                    G.edge = make_int3(e[0], e[1], e[2]);
                    G.nb = make_int3((vol_.n[0] + e[0] - 1) / e[0], (vol_.n[1] + e[1] - 1) / e[1],
                                     (vol_.n[2] + e[2] - 1) / e[2]);
                    const int64_t nwin = static_cast<int64_t>(G.nb.x) * G.nb.y * G.nb.z * det_.np;
                    G.windows = std::make_unique<DeviceBuffer>(sizeof(RayWindow) * nwin);
                    launchBrickWindows(dPoses_, vol_, det_, G.edge, G.nb,
                                       G.windows->as<RayWindow>(), nullptr, cm, kWindowSlack,
                                       kWindowPixelMargin);
                }
            }

            // (chunk, partial volume) entries per grid for adjointChunks_ view chunks (the
            // chunks holding a view that drives along the grid's axis), partial volumes numbered
            // by (chunk, axis); returns their number.
            int buildAxisEntries()
            {
                const int per = (det_.np + adjointChunks_ - 1) / adjointChunks_;
                const int used = (det_.np + per - 1) / per;
                std::vector<std::vector<int2>> byGrid(3);
                int next = 0;
                for (int c = 0; c < used; ++c)
                    for (int g = 0; g < 3; ++g) {
                        if (!grids_[g].present)
                            continue;
                        bool any = false;
                        for (int p = c * per; p < std::min(det_.np, (c + 1) * per) && !any; ++p)
                            any = (viewAxesHost_[p] >> g) & 1u;
                        if (any)
                            byGrid[g].push_back(make_int2(c, next++));
                    }
                entries_.clear();
                for (int g = 0; g < 3; ++g) {
                    grids_[g].entryBegin = static_cast<int>(entries_.size());
                    entries_.insert(entries_.end(), byGrid[g].begin(), byGrid[g].end());
                    grids_[g].entryEnd = static_cast<int>(entries_.size());
                }
                if (next == 1)
                    for (auto& e : entries_)
                        e.y = 0;
                dEntries_ = std::make_unique<DeviceBuffer>(sizeof(int2) *
                                                           std::max<size_t>(1, entries_.size()));
                if (!entries_.empty())
                    ELSA_CUDA(cudaMemcpy(dEntries_->as<int2>(), entries_.data(),
                                         sizeof(int2) * entries_.size(), cudaMemcpyHostToDevice));
                axisPartials_ = next;
                return next;
            }

            // View chunks: enough for bricks x chunks to reach kAdjointWarpsPerSm one-warp CTAs
            // per SM and at least kMinAdjointChunks, within kChunkMemory of partial volumes
            // (256^3 / 360 views: 103.8 ms with 1 chunk, 85.5 with 32).
            int defaultChunks() const
            {
                const int nb = nBricks_.x * nBricks_.y * nBricks_.z;
                const int want = std::max((kAdjointWarpsPerSm * 148 + nb - 1) / nb,
                                          kMinAdjointChunks);
                const int64_t cap = std::max<int64_t>(1, kChunkMemory / (4 * domainSize_));
                return static_cast<int>(
                    std::max<int64_t>(1, std::min<int64_t>(std::min<int64_t>(want, det_.np), cap)));
            }

            std::unique_ptr<DeviceBuffer> partial_; // adjoint: per view-chunk partial volumes
            int adjointChunks_ = 1;
            int scatter_ = 1; // until the constructor selects the brick owner (see there)
            int forwardThreads_ = kForwardThreads;
            int binary_ = 0;
            CurvedDetector curved_;
            std::unique_ptr<DeviceBuffer> rays_, cpState_, cpVoxel_, viewAxes_, windows_;
            int cpRows_ = 0;
            int classSpacing_ = 0;
            int64_t visits_ = 0;
            int3 nBricks_{};
        };
    } // namespace

    std::unique_ptr<Projector> makeSiddonProjector(const VolumeShape& vol,
                                                   const DetectorShape& det,
                                                   const std::vector<PoseRecord>& poses,
                                                   bool binary, const CurvedDetector& curved)
    {
        return std::make_unique<SiddonProjector>(vol, det, poses, binary, curved);
    }
} // namespace elsa_b200
