// TMA-staged, plane-synchronous forward projection for 3D Joseph on sm_100a.
//
// A CTA owns a kTileU x kTileV tile of detector pixels of one view; thread = ray. When every ray
// of the tile has the same driving axis g and direction, the tile's rays cross the planes of g in
// lockstep. The volume is read from a copy laid out [g][slow][fast], where `fast` is the
// non-driving axis along which neighbouring pixels of a detector row spread, so a warp (32
// neighbouring rays) reads consecutive words. Chunks of kBoxD planes are staged into shared
// memory by one cp.async.bulk.tensor.3d per chunk (kStages-deep mbarrier pipeline); taps outside
// the volume read the TMA zero fill, which matches the reference's masked taps
// (projectors/JosephsMethod.cpp:60-97). Box origins per (tile, chunk) are computed once per
// geometry from the same accumulated sample positions the kernel uses, so every tap is inside its
// box; tiles whose rays disagree on axis or direction, or do not fit the box, use the per-ray
// gather (the same arithmetic as josephForwardKernel).
//
// All waits on mbarriers are bounded (about one second of clock cycles by default); on timeout the
// CTA records bit 0 of the error word, waits (bounded again) for the copies it has issued and
// not yet consumed, and returns. For tests of that path, setWaitTest() shortens the limit and can
// withhold the copies (the barriers then expect bytes that never arrive), so the waits run out
// without any fault.
#include "joseph_tma.cuh"

#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>

namespace elsa_b200
{
    namespace
    {
        constexpr int TU = JosephForwardTma::kTileU, TV = JosephForwardTma::kTileV;
        constexpr int BW = JosephForwardTma::kBoxW, BH = JosephForwardTma::kBoxH;
        constexpr int BD = JosephForwardTma::kBoxD, NS = JosephForwardTma::kStages;
        constexpr int NT = JosephForwardTma::kThreads;
        constexpr int kStageFloats = BW * BH * BD;
        constexpr unsigned kStageBytes = kStageFloats * sizeof(float);
        constexpr int kFlagFallback = 8;
#ifndef ELSA_FWD_FULLCHUNK
#define ELSA_FWD_FULLCHUNK 1 // warp-uniform fast path for chunks without partial rays
#endif
#ifndef ELSA_FWD_NOCLAMP
#define ELSA_FWD_NOCLAMP 1 // taps indexed without clamps (in range by construction)
#endif

#ifndef ELSA_FWD_PAIR_ACC
#define ELSA_FWD_PAIR_ACC 1 // the two footprint rows summed separately, one packed fma per sample
                            // (256^3: 10.61 -> 10.49 ms)
#endif
#ifndef ELSA_FWD_PACKED
#define ELSA_FWD_PACKED 1 // the (fast, slow) pairs on the packed two-wide FP32 instructions
                          // (256^3: 12.04 -> 10.59 ms)
#endif
#ifndef ELSA_FWD_MAGIC_FLOOR
#define ELSA_FWD_MAGIC_FLOOR 1
#endif
        // floor of a tap coordinate and its integer: floorSmall on the FMA and integer pipes
        // (the conversion pipe is 62 % busy in this kernel otherwise; 256^3: 12.27 -> 12.04 ms),
        // or floorf and a conversion with ELSA_FWD_MAGIC_FLOOR 0; the same values.
        [[maybe_unused]] __device__ __forceinline__ float floorTap(float x, int& i)
        {
#if ELSA_FWD_MAGIC_FLOOR
            return floorSmall(x, i);
#else
            const float f = floorf(x);
            i = static_cast<int>(f);
            return f;
#endif
        }

        // Tap index along a box edge of E words. The box origins of every (tile, chunk) come from
        // the same accumulated positions (tileSetupKernel: identical float operations, and a tile
        // whose samples do not fit its boxes takes the per-ray gather), so i is in [0, E - 2] by
        // construction and needs no clamp; ELSA_FWD_NOCLAMP 0 clamps it anyway.
        // 256^3 / 360 views: 14.55 ms clamped, 13.84 ms without; 12.27 ms with the full-chunk
        // fast path as well.
        template <int E>
        __device__ __forceinline__ int boxIndex(int i)
        {
            return ELSA_FWD_NOCLAMP ? i : min(max(i, 0), E - 2);
        }

        __device__ __forceinline__ int floorDivI(int a, int b)
        {
            return a >= 0 ? a / b : -((-a + b - 1) / b);
        }

        __device__ __forceinline__ uint32_t smemAddr(const void* p)
        {
            return static_cast<uint32_t>(__cvta_generic_to_shared(p));
        }

        __device__ __forceinline__ void mbarInit(uint64_t* bar, unsigned count)
        {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(bar)),
                         "r"(count)
                         : "memory");
        }

        __device__ __forceinline__ void mbarExpectTx(uint64_t* bar, unsigned bytes)
        {
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                             smemAddr(bar)),
                         "r"(bytes)
                         : "memory");
        }

        __device__ __forceinline__ bool mbarTryWait(uint64_t* bar, unsigned parity)
        {
            unsigned ok;
            asm volatile("{\n\t.reg .pred p;\n\t"
                         "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                         "selp.u32 %0, 1, 0, p;\n\t}"
                         : "=r"(ok)
                         : "r"(smemAddr(bar)), "r"(parity)
                         : "memory");
            return ok != 0;
        }

        // Bounded wait of at most `limit` clock cycles; false on timeout.
        __device__ __forceinline__ bool mbarWait(uint64_t* bar, unsigned parity, long long limit)
        {
            if (mbarTryWait(bar, parity))
                return true;
            const long long t0 = clock64();
            while (!mbarTryWait(bar, parity)) {
                if (clock64() - t0 > limit)
                    return false;
            }
            return true;
        }

        // Box (c0, c1, c2) of batch element c3 of the permuted copies (a 4D tensor map whose
        // slowest dimension is the batch element; the box is one element deep there).
        __device__ __forceinline__ void tmaLoad4d(float* dst, const CUtensorMap* map, int c0,
                                                  int c1, int c2, int c3, uint64_t* bar)
        {
            asm volatile(
                "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smemAddr(dst)),
                "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
                "r"(smemAddr(bar))
                : "memory");
        }

        // out[(k * nSlow + s) * padFast + f] = x(axis values), zero in the padding columns.
        // blockIdx.y: batch element (x + b xStride into copy b of out)
        __global__ void permuteKernel(const float* __restrict__ x, VolumeShape vol, int g, int sAx,
                                      int fAx, int padFast, float* __restrict__ out,
                                      int64_t xStride)
        {
            const int nf = vol.n[fAx], ns = vol.n[sAx], ng = vol.n[g];
            const int64_t total = static_cast<int64_t>(padFast) * ns * ng;
            x += blockIdx.y * xStride;
            out += blockIdx.y * total;
            const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
            for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
                 i < total; i += stride) {
                const int f = static_cast<int>(i % padFast);
                const int s = static_cast<int>((i / padFast) % ns);
                const int k = static_cast<int>(i / (static_cast<int64_t>(padFast) * ns));
                float v = 0.0f;
                if (f < nf) {
                    int c[3];
                    c[g] = k, c[sAx] = s, c[fAx] = f;
                    v = __ldg(x + c[0] + static_cast<int64_t>(vol.n[0]) *
                                             (c[1] + static_cast<int64_t>(vol.n[1]) * c[2]));
                }
                out[i] = v;
            }
        }

        struct RayCursor {
            float pf, ps, sf, ss; // fast/slow position and step
            int t0, n;            // first plane index of the ray in tile order, sample count
        };

        __device__ __forceinline__ RayCursor cursorOf(const JosephRay& R, int fastIsA, int kStart,
                                                      int dir)
        {
            RayCursor c;
            c.pf = fastIsA ? R.pa : R.pb;
            c.ps = fastIsA ? R.pb : R.pa;
            c.sf = fastIsA ? R.sa : R.sb;
            c.ss = fastIsA ? R.sb : R.sa;
            c.t0 = (R.k0 - kStart) * dir;
            c.n = R.n;
            return c;
        }

        // Per tile: uniformity of axis/direction, plane range, and the box origin of every chunk
        // from the exact accumulated sample positions (min/max over the tile's samples).
        __global__ void __launch_bounds__(NT)
            tileSetupKernel(const JosephRay* __restrict__ rays, DetectorShape det, int tilesU,
                            int tilesV, int3 fastAxis, int maxChunks,
                            ForwardTile* __restrict__ tiles, int2* __restrict__ origins,
                            unsigned* __restrict__ fallbackCount)
        {
            constexpr int kMaxChunksSmem = 128;
            __shared__ int axisMask, dirMask, kMin, kMax, tEnd;
            __shared__ int minF[kMaxChunksSmem], maxF[kMaxChunksSmem], minS[kMaxChunksSmem],
                maxS[kMaxChunksSmem];
            __shared__ int bad;
            const int tile = blockIdx.x;
            const int p = tile / (tilesU * tilesV);
            const int tu = tile % tilesU, tv = (tile / tilesU) % tilesV;
            const int u = tu * TU + threadIdx.x % TU, v = tv * TV + threadIdx.x / TU;
            const bool valid = u < det.nu && v < det.nv;
            JosephRay R{};
            if (valid)
                R = rays[u + static_cast<int64_t>(det.nu) * (v + static_cast<int64_t>(det.nv) * p)];
            const bool live = valid && R.n > 0;
            if (threadIdx.x == 0) {
                axisMask = 0, dirMask = 0, kMin = 1 << 30, kMax = -(1 << 30), tEnd = 0, bad = 0;
            }
            for (int i = threadIdx.x; i < kMaxChunksSmem; i += NT) {
                minF[i] = 1 << 30, maxF[i] = -(1 << 30), minS[i] = 1 << 30, maxS[i] = -(1 << 30);
            }
            __syncthreads();
            if (live) {
                atomicOr(&axisMask, 1 << (R.meta & 3));
                atomicOr(&dirMask, (R.meta & 4) ? 2 : 1);
                atomicMin(&kMin, R.k0);
                atomicMax(&kMax, R.k0);
            }
            __syncthreads();
            const int g = axisMask == 4 ? 2 : (axisMask == 2 ? 1 : 0);
            const bool uniform = (axisMask == 1 || axisMask == 2 || axisMask == 4) &&
                                 (dirMask == 1 || dirMask == 2);
            const int dir = dirMask == 2 ? -1 : 1;
            const int kStart = dir > 0 ? kMin : kMax;
            int a, b;
            nonDrivingAxes(g, a, b);
            const int fast = g == 0 ? fastAxis.x : (g == 1 ? fastAxis.y : fastAxis.z);
            const bool fastIsA = fast == a;
            RayCursor c{};
            if (live && uniform) {
                c = cursorOf(R, fastIsA, kStart, dir);
                atomicMax(&tEnd, c.t0 + c.n);
            }
            __syncthreads();
            const int nChunks = (tEnd + BD - 1) / BD;
            const bool chunksOk = uniform && nChunks <= kMaxChunksSmem && nChunks <= maxChunks;
            if (live && chunksOk) {
                float pf = c.pf, ps = c.ps;
                for (int j = 0; j < c.n; ++j) {
                    const int ch = (c.t0 + j) / BD;
                    const int fi = static_cast<int>(floorf(__fsub_rn(pf, 0.5f)));
                    const int si = static_cast<int>(floorf(__fsub_rn(ps, 0.5f)));
                    atomicMin(&minF[ch], fi);
                    atomicMax(&maxF[ch], fi + 1);
                    atomicMin(&minS[ch], si);
                    atomicMax(&maxS[ch], si + 1);
                    pf = __fadd_rn(pf, c.sf);
                    ps = __fadd_rn(ps, c.ss);
                }
            }
            __syncthreads();
            if (chunksOk) {
                for (int ch = threadIdx.x; ch < nChunks; ch += NT) {
                    int2 o = make_int2(0, 0);
                    if (minF[ch] <= maxF[ch]) {
                        o.x = floorDivI(minF[ch], 4) * 4;
                        o.y = minS[ch];
                        if (maxF[ch] - o.x > BW - 1 || maxS[ch] - o.y > BH - 1)
                            atomicOr(&bad, 1);
                    }
                    origins[static_cast<int64_t>(tile) * maxChunks + ch] = o;
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                ForwardTile t;
                t.kStart = kStart;
                t.nChunks = nChunks;
                const bool fallback = !chunksOk || bad || axisMask == 0;
                t.flags = g | (dir < 0 ? 4 : 0) | (fallback ? kFlagFallback : 0);
                t.pad = 0;
                tiles[tile] = t;
                if (fallback && axisMask != 0)
                    atomicAdd(fallbackCount, 1u);
            }
        }

        // The per-ray gather (fallback tiles): the arithmetic of josephForwardKernel.
        __device__ float gatherRay(const JosephRay& R, const float* __restrict__ x,
                                   const VolumeShape& vol)
        {
            const int g = R.meta & 3;
            const int dir = (R.meta & 4) ? -1 : 1;
            int a, b;
            nonDrivingAxes(g, a, b);
            const int64_t plane = static_cast<int64_t>(vol.n[0]) * vol.n[1];
            const int64_t sg = g == 0 ? 1 : (g == 1 ? vol.n[0] : plane);
            const int64_t sa = a == 0 ? 1 : (a == 1 ? vol.n[0] : plane);
            const int ng = g == 0 ? vol.n[0] : (g == 1 ? vol.n[1] : vol.n[2]);
            const int na = a == 0 ? vol.n[0] : (a == 1 ? vol.n[1] : vol.n[2]);
            const int64_t sb = b == 1 ? vol.n[0] : plane;
            const int nb = b == 1 ? vol.n[1] : vol.n[2];
            float acc = 0.0f;
            float pa = R.pa, pb = R.pb;
            int k = R.k0;
            for (int j = 0; j < R.n; ++j, k += dir, pa = __fadd_rn(pa, R.sa),
                     pb = __fadd_rn(pb, R.sb)) {
                if (static_cast<unsigned>(k) >= static_cast<unsigned>(ng))
                    continue;
                const float fa = floorf(__fsub_rn(pa, 0.5f)), fb = floorf(__fsub_rn(pb, 0.5f));
                const float cwa = __fsub_rn(__fsub_rn(pa, fa), 0.5f);
                const float cwb = __fsub_rn(__fsub_rn(pb, fb), 0.5f);
                const float wa = __fsub_rn(1.0f, cwa), wb = __fsub_rn(1.0f, cwb);
                const int ia = static_cast<int>(fa), ib = static_cast<int>(fb);
                const bool a0 = static_cast<unsigned>(ia) < static_cast<unsigned>(na);
                const bool a1 = static_cast<unsigned>(ia + 1) < static_cast<unsigned>(na);
                const bool b0 = static_cast<unsigned>(ib) < static_cast<unsigned>(nb);
                const bool b1 = static_cast<unsigned>(ib + 1) < static_cast<unsigned>(nb);
                const float* p0 = x + k * sg + ia * sa + ib * sb;
                const float v00 = (a0 && b0) ? __ldg(p0) : 0.0f;
                const float v10 = (a1 && b0) ? __ldg(p0 + sa) : 0.0f;
                const float v01 = (a0 && b1) ? __ldg(p0 + sb) : 0.0f;
                const float v11 = (a1 && b1) ? __ldg(p0 + sa + sb) : 0.0f;
                acc += wb * (wa * v00 + cwa * v10) + cwb * (wa * v01 + cwa * v11);
            }
            return R.len * acc;
        }

        __global__ void __launch_bounds__(NT)
            forwardTmaKernel(const __grid_constant__ CUtensorMap map0,
                             const __grid_constant__ CUtensorMap map1,
                             const __grid_constant__ CUtensorMap map2,
                             const JosephRay* __restrict__ rays,
                             const ForwardTile* __restrict__ tiles,
                             const int2* __restrict__ origins, int maxChunks,
                             const float* __restrict__ x, VolumeShape vol, DetectorShape det,
                             int tilesU, int tilesV, int3 fastAxis, float* __restrict__ y,
                             unsigned* __restrict__ error, int tileBase, long long waitCycles,
                             int withhold, int64_t xStride, int64_t yStride)
        {
            // blockIdx.y: batch element (volume x + b xStride, sinogram y + b yStride)
            const int batch = static_cast<int>(blockIdx.y);
            x += batch * xStride;
            y += batch * yStride;
            extern __shared__ __align__(128) float stage[];
            __shared__ __align__(8) uint64_t full[NS];
            __shared__ int abortFlag;
            const int tile = tileBase + blockIdx.x; // tiles are view-major
            const int p = tile / (tilesU * tilesV);
            const int tu = tile % tilesU, tv = (tile / tilesU) % tilesV;
            const int u = tu * TU + threadIdx.x % TU, v = tv * TV + threadIdx.x / TU;
            const bool valid = u < det.nu && v < det.nv;
            const int64_t r = u + static_cast<int64_t>(det.nu) * (v + static_cast<int64_t>(det.nv) * p);
            JosephRay R{};
            if (valid)
                R = rays[r];
            const ForwardTile T = tiles[tile];
            if (T.flags & kFlagFallback) {
                if (valid)
                    y[r] = R.n > 0 ? gatherRay(R, x, vol) : 0.0f;
                return;
            }
            const int g = T.flags & 3;
            const int dir = (T.flags & 4) ? -1 : 1;
            const CUtensorMap* map = g == 0 ? &map0 : (g == 1 ? &map1 : &map2);
            int a, b;
            nonDrivingAxes(g, a, b);
            const int fast = g == 0 ? fastAxis.x : (g == 1 ? fastAxis.y : fastAxis.z);
            RayCursor c = cursorOf(R, fast == a, T.kStart, dir);
            if (!valid)
                c.n = 0;
            const int2* org = origins + static_cast<int64_t>(tile) * maxChunks;
            if (threadIdx.x == 0) {
                abortFlag = 0;
                for (int i = 0; i < NS; ++i)
                    mbarInit(&full[i], 1);
                asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            }
            __syncthreads();
            // box origin along g of chunk ch: planes kStart + dir * (ch*BD .. ch*BD + BD-1)
            auto issue = [&](int ch) {
                const int s = ch % NS;
                const int2 o = org[ch];
                const int gOrg = dir > 0 ? T.kStart + ch * BD : T.kStart - ch * BD - (BD - 1);
                mbarExpectTx(&full[s], kStageBytes);
                if (!withhold) // test mode: the barrier waits for bytes that never come
                    tmaLoad4d(stage + s * kStageFloats, map, o.x, o.y, gOrg, batch, &full[s]);
            };
            if (threadIdx.x == 0)
                for (int ch = 0; ch < NS && ch < T.nChunks; ++ch)
                    issue(ch);
            float acc = 0.0f;
#if ELSA_FWD_PACKED
#if ELSA_FWD_PAIR_ACC
            float2 acc2 = make_float2(0.0f, 0.0f); // the two footprint rows' sums
#endif
            float2 p2 = make_float2(c.pf, c.ps); // (fast, slow) position
            const float2 s2 = make_float2(c.sf, c.ss);
#else
            float pf = c.pf, ps = c.ps;
#endif
            int failed = -1; // chunk whose wait timed out
            for (int ch = 0; ch < T.nChunks; ++ch) {
                const int s = ch % NS;
                const bool ready = mbarWait(&full[s], (ch / NS) & 1, waitCycles);
                if (!ready) {
                    atomicOr(error, 1u);
                    abortFlag = 1;
                }
                const int2 o = org[ch];
                const float* buf = stage + s * kStageFloats;
                const int jBase = ch * BD - c.t0;
#if ELSA_FWD_FULLCHUNK
                // chunks in which every ray of the warp has all BD samples: no per-sample test
                if (__all_sync(0xffffffffu, ready && jBase >= 0 && jBase + BD <= c.n)) {
#pragma unroll
                    for (int kk = 0; kk < BD; ++kk) {
#if ELSA_FWD_PACKED
                        // (f, s) pairs on the packed two-wide FP32 path: the same roundings
                        int fi, si;
                        const float2 h = make_float2(0.5f, 0.5f);
                        const float2 fl = floorSmall2(sub2(p2, h), fi, si);
                        const float2 cw = sub2(sub2(p2, fl), h);
                        const float2 w = sub2(make_float2(1.0f, 1.0f), cw);
                        const int lf = boxIndex<BW>(fi - o.x);
                        const int ls = boxIndex<BH>(si - o.y);
                        const int lk = dir > 0 ? kk : BD - 1 - kk;
                        const float* q = buf + (lk * BH + ls) * BW + lf;
                        // rows v0 and v1 of the footprint: (wf v00 + cwf v10, wf v01 + cwf v11)
                        const float2 r = fma2(make_float2(cw.x, cw.x), make_float2(q[1], q[BW + 1]),
                                              mul2(make_float2(w.x, w.x), make_float2(q[0], q[BW])));
#if ELSA_FWD_PAIR_ACC
                        acc2 = fma2(make_float2(w.y, cw.y), r, acc2);
#else
                        acc += w.y * r.x + cw.y * r.y;
#endif
                        p2 = add2(p2, s2);
#else
                        int fi, si;
                        const float ff = floorTap(__fsub_rn(pf, 0.5f), fi);
                        const float fs = floorTap(__fsub_rn(ps, 0.5f), si);
                        const float cwf = __fsub_rn(__fsub_rn(pf, ff), 0.5f);
                        const float cws = __fsub_rn(__fsub_rn(ps, fs), 0.5f);
                        const float wf = __fsub_rn(1.0f, cwf), ws = __fsub_rn(1.0f, cws);
                        const int lf = boxIndex<BW>(fi - o.x);
                        const int ls = boxIndex<BH>(si - o.y);
                        const int lk = dir > 0 ? kk : BD - 1 - kk;
                        const float* q = buf + (lk * BH + ls) * BW + lf;
                        const float v00 = q[0], v10 = q[1], v01 = q[BW], v11 = q[BW + 1];
                        acc += ws * (wf * v00 + cwf * v10) + cws * (wf * v01 + cwf * v11);
                        pf = __fadd_rn(pf, c.sf);
                        ps = __fadd_rn(ps, c.ss);
#endif
                    }
                } else
#endif
#pragma unroll
                for (int kk = 0; kk < BD; ++kk) {
                    const int j = jBase + kk;
                    if (ready && j >= 0 && j < c.n) {
#if ELSA_FWD_PACKED
                        // (f, s) pairs on the packed two-wide FP32 path: the same roundings
                        int fi, si;
                        const float2 h = make_float2(0.5f, 0.5f);
                        const float2 fl = floorSmall2(sub2(p2, h), fi, si);
                        const float2 cw = sub2(sub2(p2, fl), h);
                        const float2 w = sub2(make_float2(1.0f, 1.0f), cw);
                        const int lf = boxIndex<BW>(fi - o.x);
                        const int ls = boxIndex<BH>(si - o.y);
                        const int lk = dir > 0 ? kk : BD - 1 - kk;
                        const float* q = buf + (lk * BH + ls) * BW + lf;
                        // rows v0 and v1 of the footprint: (wf v00 + cwf v10, wf v01 + cwf v11)
                        const float2 r = fma2(make_float2(cw.x, cw.x), make_float2(q[1], q[BW + 1]),
                                              mul2(make_float2(w.x, w.x), make_float2(q[0], q[BW])));
#if ELSA_FWD_PAIR_ACC
                        acc2 = fma2(make_float2(w.y, cw.y), r, acc2);
#else
                        acc += w.y * r.x + cw.y * r.y;
#endif
                        p2 = add2(p2, s2);
#else
                        int fi, si;
                        const float ff = floorTap(__fsub_rn(pf, 0.5f), fi);
                        const float fs = floorTap(__fsub_rn(ps, 0.5f), si);
                        const float cwf = __fsub_rn(__fsub_rn(pf, ff), 0.5f);
                        const float cws = __fsub_rn(__fsub_rn(ps, fs), 0.5f);
                        const float wf = __fsub_rn(1.0f, cwf), ws = __fsub_rn(1.0f, cws);
                        const int lf = boxIndex<BW>(fi - o.x);
                        const int ls = boxIndex<BH>(si - o.y);
                        const int lk = dir > 0 ? kk : BD - 1 - kk;
                        const float* q = buf + (lk * BH + ls) * BW + lf;
                        const float v00 = q[0], v10 = q[1], v01 = q[BW], v11 = q[BW + 1];
                        acc += ws * (wf * v00 + cwf * v10) + cws * (wf * v01 + cwf * v11);
                        pf = __fadd_rn(pf, c.sf);
                        ps = __fadd_rn(ps, c.ss);
#endif
                    }
                }
                __syncthreads();
                if (abortFlag) { // a copy never completed: issue no more
                    failed = ch;
                    break;
                }
                if (threadIdx.x == 0 && ch + NS < T.nChunks)
                    issue(ch + NS);
            }
            if (failed >= 0) {
                // chunks failed .. failed + NS - 1 were issued and not consumed: give their
                // copies a bounded time to land before the CTA's shared memory goes away
                if (threadIdx.x == 0)
                    for (int ch = failed; ch < failed + NS && ch < T.nChunks; ++ch)
                        mbarWait(&full[ch % NS], (ch / NS) & 1, waitCycles);
                __syncthreads();
            }
#if ELSA_FWD_PACKED && ELSA_FWD_PAIR_ACC
            acc = acc2.x + acc2.y;
#endif
            if (valid)
                y[r] = c.n > 0 ? R.len * acc : 0.0f;
        }
    } // namespace

    namespace
    {
        PFN_cuTensorMapEncodeTiled_v12000 tensorMapEncoder()
        {
            static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
            if (!fn) {
                void* p = nullptr;
                cudaDriverEntryPointQueryResult q{};
                ELSA_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault,
                                                  &q));
                if (!p || q != cudaDriverEntryPointSuccess)
                    throw Error(ELSA_ERROR_CUDA, "cuTensorMapEncodeTiled is not available");
                fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
            }
            return fn;
        }

        // Non-driving axis along which neighbouring pixels of a detector row spread, voted over
        // the views (centre pixel and its right neighbour).
        std::array<int, 3> fastAxes(const std::vector<float>& poses, const DetectorShape& det)
        {
            int votes[3][3] = {};
            for (int p = 0; p < det.np; ++p) {
                const float* Pinv = poses.data() + static_cast<size_t>(p) * 40 + 12;
                const float uc = det.nu / 2 + 0.5f, vc = det.nv / 2 + 0.5f;
                float D[3], E[3];
                for (int i = 0; i < 3; ++i) {
                    D[i] = Pinv[i * 3] * uc + Pinv[i * 3 + 1] * vc + Pinv[i * 3 + 2];
                    E[i] = Pinv[i * 3] * (uc + 1.0f) + Pinv[i * 3 + 1] * vc + Pinv[i * 3 + 2];
                }
                int g = 0;
                for (int i = 1; i < 3; ++i)
                    if (std::fabs(D[i]) > std::fabs(D[g]))
                        g = i;
                int a, b;
                nonDrivingAxes(g, a, b);
                const float da = std::fabs(E[a] / std::fabs(E[g]) - D[a] / std::fabs(D[g]));
                const float db = std::fabs(E[b] / std::fabs(E[g]) - D[b] / std::fabs(D[g]));
                votes[g][da >= db ? a : b] += 1;
            }
            std::array<int, 3> fast{};
            for (int g = 0; g < 3; ++g) {
                int a, b;
                nonDrivingAxes(g, a, b);
                fast[g] = votes[g][b] > votes[g][a] ? b : a;
            }
            return fast;
        }
    } // namespace

    JosephForwardTma::JosephForwardTma(const VolumeShape& vol, const DetectorShape& det,
                                       const std::vector<float>& poses, const JosephRay* dRays)
        : vol_(vol), det_(det), dRays_(dRays)
    {
        fast_ = fastAxes(poses, det);
        for (int g = 0; g < 3; ++g) {
            int a, b;
            nonDrivingAxes(g, a, b);
            slow_[g] = fast_[g] == a ? b : a;
        }
        tilesU_ = (det.nu + TU - 1) / TU;
        tilesV_ = (det.nv + TV - 1) / TV;
        nTiles_ = static_cast<int64_t>(tilesU_) * tilesV_ * det.np;
        const int maxN = std::max(vol.n[0], std::max(vol.n[1], vol.n[2]));
        maxChunks_ = (maxN + 2 + BD - 1) / BD + 1;
        ELSA_CUDA(cudaMalloc(&dTiles_, sizeof(ForwardTile) * nTiles_));
        ELSA_CUDA(cudaMalloc(&dChunkOrigins_, sizeof(int2) * nTiles_ * maxChunks_));
        ELSA_CUDA(cudaMalloc(&dError_, sizeof(unsigned) * 2));
        ELSA_CUDA(cudaMemset(dError_, 0, sizeof(unsigned) * 2));
        const int3 fa = make_int3(fast_[0], fast_[1], fast_[2]);
        tileSetupKernel<<<static_cast<unsigned>(nTiles_), NT>>>(
            dRays_, det_, tilesU_, tilesV_, fa, maxChunks_, dTiles_, dChunkOrigins_, dError_ + 1);
        ELSA_LAUNCH_CHECK("tileSetupKernel");
        std::vector<ForwardTile> tiles(static_cast<size_t>(nTiles_));
        ELSA_CUDA(cudaMemcpy(tiles.data(), dTiles_, sizeof(ForwardTile) * nTiles_,
                             cudaMemcpyDeviceToHost));
        int64_t fallback = 0, live = 0;
        for (const auto& t : tiles) {
            if (t.flags & kFlagFallback) {
                fallback += t.nChunks > 0 ? 1 : 0;
            } else {
                present_[t.flags & 3] = true;
                ++live;
            }
        }
        fallbackFraction_ = live + fallback ? double(fallback) / double(live + fallback) : 0.0;
        for (int g = 0; g < 3; ++g)
            if (present_[g])
                padFast_[g] = (vol.n[fast_[g]] + 3) / 4 * 4;
        ensureBatch(1);
        ELSA_CUDA(cudaFuncSetAttribute(forwardTmaKernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(NS * kStageBytes)));
    }

    // Permuted copies for `batch` volumes and their tensor maps (4D: fast, slow, driving axis,
    // batch element). Grows only; growing waits for the device, since launches in flight read
    // the old copies.
    void JosephForwardTma::ensureBatch(int batch)
    {
        if (batch <= batchCap_)
            return;
        if (batchCap_ > 0)
            ELSA_CUDA(cudaDeviceSynchronize());
        auto encode = tensorMapEncoder();
        for (int g = 0; g < 3; ++g) {
            if (!present_[g])
                continue;
            const int nf = vol_.n[fast_[g]], ns = vol_.n[slow_[g]], ng = vol_.n[g];
            if (dLayouts_[g])
                ELSA_CUDA(cudaFree(dLayouts_[g]));
            dLayouts_[g] = nullptr;
            ELSA_CUDA(cudaMalloc(&dLayouts_[g],
                                 sizeof(float) * padFast_[g] * ns * ng * static_cast<size_t>(batch)));
            const cuuint64_t dims[4] = {static_cast<cuuint64_t>(nf), static_cast<cuuint64_t>(ns),
                                        static_cast<cuuint64_t>(ng),
                                        static_cast<cuuint64_t>(batch)};
            const cuuint64_t strides[3] = {static_cast<cuuint64_t>(padFast_[g]) * 4,
                                           static_cast<cuuint64_t>(padFast_[g]) * ns * 4,
                                           static_cast<cuuint64_t>(padFast_[g]) * ns * ng * 4};
            const cuuint32_t box[4] = {BW, BH, BD, 1};
            const cuuint32_t estr[4] = {1, 1, 1, 1};
            const CUresult rc = encode(&maps_[g], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                                       dLayouts_[g], dims, strides, box, estr,
                                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                       CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (rc != CUDA_SUCCESS)
                throw Error(ELSA_ERROR_CUDA, "cuTensorMapEncodeTiled failed");
        }
        batchCap_ = batch;
    }

    JosephForwardTma::~JosephForwardTma()
    {
        cudaFree(dTiles_);
        cudaFree(dChunkOrigins_);
        cudaFree(dError_);
        for (auto p : dLayouts_)
            if (p)
                cudaFree(p);
    }

    void JosephForwardTma::forward(const float* x, float* y, cudaStream_t s)
    {
        prepare(x, s);
        forwardViews(x, y, 0, det_.np, s);
    }

    void JosephForwardTma::forwardBatch(const float* x, int64_t xStride, float* y,
                                        int64_t yStride, int batch, cudaStream_t s)
    {
        if (batch <= 0)
            return;
        ensureBatch(batch);
        prepare(x, s, batch, xStride);
        forwardViews(x, y, 0, det_.np, s, batch, xStride, yStride);
    }

    void JosephForwardTma::prepare(const float* x, cudaStream_t s, int batch, int64_t xStride)
    {
        for (int g = 0; g < 3; ++g) {
            if (!present_[g])
                continue;
            permuteKernel<<<dim3(148 * 8, static_cast<unsigned>(batch)), 256, 0, s>>>(
                x, vol_, g, slow_[g], fast_[g], padFast_[g], dLayouts_[g], xStride);
            ELSA_LAUNCH_CHECK("permuteKernel");
        }
    }

    void JosephForwardTma::forwardViews(const float* x, float* y, int p0, int p1, cudaStream_t s,
                                        int batch, int64_t xStride, int64_t yStride)
    {
        const int64_t perView = static_cast<int64_t>(tilesU_) * tilesV_;
        const int64_t count = perView * (p1 - p0);
        if (count <= 0)
            return;
        forwardTmaKernel<<<dim3(static_cast<unsigned>(count), static_cast<unsigned>(batch)), NT,
                           NS * kStageBytes, s>>>(
            maps_[0], maps_[1], maps_[2], dRays_, dTiles_, dChunkOrigins_, maxChunks_, x, vol_,
            det_, tilesU_, tilesV_, make_int3(fast_[0], fast_[1], fast_[2]), y, dError_,
            static_cast<int>(perView * p0), waitCycles_, withhold_ ? 1 : 0, xStride, yStride);
        ELSA_LAUNCH_CHECK("forwardTmaKernel");
    }

    void JosephForwardTma::setWaitTest(long long cycles, bool withhold)
    {
        ELSA_CUDA(cudaDeviceSynchronize()); // no launch of the old setting in flight
        waitCycles_ = cycles > 0 ? cycles : kDefaultWaitCycles;
        withhold_ = withhold;
        ELSA_CUDA(cudaMemset(dError_, 0, sizeof(unsigned)));
    }

    unsigned JosephForwardTma::errorWord() const
    {
        unsigned e = 0;
        ELSA_CUDA(cudaMemcpy(&e, dError_, sizeof(unsigned), cudaMemcpyDeviceToHost));
        return e;
    }
} // namespace elsa_b200
