// TMA-staged forward projection for 3D Joseph (see joseph_tma.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <vector>

#include "internal.cuh"

namespace elsa_b200
{
    // Per detector tile: first driving plane (in traversal order), number of box chunks and
    // flags (bits 0-1 driving axis, bit 2 negative direction, bit 3 gather fallback).
    struct __align__(16) ForwardTile {
        int kStart;
        int nChunks;
        int flags;
        int pad;
    };

    class JosephForwardTma
    {
    public:
        static constexpr int kTileU = 32, kTileV = 8;
        static constexpr int kBoxW = 48, kBoxH = 12, kBoxD = 8, kStages = 3;
        static constexpr int kThreads = kTileU * kTileV;

        JosephForwardTma(const VolumeShape& vol, const DetectorShape& det,
                         const std::vector<float>& poses, const JosephRay* dRays);
        ~JosephForwardTma();
        JosephForwardTma(const JosephForwardTma&) = delete;
        JosephForwardTma& operator=(const JosephForwardTma&) = delete;

        void forward(const float* x, float* y, cudaStream_t s);
        // batch volumes x + b xStride into sinograms y + b yStride, b < batch, in one launch
        void forwardBatch(const float* x, int64_t xStride, float* y, int64_t yStride, int batch,
                          cudaStream_t s);
        // forward() in two parts: the permuted copies of x, then the rays of views [p0, p1)
        void prepare(const float* x, cudaStream_t s, int batch = 1, int64_t xStride = 0);
        void forwardViews(const float* x, float* y, int p0, int p1, cudaStream_t s,
                          int batch = 1, int64_t xStride = 0, int64_t yStride = 0);
        // Fraction of tiles that take the gather fallback, and the error word (0 = fine;
        // synchronizes).
        double fallbackFraction() const { return fallbackFraction_; }
        // kernel launches of one forward(): one volume permutation per driving axis present,
        // plus the projection kernel
        int launchesPerForward() const
        {
            return 1 + (present_[0] ? 1 : 0) + (present_[1] ? 1 : 0) + (present_[2] ? 1 : 0);
        }
        unsigned errorWord() const;
        // Test hook for the bounded waits: limit them to `cycles` clock cycles (<= 0: the
        // default, about one second) and, with `withhold`, issue no copies, so every wait runs
        // out and sets bit 0 of the error word. Clears the error word.
        void setWaitTest(long long cycles, bool withhold);
        static constexpr long long kDefaultWaitCycles = 2000000000LL; // ~1 s at 2 GHz

    private:
        VolumeShape vol_;
        DetectorShape det_;
        const JosephRay* dRays_;
        int tilesU_ = 0, tilesV_ = 0, maxChunks_ = 0;
        int64_t nTiles_ = 0;
        ForwardTile* dTiles_ = nullptr;
        int2* dChunkOrigins_ = nullptr;
        unsigned* dError_ = nullptr;
        std::array<int, 3> fast_{{0, 0, 0}}; // fast (contiguous) non-driving axis per driving axis
        std::array<int, 3> slow_{{0, 0, 0}};
        std::array<bool, 3> present_{{false, false, false}};
        std::array<float*, 3> dLayouts_{{nullptr, nullptr, nullptr}}; // permuted copies
        std::array<int, 3> padFast_{{0, 0, 0}};
        std::array<CUtensorMap, 3> maps_{};
        double fallbackFraction_ = 0.0;
        long long waitCycles_ = kDefaultWaitCycles;
        bool withhold_ = false;
        int batchCap_ = 0; // volumes the permuted copies hold
        void ensureBatch(int batch);
    };
} // namespace elsa_b200
