// Inner product that allocates no device memory (elsa_dot_no_alloc in the C ABI).
//
// elsa_dot allocates a small buffer of partial sums on every call. Some callers cannot do that:
// cudaMalloc and cudaFree synchronize the whole device, which stalls every other stream in a
// latency-bound loop, and hosts that hand all device memory to their own pool allocator cannot
// let a library allocate behind their back. For them this variant keeps its partial sums in a
// fixed file-scope device array instead.
//
// Limits and sharing:
// * The array holds kNoAllocPartials float64 partial sums (128 KiB); each block of the reduction
//   sums up to kNoAllocElemsPerBlock elements, so n is limited to
//   ELSA_DOT_NO_ALLOC_MAX_ELEMENTS = kNoAllocPartials * kNoAllocElemsPerBlock (67,108,864).
//   Larger n is rejected with ELSA_ERROR_INVALID_ARGUMENT.
// * Every GPU that loads the library holds its own copy of the array until the process exits.
// * All calls on one device share the array. Nothing in it has to start at zero: every block
//   writes its partial sum before the final pass reads it. Two calls that can run at the same
//   time on the GPU (different streams, or different host threads without ordering) race on the
//   array and may return wrong sums; order them on one stream.
// * The device address of the array is looked up once per device (cudaGetSymbolAddress) by the
//   first call made with that device current; make that first call before any stream capture.
//   The address is kept for the life of the process: after a cudaDeviceReset (or anything else
//   that re-creates the device's primary context) the module may load elsewhere, so this entry
//   point does not support a device reset after its first call on that device.
#include "internal.cuh"
#include "vecops.cuh"

#include <mutex>
#include <string>

namespace elsa_b200
{
    namespace
    {
        constexpr int kNoAllocThreads = 256;
        constexpr int64_t kNoAllocElemsPerBlock = 4096; // 256 threads x 16 elements
        constexpr int kNoAllocPartials = 16384;        // 128 KiB of float64
        static_assert(static_cast<int64_t>(kNoAllocPartials) * kNoAllocElemsPerBlock ==
                          ELSA_DOT_NO_ALLOC_MAX_ELEMENTS,
                      "header limit and scratch size disagree");

        static __device__ __align__(256) double gDotScratch[kNoAllocPartials];

        constexpr int kMaxDevices = 64;
        std::mutex gScratchMutex;
        double* gScratchAddr[kMaxDevices] = {};

        // Device address of gDotScratch on the current device, looked up on first use.
        double* scratchAddress()
        {
            int dev = 0;
            ELSA_CUDA(cudaGetDevice(&dev));
            if (dev < 0 || dev >= kMaxDevices)
                throw Error(ELSA_ERROR_NOT_SUPPORTED, "elsa_dot_no_alloc: device index too large");
            std::lock_guard<std::mutex> lock(gScratchMutex);
            if (!gScratchAddr[dev]) {
                void* p = nullptr;
                ELSA_CUDA(cudaGetSymbolAddress(&p, gDotScratch));
                gScratchAddr[dev] = static_cast<double*>(p);
            }
            return gScratchAddr[dev];
        }

        __device__ __forceinline__ double blockSumNoAlloc(double v)
        {
            __shared__ double warpSums[kNoAllocThreads / 32];
            for (int o = 16; o > 0; o >>= 1)
                v += __shfl_down_sync(0xffffffffu, v, o);
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            if (lane == 0)
                warpSums[warp] = v;
            __syncthreads();
            double s = 0.0;
            if (warp == 0) {
                s = lane < kNoAllocThreads / 32 ? warpSums[lane] : 0.0;
                for (int o = 16; o > 0; o >>= 1)
                    s += __shfl_down_sync(0xffffffffu, s, o);
            }
            return s; // valid in thread 0
        }

        // Block b sums elements b*T + t, (b + gridDim)*T + t, ... in a fixed order and writes one
        // partial sum.
        __global__ void __launch_bounds__(kNoAllocThreads)
            dotPartialsNoAllocKernel(const float* __restrict__ x, const float* __restrict__ y,
                                     int64_t n, double* __restrict__ partials)
        {
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
            double acc = 0.0;
            for (int64_t i = tid; i < n; i += stride)
                acc += static_cast<double>(__ldg(x + i)) * __ldg(y + i);
            const double s = blockSumNoAlloc(acc);
            if (threadIdx.x == 0)
                partials[blockIdx.x] = s;
        }

        __global__ void __launch_bounds__(kNoAllocThreads)
            dotFinishNoAllocKernel(const double* __restrict__ partials, int count,
                                   double* __restrict__ result)
        {
            double v = 0.0;
            for (int i = threadIdx.x; i < count; i += blockDim.x)
                v += partials[i];
            const double s = blockSumNoAlloc(v);
            if (threadIdx.x == 0)
                *result = s;
        }
    } // namespace

    void dotNoAlloc(const float* x, const float* y, int64_t n, double* result, cudaStream_t s)
    {
        if (!result || n < 0 || (n > 0 && (!x || !y)))
            throw Error(ELSA_ERROR_INVALID_ARGUMENT, "elsa_dot_no_alloc: invalid argument");
        if (n > ELSA_DOT_NO_ALLOC_MAX_ELEMENTS)
            throw Error(ELSA_ERROR_INVALID_ARGUMENT,
                        "elsa_dot_no_alloc: n = " + std::to_string(n) +
                            " exceeds the maximum of " +
                            std::to_string(ELSA_DOT_NO_ALLOC_MAX_ELEMENTS) +
                            " elements (the fixed scratch holds " +
                            std::to_string(kNoAllocPartials) +
                            " partial sums); use elsa_dot for larger vectors");
        double* partials = scratchAddress();
        const int blocks = n == 0 ? 1
                                  : static_cast<int>((n + kNoAllocElemsPerBlock - 1) /
                                                     kNoAllocElemsPerBlock);
        dotPartialsNoAllocKernel<<<blocks, kNoAllocThreads, 0, s>>>(x, y, n, partials);
        ELSA_LAUNCH_CHECK("dotPartialsNoAllocKernel");
        dotFinishNoAllocKernel<<<1, kNoAllocThreads, 0, s>>>(partials, blocks, result);
        ELSA_LAUNCH_CHECK("dotFinishNoAllocKernel");
    }
} // namespace elsa_b200
