// Fused vector operations, see vecops.cuh.
//
// Reference semantics: storage/reductions/DotProduct.h:24-47 (dot), storage/reductions/L2.h:15-49
// (squaredL2Norm), storage/transforms/Lincomb.h:28-33 (lincomb). The reference reduces in the data
// type (float); these kernels keep float data and accumulate in float64.
#include "internal.cuh"
#include "vecops.cuh"

namespace elsa_b200
{
    namespace
    {
        __device__ __forceinline__ double blockSum(double v)
        {
            __shared__ double warpSums[kReduceThreads / 32];
            for (int o = 16; o > 0; o >>= 1)
                v += __shfl_down_sync(0xffffffffu, v, o);
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            if (lane == 0)
                warpSums[warp] = v;
            __syncthreads();
            double s = 0.0;
            if (warp == 0) {
                s = lane < kReduceThreads / 32 ? warpSums[lane] : 0.0;
                for (int o = 16; o > 0; o >>= 1)
                    s += __shfl_down_sync(0xffffffffu, s, o);
            }
            return s; // valid in thread 0
        }

        // Each thread handles float4 chunks i = tid, tid + T, ... (T = total threads), plus a
        // scalar tail; fixed assignment -> fixed summation order.
        template <bool kSquare>
        __device__ __forceinline__ void partialDot(const float* __restrict__ x,
                                                   const float* __restrict__ y, int64_t n,
                                                   double* __restrict__ partials);

        template <bool kSquare>
        __global__ void __launch_bounds__(kReduceThreads)
            partialDotKernel(const float* __restrict__ x, const float* __restrict__ y, int64_t n,
                             double* __restrict__ partials)
        {
            partialDot<kSquare>(x, y, n, partials);
        }

        template <bool kSquare>
        __device__ __forceinline__ void partialDot(const float* __restrict__ x,
                                                   const float* __restrict__ y, int64_t n,
                                                   double* __restrict__ partials)
        {
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t T = static_cast<int64_t>(gridDim.x) * blockDim.x;
            double acc = 0.0;
            const bool vec = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) &
                              15) == 0;
            int64_t done = 0;
            if (vec) {
                const int64_t n4 = n / 4;
                const float4* x4 = reinterpret_cast<const float4*>(x);
                const float4* y4 = reinterpret_cast<const float4*>(y);
                for (int64_t i = tid; i < n4; i += T) {
                    const float4 a = __ldg(x4 + i);
                    const float4 b = kSquare ? a : __ldg(y4 + i);
                    acc += static_cast<double>(a.x) * b.x + static_cast<double>(a.y) * b.y +
                           static_cast<double>(a.z) * b.z + static_cast<double>(a.w) * b.w;
                }
                done = n4 * 4;
            }
            for (int64_t i = done + tid; i < n; i += T) {
                const float a = __ldg(x + i);
                const float b = kSquare ? a : __ldg(y + i);
                acc += static_cast<double>(a) * b;
            }
            const double s = blockSum(acc);
            if (threadIdx.x == 0)
                partials[blockIdx.x] = s;
        }

        __device__ __forceinline__ double sumPartials(const double* __restrict__ partials)
        {
            double v = 0.0;
            for (int i = threadIdx.x; i < kReduceBlocks; i += blockDim.x)
                v += partials[i];
            return blockSum(v);
        }

        __global__ void __launch_bounds__(kReduceThreads)
            finishSumKernel(const double* __restrict__ partials, double* __restrict__ out)
        {
            const double s = sumPartials(partials);
            if (threadIdx.x == 0)
                *out = s;
        }

        __global__ void lincombKernel(float a, const float* x, float b, const float* y, float* out,
                                      int64_t n)
        {
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t T = static_cast<int64_t>(gridDim.x) * blockDim.x;
            for (int64_t i = tid; i < n; i += T)
                out[i] = a * x[i] + b * y[i];
        }

        __global__ void lincombDevKernel(const double* sa, float ca, const float* x,
                                         const double* sb, float cb, const float* y, float* out,
                                         int64_t n)
        {
            const float a = sa ? static_cast<float>(*sa) : ca;
            const float b = sb ? static_cast<float>(*sb) : cb;
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t T = static_cast<int64_t>(gridDim.x) * blockDim.x;
            for (int64_t i = tid; i < n; i += T)
                out[i] = a * x[i] + b * y[i];
        }

        __global__ void fillKernel(float* x, float v, int64_t n)
        {
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t T = static_cast<int64_t>(gridDim.x) * blockDim.x;
            for (int64_t i = tid; i < n; i += T)
                x[i] = v;
        }

        __global__ void scaleKernel(float* x, float v, int64_t n)
        {
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t T = static_cast<int64_t>(gridDim.x) * blockDim.x;
            for (int64_t i = tid; i < n; i += T)
                x[i] *= v;
        }

        __device__ __forceinline__ void cgStep(float* __restrict__ x, float* __restrict__ r,
                                               const float* __restrict__ c,
                                               const float* __restrict__ q, int64_t n,
                                               const SolverScalars* S,
                                               double* __restrict__ partials);

        __global__ void __launch_bounds__(kReduceThreads)
            cgStepKernel(float* __restrict__ x, float* __restrict__ r, const float* __restrict__ c,
                         const float* __restrict__ q, int64_t n, const SolverScalars* S,
                         double* __restrict__ partials)
        {
            cgStep(x, r, c, q, n, S, partials);
        }

        __device__ __forceinline__ void cgStep(float* __restrict__ x, float* __restrict__ r,
                                               const float* __restrict__ c,
                                               const float* __restrict__ q, int64_t n,
                                               const SolverScalars* S,
                                               double* __restrict__ partials)
        {
            const float alpha = static_cast<float>(S->kold / S->den);
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t T = static_cast<int64_t>(gridDim.x) * blockDim.x;
            double acc = 0.0;
            for (int64_t i = tid; i < n; i += T) {
                x[i] = x[i] + alpha * c[i];
                const float ri = r[i] - alpha * q[i];
                r[i] = ri;
                acc += static_cast<double>(ri) * ri;
            }
            const double s = blockSum(acc);
            if (threadIdx.x == 0)
                partials[blockIdx.x] = s;
        }

        __global__ void __launch_bounds__(kReduceThreads)
            cgFinishNormKernel(const double* __restrict__ partials, SolverScalars* S)
        {
            const double s = sumPartials(partials);
            if (threadIdx.x == 0) {
                S->k = s;
                S->beta = s / S->kold;
                S->kold = s;
            }
        }

        __global__ void __launch_bounds__(kReduceThreads)
            finishDenKernel(const double* __restrict__ partials, SolverScalars* S)
        {
            const double s = sumPartials(partials);
            if (threadIdx.x == 0)
                S->den = s;
        }

        __global__ void cgDirectionKernel(const float* __restrict__ r, float* __restrict__ c,
                                          int64_t n, const SolverScalars* S)
        {
            const float beta = static_cast<float>(S->beta);
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t T = static_cast<int64_t>(gridDim.x) * blockDim.x;
            for (int64_t i = tid; i < n; i += T)
                c[i] = r[i] + beta * c[i];
        }

        // batched CGNE update: blockIdx.y selects the instance, blockIdx.x is the block of
        // the single-instance launch
        __global__ void __launch_bounds__(kReduceThreads)
            dotManyKernel(const CgBatchEntry* __restrict__ e)
        {
            const CgBatchEntry E = e[blockIdx.y];
            partialDot<false>(E.c, E.q, E.n, E.partials);
        }

        __global__ void __launch_bounds__(kReduceThreads)
            finishDenManyKernel(const CgBatchEntry* __restrict__ e)
        {
            const CgBatchEntry E = e[blockIdx.y];
            const double s = sumPartials(E.partials);
            if (threadIdx.x == 0)
                E.S->den = s;
        }

        __global__ void __launch_bounds__(kReduceThreads)
            cgStepManyKernel(const CgBatchEntry* __restrict__ e)
        {
            const CgBatchEntry E = e[blockIdx.y];
            cgStep(E.x, E.r, E.c, E.q, E.n, E.S, E.partials);
        }

        __global__ void __launch_bounds__(kReduceThreads)
            cgFinishNormManyKernel(const CgBatchEntry* __restrict__ e)
        {
            const CgBatchEntry E = e[blockIdx.y];
            const double s = sumPartials(E.partials);
            if (threadIdx.x == 0) {
                E.S->k = s;
                E.S->beta = s / E.S->kold;
                E.S->kold = s;
            }
        }

        __global__ void cgDirectionManyKernel(const CgBatchEntry* __restrict__ e)
        {
            const CgBatchEntry E = e[blockIdx.y];
            const float beta = static_cast<float>(E.S->beta);
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t T = static_cast<int64_t>(gridDim.x) * blockDim.x;
            for (int64_t i = tid; i < E.n; i += T)
                E.c[i] = E.r[i] + beta * E.c[i];
        }

        unsigned gridFor(int64_t n)
        {
            const int64_t b = (n + 255) / 256;
            return static_cast<unsigned>(b < 148 * 16 ? (b < 1 ? 1 : b) : 148 * 16);
        }
    } // namespace

    void launchDot(const float* x, const float* y, int64_t n, double* partials, double* result,
                   cudaStream_t s)
    {
        partialDotKernel<false><<<kReduceBlocks, kReduceThreads, 0, s>>>(x, y, n, partials);
        finishSumKernel<<<1, kReduceThreads, 0, s>>>(partials, result);
        ELSA_LAUNCH_CHECK("dot");
    }

    void launchSquaredNorm(const float* x, int64_t n, double* partials, double* result,
                           cudaStream_t s)
    {
        partialDotKernel<true><<<kReduceBlocks, kReduceThreads, 0, s>>>(x, x, n, partials);
        finishSumKernel<<<1, kReduceThreads, 0, s>>>(partials, result);
        ELSA_LAUNCH_CHECK("squaredL2Norm");
    }

    void launchLincomb(float a, const float* x, float b, const float* y, float* out, int64_t n,
                       cudaStream_t s)
    {
        lincombKernel<<<gridFor(n), 256, 0, s>>>(a, x, b, y, out, n);
        ELSA_LAUNCH_CHECK("lincomb");
    }

    void launchLincombDev(const double* sa, float ca, const float* x, const double* sb, float cb,
                          const float* y, float* out, int64_t n, cudaStream_t s)
    {
        lincombDevKernel<<<gridFor(n), 256, 0, s>>>(sa, ca, x, sb, cb, y, out, n);
        ELSA_LAUNCH_CHECK("lincombDev");
    }

    void launchFill(float* x, float value, int64_t n, cudaStream_t s)
    {
        fillKernel<<<gridFor(n), 256, 0, s>>>(x, value, n);
        ELSA_LAUNCH_CHECK("fill");
    }

    void launchScale(float* x, float value, int64_t n, cudaStream_t s)
    {
        scaleKernel<<<gridFor(n), 256, 0, s>>>(x, value, n);
        ELSA_LAUNCH_CHECK("scale");
    }

    void launchCgStep(float* x, float* r, const float* c, const float* q, int64_t n,
                      SolverScalars* S, double* partials, cudaStream_t s)
    {
        cgStepKernel<<<kReduceBlocks, kReduceThreads, 0, s>>>(x, r, c, q, n, S, partials);
        ELSA_LAUNCH_CHECK("cgStep");
    }

    void launchCgFinishNorm(const double* partials, SolverScalars* S, cudaStream_t s)
    {
        cgFinishNormKernel<<<1, kReduceThreads, 0, s>>>(partials, S);
        ELSA_LAUNCH_CHECK("cgFinishNorm");
    }

    void launchFinishDen(const double* partials, SolverScalars* S, cudaStream_t s)
    {
        finishDenKernel<<<1, kReduceThreads, 0, s>>>(partials, S);
        ELSA_LAUNCH_CHECK("finishDen");
    }

    void launchCgDirection(const float* r, float* c, int64_t n, const SolverScalars* S,
                           cudaStream_t s)
    {
        cgDirectionKernel<<<gridFor(n), 256, 0, s>>>(r, c, n, S);
        ELSA_LAUNCH_CHECK("cgDirection");
    }

    void launchCgneUpdateBatch(const CgBatchEntry* entries, int count, int64_t maxN,
                               cudaStream_t s)
    {
        if (count <= 0)
            return;
        const unsigned nb = static_cast<unsigned>(count);
        dotManyKernel<<<dim3(kReduceBlocks, nb), kReduceThreads, 0, s>>>(entries);
        finishDenManyKernel<<<dim3(1, nb), kReduceThreads, 0, s>>>(entries);
        cgStepManyKernel<<<dim3(kReduceBlocks, nb), kReduceThreads, 0, s>>>(entries);
        cgFinishNormManyKernel<<<dim3(1, nb), kReduceThreads, 0, s>>>(entries);
        cgDirectionManyKernel<<<dim3(gridFor(maxN), nb), 256, 0, s>>>(entries);
        ELSA_LAUNCH_CHECK("cgneUpdateBatch");
    }
} // namespace elsa_b200

namespace elsa_b200
{
    namespace
    {
        __global__ void __launch_bounds__(kReduceThreads)
            cglsStepKernel(float* __restrict__ x, float* __restrict__ sres,
                           const float* __restrict__ c, const float* __restrict__ q, int64_t nx,
                           int64_t ns, const SolverScalars* S, float damp)
        {
            if (S->done)
                return;
            const double den = S->den + (damp != 0.0f ? damp * S->aux[0] : 0.0);
            const float alpha = static_cast<float>(S->kold / den);
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t T = static_cast<int64_t>(gridDim.x) * blockDim.x;
            for (int64_t i = tid; i < nx; i += T)
                x[i] = x[i] + alpha * c[i];
            for (int64_t i = tid; i < ns; i += T)
                sres[i] = sres[i] - alpha * q[i];
        }

        __global__ void __launch_bounds__(kReduceThreads)
            dampNormKernel(float* __restrict__ r, const float* __restrict__ x, float damp,
                           int64_t n, double* __restrict__ partials)
        {
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t T = static_cast<int64_t>(gridDim.x) * blockDim.x;
            double acc = 0.0;
            for (int64_t i = tid; i < n; i += T) {
                float v = r[i];
                if (damp != 0.0f) {
                    v = v - damp * x[i];
                    r[i] = v;
                }
                acc += static_cast<double>(v) * v;
            }
            const double sum = blockSum(acc);
            if (threadIdx.x == 0)
                partials[blockIdx.x] = sum;
        }

        __global__ void checkTolKernel(SolverScalars* S, double tol)
        {
            if (S->kold < tol)
                S->done = 1;
        }

        __global__ void cgDirectionGuardedKernel(const float* __restrict__ r,
                                                 float* __restrict__ c, int64_t n,
                                                 const SolverScalars* S)
        {
            if (S->done)
                return;
            const float beta = static_cast<float>(S->beta);
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t T = static_cast<int64_t>(gridDim.x) * blockDim.x;
            for (int64_t i = tid; i < n; i += T)
                c[i] = r[i] + beta * c[i];
        }

        // out may alias a or b (element-wise read before write)
        __global__ void subKernel(const float* a, const float* b, float* out, int64_t n)
        {
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t T = static_cast<int64_t>(gridDim.x) * blockDim.x;
            for (int64_t i = tid; i < n; i += T)
                out[i] = a[i] - b[i];
        }

        __global__ void axpyMinusKernel(float* __restrict__ x, float step,
                                        const float* __restrict__ q, int64_t n)
        {
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t T = static_cast<int64_t>(gridDim.x) * blockDim.x;
            for (int64_t i = tid; i < n; i += T)
                x[i] = x[i] - step * q[i];
        }

        __global__ void scaleByInvNormKernel(float* __restrict__ u, const double* normSq,
                                             int64_t n)
        {
            const float nrm = static_cast<float>(sqrt(*normSq));
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t T = static_cast<int64_t>(gridDim.x) * blockDim.x;
            for (int64_t i = tid; i < n; i += T)
                u[i] = u[i] / nrm;
        }

        __device__ __forceinline__ float applyProx(float z, const ProxSpec& p, float mu)
        {
            if (p.kind == 1) { // ProximalBoxConstraint.cpp:27-40 (clip / maximum / minimum)
                if (p.flags & 1)
                    z = fmaxf(z, p.lo);
                if (p.flags & 2)
                    z = fminf(z, p.hi);
                return z;
            }
            if (p.kind == 2) { // ProximalL1.cpp:24-38 (soft threshold at mu * sigma)
                float t = fabsf(z) - mu * p.sigma;
                t = 0.5f * (t + fabsf(t));
                const float sg = z > 0.0f ? 1.0f : (z < 0.0f ? -1.0f : 0.0f);
                return sg * t;
            }
            return z;
        }

        __global__ void __launch_bounds__(kReduceThreads)
            apgdStepKernel(float* __restrict__ x, float* __restrict__ xPrev, float* __restrict__ y,
                           const float* __restrict__ grad, float mu, ProxSpec prox, int64_t n,
                           const SolverScalars* S, double* __restrict__ partials)
        {
            const bool done = S->done != 0;
            const double tp = S->tPrev;
            const double t = (1.0 + sqrt(1.0 + 4.0 * tp * tp)) / 2.0;
            const float coef = static_cast<float>((tp - 1.0) / t);
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t T = static_cast<int64_t>(gridDim.x) * blockDim.x;
            double acc = 0.0;
            for (int64_t i = tid; i < n; i += T) {
                const float g = grad[i];
                acc += static_cast<double>(g) * g;
                if (done)
                    continue;
                const float z = y[i] - mu * g;
                const float xn = applyProx(z, prox, mu);
                y[i] = xn + coef * (xn - xPrev[i]);
                x[i] = xn;
                xPrev[i] = xn;
            }
            const double sum = blockSum(acc);
            if (threadIdx.x == 0)
                partials[blockIdx.x] = sum;
        }

        __global__ void __launch_bounds__(kReduceThreads)
            apgdFinishKernel(const double* __restrict__ partials, SolverScalars* S, double eps)
        {
            const double g2 = sumPartials(partials);
            if (threadIdx.x == 0 && !S->done) {
                const double tp = S->tPrev;
                S->tPrev = (1.0 + sqrt(1.0 + 4.0 * tp * tp)) / 2.0;
                S->k = g2;
                if (g2 <= eps)
                    S->done = 1;
            }
        }
    } // namespace

    void launchCglsStep(float* x, float* sres, const float* c, const float* q, int64_t nx,
                        int64_t ns, SolverScalars* S, float damp, cudaStream_t s)
    {
        cglsStepKernel<<<gridFor(nx > ns ? nx : ns), kReduceThreads, 0, s>>>(x, sres, c, q, nx,
                                                                             ns, S, damp);
        ELSA_LAUNCH_CHECK("cglsStep");
    }

    void launchDampNorm(float* r, const float* x, float damp, int64_t n, double* partials,
                        cudaStream_t s)
    {
        dampNormKernel<<<kReduceBlocks, kReduceThreads, 0, s>>>(r, x, damp, n, partials);
        ELSA_LAUNCH_CHECK("dampNorm");
    }

    void launchCheckTol(SolverScalars* S, double tol, cudaStream_t s)
    {
        checkTolKernel<<<1, 1, 0, s>>>(S, tol);
        ELSA_LAUNCH_CHECK("checkTol");
    }

    void launchCgDirectionGuarded(const float* r, float* c, int64_t n, const SolverScalars* S,
                                  cudaStream_t s)
    {
        cgDirectionGuardedKernel<<<gridFor(n), 256, 0, s>>>(r, c, n, S);
        ELSA_LAUNCH_CHECK("cgDirectionGuarded");
    }

    void launchSub(const float* in, const float* b, float* out, int64_t n, cudaStream_t s)
    {
        subKernel<<<gridFor(n), 256, 0, s>>>(in, b, out, n);
        ELSA_LAUNCH_CHECK("sub");
    }

    void launchAxpyMinus(float* x, float step, const float* q, int64_t n, cudaStream_t s)
    {
        axpyMinusKernel<<<gridFor(n), 256, 0, s>>>(x, step, q, n);
        ELSA_LAUNCH_CHECK("axpyMinus");
    }

    void launchScaleByInvNorm(float* u, const double* normSq, int64_t n, cudaStream_t s)
    {
        scaleByInvNormKernel<<<gridFor(n), 256, 0, s>>>(u, normSq, n);
        ELSA_LAUNCH_CHECK("scaleByInvNorm");
    }

    void launchApgdStep(float* x, float* xPrev, float* y, const float* grad, float mu,
                        ProxSpec prox, int64_t n, const SolverScalars* S, double* partials,
                        cudaStream_t s)
    {
        apgdStepKernel<<<kReduceBlocks, kReduceThreads, 0, s>>>(x, xPrev, y, grad, mu, prox, n,
                                                                S, partials);
        ELSA_LAUNCH_CHECK("apgdStep");
    }

    void launchApgdFinish(const double* partials, SolverScalars* S, double eps, cudaStream_t s)
    {
        apgdFinishKernel<<<1, kReduceThreads, 0, s>>>(partials, S, eps);
        ELSA_LAUNCH_CHECK("apgdFinish");
    }

    namespace
    {
        __global__ void reciprocalKernel(const float* __restrict__ in, float lift,
                                         float* __restrict__ out, int64_t n)
        {
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t T = static_cast<int64_t>(gridDim.x) * blockDim.x;
            for (int64_t i = tid; i < n; i += T)
                out[i] = 1.0f / (in[i] + lift);
        }

        __global__ void subMulKernel(const float* a, const float* __restrict__ b,
                                     const float* __restrict__ m, float* out, int64_t n)
        {
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t T = static_cast<int64_t>(gridDim.x) * blockDim.x;
            for (int64_t i = tid; i < n; i += T)
                out[i] = (a[i] - b[i]) * m[i];
        }

        __global__ void scaledStepKernel(float* __restrict__ x, float step,
                                         const float* __restrict__ t,
                                         const float* __restrict__ q, int64_t n)
        {
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t T = static_cast<int64_t>(gridDim.x) * blockDim.x;
            for (int64_t i = tid; i < n; i += T)
                x[i] = x[i] - step * (t[i] * q[i]);
        }

        __global__ void mulKernel(float* __restrict__ u, const float* __restrict__ m, int64_t n)
        {
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t T = static_cast<int64_t>(gridDim.x) * blockDim.x;
            for (int64_t i = tid; i < n; i += T)
                u[i] = u[i] * m[i];
        }

        __global__ void __launch_bounds__(kReduceThreads)
            momentumStepKernel(float* __restrict__ x, float* __restrict__ yPrev,
                               const float* __restrict__ grad, float lipschitz, float f, int ogm,
                               int64_t n, const SolverScalars* S, double* __restrict__ partials)
        {
            const bool done = S->done != 0;
            const double tp = S->tPrev;
            const double th = 0.5 * (1.0 + sqrt(1.0 + f * tp * tp));
            const float c1 = static_cast<float>((tp - 1.0) / th);
            const float c2 = static_cast<float>(tp / th);
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t T = static_cast<int64_t>(gridDim.x) * blockDim.x;
            double acc = 0.0;
            for (int64_t i = tid; i < n; i += T) {
                const float g = grad[i];
                acc += static_cast<double>(g) * g;
                if (done)
                    continue;
                const float gl = g / lipschitz;
                const float y = x[i] - gl;
                float xn = y + c1 * (y - yPrev[i]);
                if (ogm)
                    xn = xn - c2 * gl;
                x[i] = xn;
                yPrev[i] = y;
            }
            const double sum = blockSum(acc);
            if (threadIdx.x == 0)
                partials[blockIdx.x] = sum;
        }

        __global__ void __launch_bounds__(kReduceThreads)
            momentumFinishKernel(const double* __restrict__ partials, SolverScalars* S, float f,
                                 double relTol)
        {
            const double g2 = sumPartials(partials);
            if (threadIdx.x == 0 && !S->done) {
                const double tp = S->tPrev;
                S->tPrev = 0.5 * (1.0 + sqrt(1.0 + f * tp * tp));
                S->k = g2;
                if (g2 <= relTol * S->aux[1])
                    S->done = 1;
            }
        }
    } // namespace

    namespace
    {
        // nextT of SQS.cpp:123-124, in float: 1 + sqrt(1 + 4 * t * t) / 2
        __device__ __forceinline__ float sqsNextT(float t)
        {
            const float q = __fadd_rn(1.0f, __fmul_rn(__fmul_rn(4.0f, t), t));
            return __fadd_rn(1.0f, __fdiv_rn(__fsqrt_rn(q), 2.0f));
        }

        __global__ void __launch_bounds__(kReduceThreads)
            sqsStepKernel(float* __restrict__ x, float* __restrict__ prevX,
                          const float* __restrict__ g, const float* __restrict__ D,
                          const float* __restrict__ P, float nSub, int momentum, int64_t n,
                          const SolverScalars* S, double* __restrict__ partials)
        {
            const bool done = S->done != 0;
            const float t = static_cast<float>(S->alpha);
            const float prevT = static_cast<float>(S->beta);
            const float coef = __fdiv_rn(prevT, sqsNextT(t));
            const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
            const int64_t T = static_cast<int64_t>(gridDim.x) * blockDim.x;
            double acc = 0.0;
            for (int64_t i = tid; i < n; i += T) {
                float gi = g[i];
                if (P)
                    gi = __fmul_rn(P[i], gi);
                acc += static_cast<double>(gi) * gi;
                if (done)
                    continue;
                float xn = __fsub_rn(x[i], __fmul_rn(nSub, __fmul_rn(D[i], gi)));
                if (momentum) {
                    xn = __fadd_rn(xn, __fmul_rn(coef, __fsub_rn(xn, prevX[i])));
                    prevX[i] = xn;
                }
                x[i] = xn;
            }
            const double sum = blockSum(acc);
            if (threadIdx.x == 0)
                partials[blockIdx.x] = sum;
        }

        __global__ void __launch_bounds__(kReduceThreads)
            sqsFinishKernel(const double* __restrict__ partials, SolverScalars* S, int subsetMode,
                            int momentum)
        {
            const double g2 = sumPartials(partials);
            if (threadIdx.x == 0) {
                S->k = g2;
                if (!S->done) {
                    if (g2 <= S->aux[1]) {
                        if (subsetMode)
                            S->aux[0] = 1.0;
                        else
                            S->done = 1;
                    }
                    if (momentum) {
                        const float t = static_cast<float>(S->alpha);
                        S->beta = t;
                        S->alpha = sqsNextT(t);
                    }
                }
            }
        }

        __global__ void sqsBeginKernel(SolverScalars* S, double eps2)
        {
            S->alpha = 1.0;
            S->beta = 1.0;
            S->aux[0] = 0.0;
            S->aux[1] = S->k * eps2;
            S->done = 0;
        }

        __global__ void setFlagKernel(int* flag)
        {
            *flag = 1;
        }
    } // namespace

    void launchSqsStep(float* x, float* prevX, const float* g, const float* D, const float* P,
                       float nSub, int momentum, int64_t n, const SolverScalars* S,
                       double* partials, cudaStream_t s)
    {
        sqsStepKernel<<<kReduceBlocks, kReduceThreads, 0, s>>>(x, prevX, g, D, P, nSub, momentum,
                                                               n, S, partials);
        ELSA_LAUNCH_CHECK("sqsStep");
    }

    void launchSqsFinish(const double* partials, SolverScalars* S, int subsetMode, int momentum,
                         cudaStream_t s)
    {
        sqsFinishKernel<<<1, kReduceThreads, 0, s>>>(partials, S, subsetMode, momentum);
        ELSA_LAUNCH_CHECK("sqsFinish");
    }

    void launchSqsBegin(SolverScalars* S, double eps2, cudaStream_t s)
    {
        sqsBeginKernel<<<1, 1, 0, s>>>(S, eps2);
        ELSA_LAUNCH_CHECK("sqsBegin");
    }

    void launchSetFlag(int* flag, cudaStream_t s)
    {
        setFlagKernel<<<1, 1, 0, s>>>(flag);
        ELSA_LAUNCH_CHECK("setFlag");
    }

    void launchReciprocal(const float* in, float lift, float* out, int64_t n, cudaStream_t s)
    {
        reciprocalKernel<<<gridFor(n), 256, 0, s>>>(in, lift, out, n);
        ELSA_LAUNCH_CHECK("reciprocal");
    }

    void launchSubMul(const float* a, const float* b, const float* m, float* out, int64_t n,
                      cudaStream_t s)
    {
        subMulKernel<<<gridFor(n), 256, 0, s>>>(a, b, m, out, n);
        ELSA_LAUNCH_CHECK("subMul");
    }

    void launchScaledStep(float* x, float step, const float* t, const float* q, int64_t n,
                          cudaStream_t s)
    {
        scaledStepKernel<<<gridFor(n), 256, 0, s>>>(x, step, t, q, n);
        ELSA_LAUNCH_CHECK("scaledStep");
    }

    void launchMul(float* u, const float* m, int64_t n, cudaStream_t s)
    {
        mulKernel<<<gridFor(n), 256, 0, s>>>(u, m, n);
        ELSA_LAUNCH_CHECK("mul");
    }

    void launchMomentumStep(float* x, float* yPrev, const float* grad, float lipschitz, float f,
                            int ogm, int64_t n, const SolverScalars* S, double* partials,
                            cudaStream_t s)
    {
        momentumStepKernel<<<kReduceBlocks, kReduceThreads, 0, s>>>(x, yPrev, grad, lipschitz, f,
                                                                    ogm, n, S, partials);
        ELSA_LAUNCH_CHECK("momentumStep");
    }

    void launchMomentumFinish(const double* partials, SolverScalars* S, float f, double relTol,
                              cudaStream_t s)
    {
        momentumFinishKernel<<<1, kReduceThreads, 0, s>>>(partials, S, f, relTol);
        ELSA_LAUNCH_CHECK("momentumFinish");
    }
} // namespace elsa_b200
