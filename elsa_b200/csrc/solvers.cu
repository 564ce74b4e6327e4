// Iterative solvers on the device: every vector operation is a fused kernel, inner products and
// residual norms accumulate in float64, and all scalars (alpha, beta, ...) stay in device memory,
// so an iteration is a fixed sequence of asynchronous launches on one stream (capturable in a
// CUDA graph).
#include "projector.hpp"
#include "solvers.hpp"
#include "vecops.cuh"

namespace elsa_b200
{
    Projector::Projector(int kind, const VolumeShape& vol, const DetectorShape& det,
                         const std::vector<PoseRecord>& poses)
        : kind_(kind), vol_(vol), det_(det), poses_(poses)
    {
        ELSA_CUDA(cudaGetDevice(&device_));
        domainSize_ = static_cast<int64_t>(vol.n[0]) * vol.n[1] * vol.n[2];
        rangeSize_ = static_cast<int64_t>(det.nu) * det.nv * det.np;
        ELSA_CUDA(cudaMalloc(&dPoses_, sizeof(PoseRecord) * poses.size()));
        ELSA_CUDA(cudaMemcpy(dPoses_, poses.data(), sizeof(PoseRecord) * poses.size(),
                             cudaMemcpyHostToDevice));
    }

    Projector::~Projector()
    {
        cudaFree(dPoses_);
    }

    DeviceBuffer::DeviceBuffer(size_t bytes) : bytes_(bytes)
    {
        if (bytes)
            ELSA_CUDA(cudaMalloc(&ptr_, bytes));
    }

    DeviceBuffer::~DeviceBuffer()
    {
        if (ptr_)
            cudaFree(ptr_);
    }

    SolverWorkspace::SolverWorkspace(int64_t domain, int64_t range)
        : vol0(sizeof(float) * domain), vol1(sizeof(float) * domain),
          vol2(sizeof(float) * domain), vol3(sizeof(float) * domain),
          sino0(sizeof(float) * range), partials(sizeof(double) * kReduceBlocks),
          scalars(sizeof(SolverScalars))
    {
    }

    // CGNE: CG on the normal equations A^T A x = A^T b, solvers/CGNE.cpp:20-78.
    void cgneSolve(Projector& A, const float* b, float* x, int iterations, bool useX0,
                   SolverWorkspace& ws, cudaStream_t s)
    {
        const int64_t n = A.domainSize();
        float* r = ws.vol0.as<float>();
        float* c = ws.vol1.as<float>();
        float* q = ws.vol2.as<float>();
        float* sino = ws.sino0.as<float>();
        double* partials = ws.partials.as<double>();
        SolverScalars* S = ws.scalars.as<SolverScalars>();
        ELSA_CUDA(cudaMemsetAsync(S, 0, sizeof(SolverScalars), s));

        A.adjoint(b, r, s); // A^T b
        if (useX0) {
            A.forward(x, sino, s);
            A.adjoint(sino, q, s);
            launchLincomb(1.0f, r, -1.0f, q, r, n, s); // r = A^T b - A^T A x
        } else {
            launchFill(x, 0.0f, n, s);
        }
        ELSA_CUDA(cudaMemcpyAsync(c, r, sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
        launchSquaredNorm(r, n, partials, &S->kold, s);
        for (int it = 0; it < iterations; ++it)
            cgneIteration(A, x, r, c, q, sino, partials, S, s);
    }

    void cgneIteration(Projector& A, float* x, float* r, float* c, float* q, float* sino,
                       double* partials, SolverScalars* S, cudaStream_t s)
    {
        const int64_t n = A.domainSize();
        A.forward(c, sino, s);
        A.adjoint(sino, q, s);                         // q = A^T A c
        launchDot(c, q, n, partials, &S->den, s);      // <c, A^T A c>
        launchCgStep(x, r, c, q, n, S, partials, s);   // x += a c, r -= a q, |r|^2 partials
        launchCgFinishNorm(partials, S, s);            // k, beta = k/kold, kold = k
        launchCgDirection(r, c, n, S, s);              // c = r + beta c
    }
} // namespace elsa_b200
