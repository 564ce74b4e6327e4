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

    KernelTimer::~KernelTimer()
    {
        for (auto e : pending_)
            cudaEventDestroy(e);
        for (auto e : pool_)
            cudaEventDestroy(e);
    }

    void KernelTimer::mark(cudaStream_t s)
    {
        if (!enabled_)
            return;
        cudaEvent_t e;
        if (!pool_.empty()) {
            e = pool_.back();
            pool_.pop_back();
        } else {
            ELSA_CUDA(cudaEventCreate(&e));
        }
        ELSA_CUDA(cudaEventRecord(e, s));
        pending_.push_back(e);
    }

    void KernelTimer::collect(double& fwdMs, double& adjMs, int64_t& count)
    {
        for (size_t i = 0; i + 2 < pending_.size(); i += 3) {
            ELSA_CUDA(cudaEventSynchronize(pending_[i + 2]));
            float a = 0, b = 0;
            ELSA_CUDA(cudaEventElapsedTime(&a, pending_[i], pending_[i + 1]));
            ELSA_CUDA(cudaEventElapsedTime(&b, pending_[i + 1], pending_[i + 2]));
            fwdMs_ += a;
            adjMs_ += b;
            ++count_;
        }
        pool_.insert(pool_.end(), pending_.begin(), pending_.end());
        pending_.clear();
        fwdMs = fwdMs_;
        adjMs = adjMs_;
        count = count_;
    }

    // CGNE: CG on the normal equations A^T A x = A^T b, solvers/CGNE.cpp:20-78.
    static void cgneBegin(Projector& A, const float* b, float* x, bool useX0,
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
    }

    static void cgneStep(Projector& A, float* x, SolverWorkspace& ws, KernelTimer& t,
                         cudaStream_t s)
    {
        const int64_t n = A.domainSize();
        float* r = ws.vol0.as<float>();
        float* c = ws.vol1.as<float>();
        float* q = ws.vol2.as<float>();
        float* sino = ws.sino0.as<float>();
        double* partials = ws.partials.as<double>();
        SolverScalars* S = ws.scalars.as<SolverScalars>();
        t.mark(s);
        A.forward(c, sino, s);
        t.mark(s);
        A.adjoint(sino, q, s); // q = A^T A c
        t.mark(s);
        launchDot(c, q, n, partials, &S->den, s);    // <c, A^T A c>
        launchCgStep(x, r, c, q, n, S, partials, s); // x += a c, r -= a q, |r|^2 partials
        launchCgFinishNorm(partials, S, s);          // k, beta = k/kold, kold = k
        launchCgDirection(r, c, n, S, s);            // c = r + beta c
    }

    void cgneSolve(Projector& A, const float* b, float* x, int iterations, bool useX0,
                   SolverWorkspace& ws, cudaStream_t s)
    {
        KernelTimer off;
        cgneBegin(A, b, x, useX0, ws, s);
        for (int it = 0; it < iterations; ++it)
            cgneStep(A, x, ws, off, s);
    }

    SolverSession::SolverSession(SolverKind kind, Projector& A, const float* b, float* x,
                                 bool useX0, cudaStream_t s)
        : kind_(kind), A_(A), b_(b), x_(x), ws_(A.domainSize(), A.rangeSize())
    {
        switch (kind_) {
        case SolverKind::CGNE:
            cgneBegin(A_, b_, x_, useX0, ws_, s);
            break;
        }
    }

    void SolverSession::iterate(int iterations, cudaStream_t s)
    {
        for (int it = 0; it < iterations; ++it) {
            switch (kind_) {
            case SolverKind::CGNE:
                cgneStep(A_, x_, ws_, timer_, s);
                break;
            }
        }
    }

    double SolverSession::squaredResidual(cudaStream_t s)
    {
        SolverScalars h;
        ELSA_CUDA(cudaMemcpyAsync(&h, ws_.scalars.as<SolverScalars>(), sizeof(h),
                                  cudaMemcpyDeviceToHost, s));
        ELSA_CUDA(cudaStreamSynchronize(s));
        return h.kold;
    }
} // namespace elsa_b200
