// Iterative solvers on the device: every vector operation is a fused kernel, inner products and
// residual norms accumulate in float64, and all scalars (alpha, beta, ...) stay in device memory,
// so an iteration is a fixed sequence of asynchronous launches on one stream (capturable in a
// CUDA graph).
#include "geometry.hpp"
#include "projector.hpp"
#include "solvers.hpp"
#include "vecops.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

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

    CurvedTables::CurvedTables() = default;
    CurvedTables::~CurvedTables() = default;
    CurvedTables::CurvedTables(CurvedTables&&) noexcept = default;
    CurvedTables& CurvedTables::operator=(CurvedTables&&) noexcept = default;

    CurvedTables::CurvedTables(int dim, const DetectorShape& det, const CurvedDetector& c)
    {
        if (!c.enabled())
            return;
        if (!(c.s2d > 0.0f) || !std::isfinite(c.angle) || !std::isfinite(c.s2d))
            throw Error(ELSA_ERROR_INVALID_ARGUMENT,
                        "CurvedDetectorDescriptor: angle and source-to-detector distance must be "
                        "positive");
        std::vector<float> factor;
        const std::vector<float> xy =
            curvedPlanarCoords(dim, det.nu, det.nv, c.angle, c.s2d, &factor);
        std::vector<float> column(static_cast<size_t>(det.nu));
        for (int u = 0; u < det.nu; ++u) {
            column[static_cast<size_t>(u)] = xy[static_cast<size_t>(u) * 2];
            if (u > 0 && !(column[static_cast<size_t>(u)] > column[static_cast<size_t>(u - 1)]))
                throw Error(ELSA_ERROR_NOT_SUPPORTED,
                            "CurvedDetectorDescriptor: the pixel columns do not map to increasing "
                            "planar coordinates (opening angle too large)");
        }
        fmin_ = *std::min_element(factor.begin(), factor.end());
        fmax_ = *std::max_element(factor.begin(), factor.end());
        if (!(fmin_ > 0.0f))
            throw Error(ELSA_ERROR_NOT_SUPPORTED,
                        "CurvedDetectorDescriptor: the arc reaches behind the source");
        planar_ = std::make_unique<DeviceBuffer>(sizeof(float) * xy.size());
        column_ = std::make_unique<DeviceBuffer>(sizeof(float) * column.size());
        ELSA_CUDA(cudaMemcpy(planar_->as<float>(), xy.data(), sizeof(float) * xy.size(),
                             cudaMemcpyHostToDevice));
        ELSA_CUDA(cudaMemcpy(column_->as<float>(), column.data(), sizeof(float) * column.size(),
                             cudaMemcpyHostToDevice));
    }

    const float2* CurvedTables::planar() const
    {
        return planar_ ? planar_->as<float2>() : nullptr;
    }

    CurvedMap CurvedTables::map() const
    {
        CurvedMap m;
        m.planarU = column_ ? column_->as<float>() : nullptr;
        m.fmin = fmin_;
        m.fmax = fmax_;
        return m;
    }

    void CurvedTables::release()
    {
        planar_.reset();
        column_.reset();
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
          sino0(sizeof(float) * range), sino1(sizeof(float) * range),
          partials(sizeof(double) * kReduceBlocks),
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

    SplitCgne::SplitCgne(Projector& A, float* x) : A_(A), x_(x), ws_(A.domainSize(), A.rangeSize())
    {
    }

    void SplitCgne::backprojectData(const float* b, float* atb, cudaStream_t s)
    {
        A_.adjoint(b, atb, s);
    }

    void SplitCgne::begin(const float* atb, cudaStream_t s)
    {
        const int64_t n = A_.domainSize();
        float* r = ws_.vol0.as<float>();
        float* c = ws_.vol1.as<float>();
        SolverScalars* S = ws_.scalars.as<SolverScalars>();
        ELSA_CUDA(cudaMemsetAsync(S, 0, sizeof(SolverScalars), s));
        launchFill(x_, 0.0f, n, s);
        ELSA_CUDA(cudaMemcpyAsync(r, atb, sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
        ELSA_CUDA(cudaMemcpyAsync(c, atb, sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
        launchSquaredNorm(r, n, ws_.partials.as<double>(), &S->kold, s);
    }

    void SplitCgne::applyNormal(float* q, cudaStream_t s)
    {
        float* c = ws_.vol1.as<float>();
        float* sino = ws_.sino0.as<float>();
        A_.forward(c, sino, s);
        A_.adjoint(sino, q, s);
    }

    void SplitCgne::update(const float* q, cudaStream_t s)
    {
        const int64_t n = A_.domainSize();
        float* r = ws_.vol0.as<float>();
        float* c = ws_.vol1.as<float>();
        double* partials = ws_.partials.as<double>();
        SolverScalars* S = ws_.scalars.as<SolverScalars>();
        launchDot(c, q, n, partials, &S->den, s);     // <c, sum_r A_r^T A_r c>
        launchCgStep(x_, r, c, q, n, S, partials, s); // x += a c, r -= a q, |r|^2 partials
        launchCgFinishNorm(partials, S, s);           // k, beta = k/kold, kold = k
        launchCgDirection(r, c, n, S, s);             // c = r + beta c
    }

    const double* SplitCgne::squaredResidualDevice() const
    {
        return &ws_.scalars.as<SolverScalars>()->kold;
    }

    void cgneSolve(Projector& A, const float* b, float* x, int iterations, bool useX0,
                   SolverWorkspace& ws, cudaStream_t s)
    {
        KernelTimer off;
        cgneBegin(A, b, x, useX0, ws, s);
        for (int it = 0; it < iterations; ++it)
            cgneStep(A, x, ws, off, s);
    }

    double powerIterationsAtA(Projector& A, SolverWorkspace& ws, int iterations, cudaStream_t s,
                              const float* rangeScale, const float* domainScale)
    {
        const int64_t n = A.domainSize();
        float* u = ws.vol0.as<float>();
        float* v = ws.vol1.as<float>();
        float* sino = ws.sino0.as<float>();
        double* partials = ws.partials.as<double>();
        SolverScalars* S = ws.scalars.as<SolverScalars>();
        launchFill(u, 1.0f, n, s);
        const int64_t m = A.rangeSize();
        auto apply = [&](const float* in, float* out) {
            A.forward(in, sino, s);
            if (rangeScale)
                launchMul(sino, rangeScale, m, s);
            A.adjoint(sino, out, s);
            if (domainScale)
                launchMul(out, domainScale, n, s);
        };
        for (int i = 0; i < iterations; ++i) {
            apply(u, u); // u = A^T A u (scaled)
            launchSquaredNorm(u, n, partials, &S->k, s);
            launchScaleByInvNorm(u, &S->k, n, s);
        }
        apply(u, v);
        launchDot(u, v, n, partials, &S->den, s);
        launchSquaredNorm(u, n, partials, &S->k, s);
        SolverScalars h;
        ELSA_CUDA(cudaMemcpyAsync(&h, S, sizeof(h), cudaMemcpyDeviceToHost, s));
        ELSA_CUDA(cudaStreamSynchronize(s));
        return h.den / std::sqrt(h.k);
    }

    // CGLS: solvers/CGLS.cpp:19-91 (damping eps^2, stop once |r|^2 < tol).
    static void cglsBegin(Projector& A, const float* b, float* x, bool useX0, float damp,
                          SolverWorkspace& ws, cudaStream_t s)
    {
        const int64_t n = A.domainSize(), m = A.rangeSize();
        float* r = ws.vol0.as<float>();
        float* c = ws.vol1.as<float>();
        float* sres = ws.sino0.as<float>();
        double* partials = ws.partials.as<double>();
        SolverScalars* S = ws.scalars.as<SolverScalars>();
        ELSA_CUDA(cudaMemsetAsync(S, 0, sizeof(SolverScalars), s));
        if (useX0) {
            A.forward(x, sres, s);
            launchSub(b, sres, sres, m, s); // s = b - A x
            A.adjoint(sres, r, s);
            launchDampNorm(r, x, damp, n, partials, s); // r -= damp x
        } else {
            launchFill(x, 0.0f, n, s);
            ELSA_CUDA(cudaMemcpyAsync(sres, b, sizeof(float) * m, cudaMemcpyDeviceToDevice, s));
            A.adjoint(sres, r, s);
        }
        ELSA_CUDA(cudaMemcpyAsync(c, r, sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
        launchSquaredNorm(r, n, partials, &S->kold, s);
    }

    static void cglsStep(Projector& A, float* x, float damp, double tol, SolverWorkspace& ws,
                         KernelTimer& t, cudaStream_t s)
    {
        const int64_t n = A.domainSize(), m = A.rangeSize();
        float* r = ws.vol0.as<float>();
        float* c = ws.vol1.as<float>();
        float* sres = ws.sino0.as<float>();
        float* q = ws.sino1.as<float>();
        double* partials = ws.partials.as<double>();
        SolverScalars* S = ws.scalars.as<SolverScalars>();
        launchCheckTol(S, tol, s);
        t.mark(s);
        A.forward(c, q, s);
        t.mark(s);
        launchSquaredNorm(q, m, partials, &S->den, s);
        if (damp != 0.0f)
            launchSquaredNorm(c, n, partials, &S->aux[0], s);
        launchCglsStep(x, sres, c, q, n, m, S, damp, s);
        A.adjoint(sres, r, s);
        t.mark(s);
        launchDampNorm(r, x, damp, n, partials, s);
        launchCgFinishNorm(partials, S, s);
        launchCgDirectionGuarded(r, c, n, S, s);
    }

    // Landweber: solvers/LandweberIteration.cpp:26-72 with Landweber.cpp:20-25 (T = A^T).
    static void landweberStep(Projector& A, const float* b, float* x, float step,
                              SolverWorkspace& ws, KernelTimer& t, cudaStream_t s)
    {
        const int64_t n = A.domainSize(), m = A.rangeSize();
        float* q = ws.vol2.as<float>();
        float* sino = ws.sino0.as<float>();
        t.mark(s);
        A.forward(x, sino, s);
        t.mark(s);
        launchSub(sino, b, sino, m, s); // A x - b
        A.adjoint(sino, q, s);
        t.mark(s);
        launchAxpyMinus(x, step, q, n, s); // x -= step A^T (A x - b)
    }

    // APGD (FISTA): solvers/APGD.cpp:34-102; gradient A^T (A y) - A^T b.
    static void apgdGradient(Projector& A, SolverWorkspace& ws, KernelTimer& t, cudaStream_t s)
    {
        const int64_t n = A.domainSize();
        float* y = ws.vol1.as<float>();
        float* grad = ws.vol2.as<float>();
        float* atb = ws.vol3.as<float>();
        float* sino = ws.sino0.as<float>();
        t.mark(s);
        A.forward(y, sino, s);
        t.mark(s);
        A.adjoint(sino, grad, s);
        t.mark(s);
        launchSub(grad, atb, grad, n, s);
    }

    static void apgdBegin(Projector& A, const float* b, float* x, bool useX0,
                          SolverWorkspace& ws, cudaStream_t s)
    {
        const int64_t n = A.domainSize();
        SolverScalars* S = ws.scalars.as<SolverScalars>();
        ELSA_CUDA(cudaMemsetAsync(S, 0, sizeof(SolverScalars), s));
        static const double one = 1.0;
        ELSA_CUDA(cudaMemcpyAsync(&S->tPrev, &one, sizeof(double), cudaMemcpyHostToDevice, s));
        if (!useX0)
            launchFill(x, 0.0f, n, s);
        ELSA_CUDA(cudaMemcpyAsync(ws.vol0.as<float>(), x, sizeof(float) * n,
                                  cudaMemcpyDeviceToDevice, s)); // xPrev
        ELSA_CUDA(cudaMemcpyAsync(ws.vol1.as<float>(), x, sizeof(float) * n,
                                  cudaMemcpyDeviceToDevice, s)); // y
        A.adjoint(b, ws.vol3.as<float>(), s);                   // A^T b
        KernelTimer off;
        apgdGradient(A, ws, off, s);
    }

    static void apgdStep(Projector& A, float* x, float mu, const SolverOptions& opt,
                         SolverWorkspace& ws, KernelTimer& t, cudaStream_t s)
    {
        const int64_t n = A.domainSize();
        SolverScalars* S = ws.scalars.as<SolverScalars>();
        double* partials = ws.partials.as<double>();
        launchApgdStep(x, ws.vol0.as<float>(), ws.vol1.as<float>(), ws.vol2.as<float>(), mu,
                       opt.prox, n, S, partials, s);
        launchApgdFinish(partials, S, opt.apgdEpsilon, s);
        apgdGradient(A, ws, t, s);
    }

    // SIRT: Landweber with T A^T M, M = 1 / (A 1 + 1e-10), T = 1 / (A^T 1),
    // solvers/SIRT.cpp:20-45 with LandweberIteration.cpp:57-67. ws.vol3 = T, ws.sino1 = M (the
    // power iterations use vol0, vol1 and sino0).
    static void sirtBegin(Projector& A, SolverWorkspace& ws, cudaStream_t s)
    {
        const int64_t n = A.domainSize(), m = A.rangeSize();
        float* tinv = ws.vol3.as<float>();
        float* minv = ws.sino1.as<float>();
        launchFill(ws.vol1.as<float>(), 1.0f, n, s);
        A.forward(ws.vol1.as<float>(), minv, s); // row sums
        launchReciprocal(minv, 1e-10f, minv, m, s);
        launchFill(ws.sino0.as<float>(), 1.0f, m, s);
        A.adjoint(ws.sino0.as<float>(), tinv, s); // column sums
        launchReciprocal(tinv, 0.0f, tinv, n, s);
    }

    static void sirtStep(Projector& A, const float* b, float* x, float step, SolverWorkspace& ws,
                         KernelTimer& t, cudaStream_t s)
    {
        const int64_t n = A.domainSize(), m = A.rangeSize();
        float* sino = ws.sino0.as<float>();
        float* q = ws.vol2.as<float>();
        t.mark(s);
        A.forward(x, sino, s);
        t.mark(s);
        launchSubMul(sino, b, ws.sino1.as<float>(), sino, m, s); // M (A x - b)
        A.adjoint(sino, q, s);
        t.mark(s);
        launchScaledStep(x, step, ws.vol3.as<float>(), q, n, s); // x -= step T A^T M (A x - b)
    }

    // FGM / OGM on the least-squares problem 0.5 |A x - b|^2 (solvers/FGM.cpp:33-78,
    // OGM.cpp:40-95 with functionals/LeastSquares.cpp:45-59): gradient A^T (A x - b) into vol2,
    // previous y in vol1; S->aux[1] holds |grad_0|^2.
    static void lsqGradient(Projector& A, const float* b, const float* x, SolverWorkspace& ws,
                            KernelTimer& t, cudaStream_t s)
    {
        const int64_t m = A.rangeSize();
        float* sino = ws.sino0.as<float>();
        t.mark(s);
        A.forward(x, sino, s);
        t.mark(s);
        launchSub(sino, b, sino, m, s);
        A.adjoint(sino, ws.vol2.as<float>(), s);
        t.mark(s);
    }

    static void momentumBegin(Projector& A, const float* b, float* x, bool useX0,
                              SolverWorkspace& ws, cudaStream_t s)
    {
        const int64_t n = A.domainSize();
        SolverScalars* S = ws.scalars.as<SolverScalars>();
        if (!useX0)
            launchFill(x, 0.0f, n, s);
        ELSA_CUDA(cudaMemcpyAsync(ws.vol1.as<float>(), x, sizeof(float) * n,
                                  cudaMemcpyDeviceToDevice, s)); // yPrev = x
        KernelTimer off;
        lsqGradient(A, b, x, ws, off, s);
        ELSA_CUDA(cudaMemsetAsync(S, 0, sizeof(SolverScalars), s));
        launchSquaredNorm(ws.vol2.as<float>(), n, ws.partials.as<double>(), &S->aux[1], s);
        static const double one = 1.0;
        ELSA_CUDA(cudaMemcpyAsync(&S->tPrev, &one, sizeof(double), cudaMemcpyHostToDevice, s));
    }

    // SQS: solvers/SQS.cpp:87-170 on the least-squares problem 0.5 |A x - b|^2
    // (functionals/LeastSquares.cpp:45-59: gradient A^T (A x - b), Hessian A^T A). ws.vol0 =
    // prevX, vol1 = gradient, vol2 = D = 1 / (A^T A 1), vol3 = full gradient for the subset-mode
    // convergence check; S->alpha = t, S->beta = prevT.
    static void sqsGradient(Projector& A, const float* b, const float* x, float* g,
                            SolverWorkspace& ws, KernelTimer& t, cudaStream_t s)
    {
        float* sino = ws.sino0.as<float>();
        t.mark(s);
        A.forward(x, sino, s);
        t.mark(s);
        launchSub(sino, b, sino, A.rangeSize(), s);
        A.adjoint(sino, g, s);
        t.mark(s);
    }

    static void sqsBegin(Projector& A, const float* b, float* x, bool useX0, double eps,
                         SolverWorkspace& ws, cudaStream_t s)
    {
        const int64_t n = A.domainSize();
        SolverScalars* S = ws.scalars.as<SolverScalars>();
        double* partials = ws.partials.as<double>();
        ELSA_CUDA(cudaMemsetAsync(S, 0, sizeof(SolverScalars), s));
        if (!useX0)
            launchFill(x, 0.0f, n, s);
        KernelTimer off;
        sqsGradient(A, b, x, ws.vol1.as<float>(), ws, off, s);
        launchSquaredNorm(ws.vol1.as<float>(), n, partials, &S->k, s);
        launchSqsBegin(S, eps * eps, s);
        float* D = ws.vol2.as<float>();
        launchFill(D, 1.0f, n, s);
        A.forward(D, ws.sino0.as<float>(), s);
        A.adjoint(ws.sino0.as<float>(), D, s); // A^T A 1
        launchReciprocal(D, 0.0f, D, n, s);
        ELSA_CUDA(cudaMemcpyAsync(ws.vol0.as<float>(), x, sizeof(float) * n,
                                  cudaMemcpyDeviceToDevice, s)); // prevX
    }

    void SolverSession::sqsIterate(int iterations, cudaStream_t s)
    {
        const int64_t n = A_.domainSize();
        SolverScalars* S = ws_.scalars.as<SolverScalars>();
        double* partials = ws_.partials.as<double>();
        const bool subsetMode = !subsets_.empty();
        const int nSub = subsetMode ? static_cast<int>(subsets_.size()) : 1;
        const int momentum = opt_.sqsMomentum ? 1 : 0;
        for (int it = 0; it < iterations && !hostDone_; ++it) {
            for (int m = 0; m < nSub && !hostDone_; ++m) {
                Projector& Am = subsetMode ? *subsets_[static_cast<size_t>(m)].A : A_;
                const float* bm = subsetMode ? subsets_[static_cast<size_t>(m)].b : b_;
                sqsGradient(Am, bm, x_, ws_.vol1.as<float>(), ws_, timer_, s);
                launchSqsStep(x_, ws_.vol0.as<float>(), ws_.vol1.as<float>(),
                              ws_.vol2.as<float>(), opt_.sqsPreconditioner,
                              static_cast<float>(nSub), momentum, n, S, partials, s);
                launchSqsFinish(partials, S, subsetMode ? 1 : 0, momentum, s);
                if (!subsetMode)
                    continue;
                // the subset gradient passed the threshold: SQS.cpp:131-133 confirms with the
                // full problem's gradient at the new iterate (one host synchronization per
                // subset step)
                double candidate = 0.0;
                ELSA_CUDA(cudaMemcpyAsync(&candidate, &S->aux[0], sizeof(double),
                                          cudaMemcpyDeviceToHost, s));
                ELSA_CUDA(cudaStreamSynchronize(s));
                if (candidate == 0.0)
                    continue;
                static const double zero = 0.0;
                ELSA_CUDA(cudaMemcpyAsync(&S->aux[0], &zero, sizeof(double),
                                          cudaMemcpyHostToDevice, s));
                KernelTimer off;
                sqsGradient(A_, b_, x_, ws_.vol3.as<float>(), ws_, off, s);
                launchSquaredNorm(ws_.vol3.as<float>(), n, partials, &S->den, s);
                SolverScalars h;
                ELSA_CUDA(cudaMemcpyAsync(&h, S, sizeof(h), cudaMemcpyDeviceToHost, s));
                ELSA_CUDA(cudaStreamSynchronize(s));
                if (h.den <= h.aux[1]) {
                    launchSetFlag(&S->done, s);
                    hostDone_ = true;
                }
            }
        }
    }

    SolverSession::SolverSession(SolverKind kind, Projector& A, const float* b, float* x,
                                 bool useX0, const SolverOptions& opt, cudaStream_t s,
                                 std::vector<SubsetRef> subsets)
        : kind_(kind), opt_(opt), A_(A), b_(b), x_(x), ws_(A.domainSize(), A.rangeSize()),
          subsets_(std::move(subsets))
    {
        if (!subsets_.empty() && kind_ != SolverKind::SQS)
            throw Error(ELSA_ERROR_INVALID_ARGUMENT, "only SQS takes ordered subsets");
        for (const SubsetRef& r : subsets_) {
            if (!r.A || !r.b)
                throw Error(ELSA_ERROR_INVALID_ARGUMENT, "SQS: null subset");
            if (r.A->domainSize() != A.domainSize() || r.A->rangeSize() > A.rangeSize())
                throw Error(ELSA_ERROR_INVALID_ARGUMENT,
                            "SQS: a subset projector must share the volume and have at most "
                            "the full problem's views");
            if (r.A->device() != A.device())
                throw Error(ELSA_ERROR_INVALID_ARGUMENT, "SQS: subsets on another device");
        }
        switch (kind_) {
        case SolverKind::CGNE:
            cgneBegin(A_, b_, x_, useX0, ws_, s);
            break;
        case SolverKind::CGLS:
            cglsBegin(A_, b_, x_, useX0, static_cast<float>(opt_.cglsEps * opt_.cglsEps), ws_,
                      s);
            break;
        case SolverKind::LANDWEBER:
            step_ = opt_.landweberStep > 0.0
                        ? opt_.landweberStep
                        : 0.9 * (2.0 / powerIterationsAtA(A_, ws_, opt_.powerIterations, s));
            if (!useX0)
                launchFill(x_, 0.0f, A_.domainSize(), s);
            ELSA_CUDA(cudaMemsetAsync(ws_.scalars.as<SolverScalars>(), 0, sizeof(SolverScalars),
                                      s));
            break;
        case SolverKind::APGD:
            step_ = opt_.apgdMu > 0.0
                        ? opt_.apgdMu
                        : 0.45 / powerIterationsAtA(A_, ws_, opt_.powerIterations, s);
            apgdBegin(A_, b_, x_, useX0, ws_, s);
            break;
        case SolverKind::SIRT:
            sirtBegin(A_, ws_, s);
            step_ = opt_.sirtStep > 0.0
                        ? opt_.sirtStep
                        : 0.9 * (2.0 / powerIterationsAtA(A_, ws_, opt_.powerIterations, s,
                                                          ws_.sino1.as<float>(),
                                                          ws_.vol3.as<float>()));
            if (!useX0)
                launchFill(x_, 0.0f, A_.domainSize(), s);
            ELSA_CUDA(cudaMemsetAsync(ws_.scalars.as<SolverScalars>(), 0, sizeof(SolverScalars),
                                      s));
            break;
        case SolverKind::FGM:
        case SolverKind::OGM: {
            // FGM uses 5 power iterations, OGM 20 (OGM.cpp:57-60)
            const int pi = kind_ == SolverKind::OGM ? 20 : 5;
            lipschitz_ = static_cast<float>(powerIterationsAtA(A_, ws_, pi, s));
            step_ = 1.0 / lipschitz_;
            momentumBegin(A_, b_, x_, useX0, ws_, s);
            break;
        }
        case SolverKind::SQS:
            sqsBegin(A_, b_, x_, useX0, opt_.sqsEpsilon, ws_, s);
            break;
        }
    }

    void SolverSession::iterate(int iterations, cudaStream_t s)
    {
        if (kind_ == SolverKind::SQS) {
            sqsIterate(iterations, s);
            return;
        }
        for (int it = 0; it < iterations; ++it) {
            switch (kind_) {
            case SolverKind::CGNE:
                cgneStep(A_, x_, ws_, timer_, s);
                break;
            case SolverKind::CGLS:
                cglsStep(A_, x_, static_cast<float>(opt_.cglsEps * opt_.cglsEps), opt_.cglsTol,
                         ws_, timer_, s);
                break;
            case SolverKind::LANDWEBER:
                landweberStep(A_, b_, x_, static_cast<float>(step_), ws_, timer_, s);
                break;
            case SolverKind::APGD:
                apgdStep(A_, x_, static_cast<float>(step_), opt_, ws_, timer_, s);
                break;
            case SolverKind::SIRT:
                sirtStep(A_, b_, x_, static_cast<float>(step_), ws_, timer_, s);
                break;
            case SolverKind::FGM:
            case SolverKind::OGM: {
                const bool ogm = kind_ == SolverKind::OGM;
                // OGM's last iteration uses the factor 8 (OGM.cpp:73): the last of this call
                const float f = (ogm && it == iterations - 1) ? 8.0f : 4.0f;
                const int64_t n = A_.domainSize();
                SolverScalars* S = ws_.scalars.as<SolverScalars>();
                lsqGradient(A_, b_, x_, ws_, timer_, s);
                launchMomentumStep(x_, ws_.vol1.as<float>(), ws_.vol2.as<float>(), lipschitz_,
                                   f, ogm ? 1 : 0, n, S, ws_.partials.as<double>(), s);
                launchMomentumFinish(ws_.partials.as<double>(), S, f,
                                        opt_.momentumEpsilon * opt_.momentumEpsilon, s);
                break;
            }
            case SolverKind::SQS:
                break; // handled above
            }
        }
    }

    SolverSession::~SolverSession()
    {
        if (graph_)
            cudaGraphExecDestroy(graph_);
    }

    void SolverSession::iterateGraph(int iterations, cudaStream_t s)
    {
        if (s == nullptr || s == cudaStreamLegacy)
            throw Error(ELSA_ERROR_INVALID_ARGUMENT,
                        "solver graphs need an explicitly created stream");
        if (timer_.enabled())
            throw Error(ELSA_ERROR_INVALID_ARGUMENT, "solver graphs need timing disabled");
        if (!subsets_.empty())
            throw Error(ELSA_ERROR_NOT_SUPPORTED,
                        "SQS with ordered subsets confirms convergence on the host and cannot "
                        "run as a CUDA graph");
        if (!graph_ || graphIterations_ != iterations) {
            if (graph_) {
                ELSA_CUDA(cudaGraphExecDestroy(graph_));
                graph_ = nullptr;
            }
            cudaGraph_t g = nullptr;
            ELSA_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            try {
                iterate(iterations, s);
            } catch (...) {
                cudaStreamEndCapture(s, &g);
                if (g)
                    cudaGraphDestroy(g);
                throw;
            }
            ELSA_CUDA(cudaStreamEndCapture(s, &g));
            const cudaError_t e = cudaGraphInstantiate(&graph_, g, 0);
            cudaGraphDestroy(g);
            ELSA_CUDA(e);
            graphIterations_ = iterations;
        }
        ELSA_CUDA(cudaGraphLaunch(graph_, s));
    }

    BatchedCgne::BatchedCgne(std::vector<Projector*> ops, std::vector<const float*> b,
                             std::vector<float*> x, cudaStream_t s)
        : ops_(std::move(ops)), x_(std::move(x))
    {
        const size_t n = ops_.size();
        if (n == 0 || b.size() != n || x_.size() != n)
            throw Error(ELSA_ERROR_INVALID_ARGUMENT, "BatchedCgne: invalid instance lists");
        scalars_ = std::make_unique<DeviceBuffer>(sizeof(SolverScalars) * n);
        ELSA_CUDA(cudaMemsetAsync(scalars_->as<SolverScalars>(), 0, sizeof(SolverScalars) * n, s));
        std::vector<const float*> sinos;
        std::vector<float*> qs;
        std::vector<CgBatchEntry> entries(n);
        for (size_t i = 0; i < n; ++i) {
            Projector& A = *ops_[i];
            const int64_t dn = A.domainSize();
            maxN_ = std::max(maxN_, dn);
            r_.push_back(std::make_unique<DeviceBuffer>(sizeof(float) * dn));
            c_.push_back(std::make_unique<DeviceBuffer>(sizeof(float) * dn));
            q_.push_back(std::make_unique<DeviceBuffer>(sizeof(float) * dn));
            sino_.push_back(std::make_unique<DeviceBuffer>(sizeof(float) * A.rangeSize()));
            partials_.push_back(std::make_unique<DeviceBuffer>(sizeof(double) * kReduceBlocks));
            sinos.push_back(sino_.back()->as<float>());
            qs.push_back(q_.back()->as<float>());
            SolverScalars* S = scalars_->as<SolverScalars>() + i;
            entries[i] = CgBatchEntry{x_[i], r_[i]->as<float>(), c_[i]->as<float>(),
                                      q_[i]->as<float>(), dn, S, partials_[i]->as<double>()};
        }
        plan_ = planJosephAdjointMany(ops_, sinos, qs); // checks that every operator qualifies
        entries_ = std::make_unique<DeviceBuffer>(sizeof(CgBatchEntry) * n);
        ELSA_CUDA(cudaMemcpy(entries_->as<CgBatchEntry>(), entries.data(),
                             sizeof(CgBatchEntry) * n, cudaMemcpyHostToDevice));
        // the begin of cgneBegin (x0 = 0): r = A^T b, x = 0, c = r, kold = |r|^2
        for (size_t i = 0; i < n; ++i) {
            const int64_t dn = ops_[i]->domainSize();
            float* r = r_[i]->as<float>();
            ops_[i]->adjoint(b[i], r, s);
            launchFill(x_[i], 0.0f, dn, s);
            ELSA_CUDA(cudaMemcpyAsync(c_[i]->as<float>(), r, sizeof(float) * dn,
                                      cudaMemcpyDeviceToDevice, s));
            launchSquaredNorm(r, dn, partials_[i]->as<double>(),
                              &(scalars_->as<SolverScalars>() + i)->kold, s);
        }
        for (int k = 0; k < kSideStreams; ++k) {
            ELSA_CUDA(cudaStreamCreateWithFlags(&side_[k], cudaStreamNonBlocking));
            ELSA_CUDA(cudaEventCreateWithFlags(&join_[k], cudaEventDisableTiming));
        }
        ELSA_CUDA(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
    }

    BatchedCgne::~BatchedCgne()
    {
        if (graph_)
            cudaGraphExecDestroy(graph_);
        for (int k = 0; k < kSideStreams; ++k) {
            if (side_[k]) {
                cudaStreamSynchronize(side_[k]);
                cudaStreamDestroy(side_[k]);
            }
            if (join_[k])
                cudaEventDestroy(join_[k]);
        }
        if (fork_)
            cudaEventDestroy(fork_);
    }

    void BatchedCgne::step(cudaStream_t s)
    {
        // forwards: instance i on side stream i mod kSideStreams, joined before the adjoints
        ELSA_CUDA(cudaEventRecord(fork_, s));
        for (int k = 0; k < kSideStreams; ++k)
            ELSA_CUDA(cudaStreamWaitEvent(side_[k], fork_, 0));
        for (size_t i = 0; i < ops_.size(); ++i)
            ops_[i]->forward(c_[i]->as<float>(), sino_[i]->as<float>(), side_[i % kSideStreams]);
        for (int k = 0; k < kSideStreams; ++k) {
            ELSA_CUDA(cudaEventRecord(join_[k], side_[k]));
            ELSA_CUDA(cudaStreamWaitEvent(s, join_[k], 0));
        }
        runJosephAdjointMany(*plan_, s); // q_i = A_i^T A_i c_i
        launchCgneUpdateBatch(entries_->as<CgBatchEntry>(), size(), maxN_, s);
    }

    void BatchedCgne::iterate(int iterations, cudaStream_t s)
    {
        for (int it = 0; it < iterations; ++it)
            step(s);
    }

    void BatchedCgne::iterateGraph(int iterations, cudaStream_t s)
    {
        if (s == nullptr || s == cudaStreamLegacy)
            throw Error(ELSA_ERROR_INVALID_ARGUMENT,
                        "batched solver graphs need an explicitly created stream");
        if (!graph_ || graphIterations_ != iterations) {
            if (graph_) {
                ELSA_CUDA(cudaGraphExecDestroy(graph_));
                graph_ = nullptr;
            }
            cudaGraph_t g = nullptr;
            ELSA_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            try {
                iterate(iterations, s);
            } catch (...) {
                cudaStreamEndCapture(s, &g);
                if (g)
                    cudaGraphDestroy(g);
                throw;
            }
            ELSA_CUDA(cudaStreamEndCapture(s, &g));
            const cudaError_t e = cudaGraphInstantiate(&graph_, g, 0);
            cudaGraphDestroy(g);
            ELSA_CUDA(e);
            graphIterations_ = iterations;
        }
        ELSA_CUDA(cudaGraphLaunch(graph_, s));
    }

    void BatchedCgne::squaredResiduals(double* out, cudaStream_t s)
    {
        std::vector<SolverScalars> h(ops_.size());
        ELSA_CUDA(cudaMemcpyAsync(h.data(), scalars_->as<SolverScalars>(),
                                  sizeof(SolverScalars) * h.size(), cudaMemcpyDeviceToHost, s));
        ELSA_CUDA(cudaStreamSynchronize(s));
        for (size_t i = 0; i < h.size(); ++i)
            out[i] = h[i].kold;
    }

    void solveBatch(SolverSession* const* sessions, int n, int iterations, int streams)
    {
        if (n < 0 || iterations < 0 || streams < 1 || streams > 64)
            throw Error(ELSA_ERROR_INVALID_ARGUMENT, "solveBatch: invalid argument");
        std::vector<cudaStream_t> pool(static_cast<size_t>(streams), nullptr);
        try {
            for (auto& st : pool)
                ELSA_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            for (int i = 0; i < n; ++i)
                sessions[i]->iterateGraph(iterations, pool[static_cast<size_t>(i % streams)]);
            for (auto st : pool)
                ELSA_CUDA(cudaStreamSynchronize(st));
        } catch (...) {
            for (auto st : pool)
                if (st) {
                    cudaStreamSynchronize(st);
                    cudaStreamDestroy(st);
                }
            throw;
        }
        for (auto st : pool)
            cudaStreamDestroy(st);
    }

    double SolverSession::squaredResidual(cudaStream_t s)
    {
        SolverScalars h;
        ELSA_CUDA(cudaMemcpyAsync(&h, ws_.scalars.as<SolverScalars>(), sizeof(h),
                                  cudaMemcpyDeviceToHost, s));
        ELSA_CUDA(cudaStreamSynchronize(s));
        if (kind_ == SolverKind::APGD || kind_ == SolverKind::FGM || kind_ == SolverKind::OGM ||
            kind_ == SolverKind::SQS)
            return h.k;
        if (kind_ == SolverKind::SIRT)
            return 0.0;
        if (kind_ == SolverKind::LANDWEBER)
            return 0.0;
        return h.kold;
    }
} // namespace elsa_b200
