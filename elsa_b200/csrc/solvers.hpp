// Device solvers and their scratch buffers.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "projector.hpp"
#include "vecops.cuh"

namespace elsa_b200
{
    class DeviceBuffer
    {
    public:
        DeviceBuffer() = default;
        explicit DeviceBuffer(size_t bytes);
        ~DeviceBuffer();
        DeviceBuffer(const DeviceBuffer&) = delete;
        DeviceBuffer& operator=(const DeviceBuffer&) = delete;
        template <typename T>
        T* as() const
        {
            return static_cast<T*>(ptr_);
        }
        size_t bytes() const { return bytes_; }

    private:
        void* ptr_ = nullptr;
        size_t bytes_ = 0;
    };

    // Scratch for one solver run: four volume-sized and two sinogram-sized float buffers, the
    // reduction partials and the device scalars.
    struct SolverWorkspace {
        SolverWorkspace(int64_t domain, int64_t range);
        DeviceBuffer vol0, vol1, vol2, vol3, sino0, sino1, partials, scalars;
    };

    void cgneSolve(Projector& A, const float* b, float* x, int iterations, bool useX0,
                   SolverWorkspace& ws, cudaStream_t s);

    // CUDA-event timing of the projector kernels inside solver iterations.
    class KernelTimer
    {
    public:
        ~KernelTimer();
        void enable(bool on) { enabled_ = on; }
        bool enabled() const { return enabled_; }
        // Record a marker on the stream; markers come in (begin, after forward, after adjoint)
        // triples per timed iteration.
        void mark(cudaStream_t s);
        // Synchronize and fold all pending triples into the totals.
        void collect(double& fwdMs, double& adjMs, int64_t& count);

    private:
        bool enabled_ = false;
        std::vector<cudaEvent_t> pending_, pool_;
        double fwdMs_ = 0.0, adjMs_ = 0.0;
        int64_t count_ = 0;
    };

    enum class SolverKind {
        CGNE = 0,
        CGLS = 1,
        LANDWEBER = 2,
        APGD = 3,
        SIRT = 4,
        FGM = 5,
        OGM = 6,
        SQS = 7
    };

    // One ordered subset of an SQS problem: the subset's projector (its views) and measurements.
    struct SubsetRef {
        Projector* A;
        const float* b;
    };

    // Solver options (elsa's constructor arguments). Step sizes <= 0 mean "derive from power
    // iterations", as the reference does when none is given.
    struct SolverOptions {
        double cglsEps = 0.0;  // CGLS damping eps (damp = eps^2), solvers/CGLS.cpp:12-17
        double cglsTol = 1e-4; // CGLS stops once |r|^2 < tol, solvers/CGLS.h:46
        double landweberStep = 0.0; // <= 0: 0.9 * 2 / lambda_max(A^T A)
        double apgdMu = 0.0;        // <= 0: 0.45 / lambda_max(A^T A)
        double apgdEpsilon = 1.1920928955078125e-07; // APGD stops once |grad|^2 <= epsilon
        ProxSpec prox{0, 0, 0.0f, 0.0f, 0.0f};
        int powerIterations = 5; // solvers/PowerIterations.h:11
        double sirtStep = 0.0;   // <= 0: 0.9 * 2 / lambda_max(T A^T M A), solvers/SIRT.cpp
        double momentumEpsilon = 1.1920928955078125e-07; // FGM / OGM: stop once
                                                          // |grad|^2 <= eps^2 |grad_0|^2
        bool sqsMomentum = true;                     // SQS momentum acceleration
        double sqsEpsilon = 1.1920928955078125e-07;  // SQS: stop once |g|^2 <= eps^2 |grad_0|^2
        const float* sqsPreconditioner = nullptr;    // SQS: diagonal applied to the gradient
    };

    // Largest eigenvalue of A^T A by power iterations, solvers/PowerIterations.cpp:10-27
    // (synchronizes once at the end).
    // With rangeScale / domainScale (element-wise, may be null) the operator is
    // diag(domainScale) A^T diag(rangeScale) A (SIRT's T A^T M A).
    double powerIterationsAtA(Projector& A, SolverWorkspace& ws, int iterations, cudaStream_t s,
                              const float* rangeScale = nullptr,
                              const float* domainScale = nullptr);

    // A solver run split into setup and iterations: begin() computes the initial residual,
    // iterate() enqueues iterations asynchronously on the stream (capturable in a CUDA graph
    // when timing is off).
    class SolverSession
    {
    public:
        // subsets: SQS in ordered-subset mode (every subset projector has A's domain and at
        // most A's range); empty for the full problem and for the other kinds.
        SolverSession(SolverKind kind, Projector& A, const float* b, float* x, bool useX0,
                      const SolverOptions& opt, cudaStream_t s,
                      std::vector<SubsetRef> subsets = {});
        ~SolverSession();
        SolverSession(const SolverSession&) = delete;
        SolverSession& operator=(const SolverSession&) = delete;
        void iterate(int iterations, cudaStream_t s);
        // The same iterations as one CUDA graph: captured from iterate() on the first call (and
        // again when `iterations` changes), then launched on s. s must not be the legacy default
        // stream; timing must be off.
        void iterateGraph(int iterations, cudaStream_t s);
        double squaredResidual(cudaStream_t s); // synchronizes
        KernelTimer& timer() { return timer_; }
        Projector& op() { return A_; }
        double stepSize() const { return step_; }

    private:
        SolverKind kind_;
        SolverOptions opt_;
        double step_ = 0.0;
        Projector& A_;
        const float* b_;
        float* x_;
        SolverWorkspace ws_;
        KernelTimer timer_;
        float lipschitz_ = 0.0f;
        cudaGraphExec_t graph_ = nullptr;
        int graphIterations_ = -1;
        std::vector<SubsetRef> subsets_;
        bool hostDone_ = false; // SQS with subsets: convergence confirmed on the host
        void sqsIterate(int iterations, cudaStream_t s);
    };

    // CGNE split around the reduction of its normal-operator results, for solves whose
    // projector is spread over ranks by views (A = [A_0; A_1; ...], A^T A = sum_r A_r^T A_r):
    // every rank computes its local A_r^T b and A_r^T A_r c into caller buffers, the caller sums
    // them across the ranks in place (an all-reduce), and every rank then performs the same
    // update, so all ranks hold identical x, r, c and scalars. Scalars stay in device memory; no
    // call waits on the host. solvers/CGNE.cpp:20-78 with x0 = 0.
    class SplitCgne
    {
    public:
        SplitCgne(Projector& A, float* x);
        void backprojectData(const float* b, float* atb, cudaStream_t s); // atb = A_r^T b_r
        void begin(const float* atb, cudaStream_t s); // x = 0, r = c = atb (reduced), kold = |r|^2
        void applyNormal(float* q, cudaStream_t s);   // q = A_r^T A_r c
        void update(const float* q, cudaStream_t s);  // alpha, x, r, beta, c from the reduced q
        const double* squaredResidualDevice() const;  // |r|^2 of the last update (device)
        Projector& op() { return A_; }

    private:
        Projector& A_;
        float* x_;
        SolverWorkspace ws_;
    };

    // Many CGNE solves (x0 = 0) on 3D Joseph operators advanced together: per iteration every
    // operator's forward (fanned out over side streams), then all matched adjoints in one launch
    // per driving-axis grid (planJosephAdjointMany), then all vector updates in five launches
    // (launchCgneUpdateBatch). Every instance's iterates equal those of its own SolverSession
    // bit for bit. iterateGraph captures the batched iterations as one CUDA graph.
    class BatchedCgne
    {
    public:
        BatchedCgne(std::vector<Projector*> ops, std::vector<const float*> b,
                    std::vector<float*> x, cudaStream_t s);
        ~BatchedCgne();
        BatchedCgne(const BatchedCgne&) = delete;
        BatchedCgne& operator=(const BatchedCgne&) = delete;
        void iterate(int iterations, cudaStream_t s);
        void iterateGraph(int iterations, cudaStream_t s);
        void squaredResiduals(double* out, cudaStream_t s); // |r|^2 per instance; synchronizes
        int size() const { return static_cast<int>(ops_.size()); }

    private:
        static constexpr int kSideStreams = 4;
        std::vector<Projector*> ops_;
        std::vector<float*> x_;
        std::vector<std::unique_ptr<DeviceBuffer>> r_, c_, q_, sino_, partials_;
        std::unique_ptr<DeviceBuffer> scalars_, entries_;
        std::shared_ptr<AdjointManyPlan> plan_;
        int64_t maxN_ = 0;
        cudaStream_t side_[kSideStreams] = {};
        cudaEvent_t fork_ = nullptr, join_[kSideStreams] = {};
        cudaGraphExec_t graph_ = nullptr;
        int graphIterations_ = -1;
        void step(cudaStream_t s);
    };

    // Runs `iterations` iterations of every session, each as its CUDA graph, spread round-robin
    // over `streams` concurrent streams (the sessions must use distinct projectors and buffers);
    // returns when all have finished.
    void solveBatch(SolverSession* const* sessions, int n, int iterations, int streams);
} // namespace elsa_b200
