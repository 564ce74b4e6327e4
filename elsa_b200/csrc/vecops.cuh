// Fused vector operations on float data with float64 reductions.
//
// Reductions are deterministic: a fixed grid of kReduceBlocks blocks writes one partial per
// block (each thread sums a fixed subset of the elements), and a single block folds the partials
// in a fixed tree order. Scalars stay in device memory so that solver iterations never wait for
// the host.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace elsa_b200
{
    constexpr int kReduceBlocks = 592; // 4 x 148 SMs
    constexpr int kReduceThreads = 256;

    // Solver scalars kept on the device (float64).
    struct SolverScalars {
        double kold;   // previous squared residual norm
        double k;      // current squared residual norm
        double den;    // denominator of the step (e.g. <c, A^T A c>)
        double alpha;  // step length
        double beta;   // direction update
        double tPrev;  // FISTA momentum t_{k-1}
        double aux[2]; // spare
    };

    // partials: device buffer of kReduceBlocks doubles.
    void launchDot(const float* x, const float* y, int64_t n, double* partials, double* result,
                   cudaStream_t s);
    void launchSquaredNorm(const float* x, int64_t n, double* partials, double* result,
                           cudaStream_t s);
    // out = a*x + b*y (out may alias x or y)
    void launchLincomb(float a, const float* x, float b, const float* y, float* out, int64_t n,
                       cudaStream_t s);
    // out = a*x + b*y with a, b read from the device (a = sa ? *sa : ca, same for b)
    void launchLincombDev(const double* sa, float ca, const float* x, const double* sb, float cb,
                          const float* y, float* out, int64_t n, cudaStream_t s);
    void launchFill(float* x, float value, int64_t n, cudaStream_t s);
    void launchScale(float* x, float value, int64_t n, cudaStream_t s);

    // CG building blocks (see CGNE/CGLS in solvers.cu).
    // x += alpha*c; r -= alpha*q with alpha = S->kold / S->den; partial sums of |r|^2.
    void launchCgStep(float* x, float* r, const float* c, const float* q, int64_t n,
                      SolverScalars* S, double* partials, cudaStream_t s);
    // S->k = sum(partials); S->beta = S->k / S->kold; S->kold = S->k
    void launchCgFinishNorm(const double* partials, SolverScalars* S, cudaStream_t s);
    // S->den = sum(partials) (+ extra * S->aux[0] if extra != 0)
    void launchFinishDen(const double* partials, SolverScalars* S, cudaStream_t s);
    // c = r + beta*c
    void launchCgDirection(const float* r, float* c, int64_t n, const SolverScalars* S,
                           cudaStream_t s);
} // namespace elsa_b200
