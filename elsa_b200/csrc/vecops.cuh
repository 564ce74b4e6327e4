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
        double aux[2]; // aux[0]: |c|^2 for damped CGLS
        int done;      // set once a convergence test passed; later updates become no-ops
        int pad;
    };

    // Proximal operators of APGD (proximal_operators/ProximalBoxConstraint.cpp,
    // ProximalL1.cpp): kind 0 identity, 1 box [lo, hi] (flags bit 0 lower, bit 1 upper),
    // 2 L1 with weight sigma.
    struct ProxSpec {
        int kind;
        int flags;
        float lo, hi, sigma;
    };

    // One CG instance of a batched solve: x, r, c (direction), q (normal-operator result), the
    // element count, its scalars and its kReduceBlocks partial sums.
    struct CgBatchEntry {
        float* x;
        float* r;
        float* c;
        const float* q;
        int64_t n;
        SolverScalars* S;
        double* partials;
    };

    // The CGNE update (dot <c, q> -> den, step, norm, direction) of `count` instances in five
    // launches; every instance runs the blocks and summation order of the single-instance
    // launches (launchDot, launchCgStep, launchCgFinishNorm, launchCgDirection), so its results
    // are bit-identical to theirs. entries: device array; maxN: largest n.
    void launchCgneUpdateBatch(const CgBatchEntry* entries, int count, int64_t maxN,
                               cudaStream_t s);

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

    // CGLS: alpha = kold / (den (+ damp*|c|^2)); x += alpha c; s -= alpha q (no-op once done)
    void launchCglsStep(float* x, float* sres, const float* c, const float* q, int64_t nx,
                        int64_t ns, SolverScalars* S, float damp, cudaStream_t s);
    // r -= damp*x (damping), partial |r|^2 -> partials
    void launchDampNorm(float* r, const float* x, float damp, int64_t n, double* partials,
                        cudaStream_t s);
    // S->done |= (S->kold < tol)
    void launchCheckTol(SolverScalars* S, double tol, cudaStream_t s);
    // c = r + beta*c unless done
    void launchCgDirectionGuarded(const float* r, float* c, int64_t n, const SolverScalars* S,
                                  cudaStream_t s);
    // out = in - b (out may alias in or b)
    void launchSub(const float* in, const float* b, float* out, int64_t n, cudaStream_t s);
    // x -= step*q (Landweber)
    void launchAxpyMinus(float* x, float step, const float* q, int64_t n, cudaStream_t s);
    // u = u / sqrt(*normSq) (power iterations)
    void launchScaleByInvNorm(float* u, const double* normSq, int64_t n, cudaStream_t s);
    // APGD iteration body on the domain: z = y - mu*grad; x = prox(z); t = (1+sqrt(1+4tp^2))/2;
    // y = x + ((tp-1)/t)(x - xPrev); xPrev = x; partial |grad|^2 -> partials. No-op once done.
    void launchApgdStep(float* x, float* xPrev, float* y, const float* grad, float mu,
                        ProxSpec prox, int64_t n, const SolverScalars* S, double* partials,
                        cudaStream_t s);
    // *result = <x, y> with the partial sums in a fixed device array instead of caller scratch
    // (noalloc.cu; asynchronous, allocates nothing, n <= ELSA_DOT_NO_ALLOC_MAX_ELEMENTS).
    void dotNoAlloc(const float* x, const float* y, int64_t n, double* result, cudaStream_t s);
    // out = 1 / (in + lift) (SIRT's row and column sums, solvers/SIRT.cpp:28-41)
    void launchReciprocal(const float* in, float lift, float* out, int64_t n, cudaStream_t s);
    // out = (a - b) * m (out may alias a)
    void launchSubMul(const float* a, const float* b, const float* m, float* out, int64_t n,
                      cudaStream_t s);
    // x = x - step * (t * q) (SIRT update)
    void launchScaledStep(float* x, float step, const float* t, const float* q, int64_t n,
                          cudaStream_t s);
    // u = u * m (element-wise, in place)
    void launchMul(float* u, const float* m, int64_t n, cudaStream_t s);
    // FGM / OGM body (solvers/FGM.cpp:48-73, OGM.cpp:62-90): y = x - grad / L;
    // theta = 0.5 (1 + sqrt(1 + f theta_prev^2)); x = y + (theta_prev - 1) / theta (y - yPrev)
    // [- ogm * theta_prev / theta * grad / L]; yPrev = y; partial |grad|^2. No-op once done.
    void launchMomentumStep(float* x, float* yPrev, const float* grad, float lipschitz, float f,
                            int ogm, int64_t n, const SolverScalars* S, double* partials,
                            cudaStream_t s);
    // S->tPrev = theta (with factor f); S->k = sum(partials);
    // S->done |= (S->k <= relTol * S->aux[1])
    void launchMomentumFinish(const double* partials, SolverScalars* S, float f, double relTol,
                              cudaStream_t s);
    // S->tPrev = t; S->k = sum(partials); S->done |= (S->k <= eps)
    void launchApgdFinish(const double* partials, SolverScalars* S, double eps, cudaStream_t s);

    // SQS (solvers/SQS.cpp:105-142), S->alpha = t, S->beta = prevT (float values), S->aux[1] =
    // the convergence threshold. Step: g = P g (when P is given); partials = sum g^2; unless
    // S->done: x = x - nSub * (D g) and, with momentum, nextT = 1 + sqrt(1 + 4 t t) / 2,
    // x = x + prevT / nextT * (x - prevX), prevX = x. Float operations in the reference's order.
    void launchSqsStep(float* x, float* prevX, const float* g, const float* D, const float* P,
                       float nSub, int momentum, int64_t n, const SolverScalars* S,
                       double* partials, cudaStream_t s);
    // S->k = sum(partials); unless S->done: if S->k <= S->aux[1] set S->done (full problem) or
    // S->aux[0] = 1 (ordered subsets: the caller confirms with the full gradient); with momentum
    // prevT = t, t = nextT.
    void launchSqsFinish(const double* partials, SolverScalars* S, int subsetMode, int momentum,
                         cudaStream_t s);
    // S->alpha = S->beta = 1, S->aux[0] = 0, S->done = 0, S->aux[1] = S->k * eps2 (S->k holds
    // |grad_0|^2).
    void launchSqsBegin(SolverScalars* S, double eps2, cudaStream_t s);
    // *value = 1 (device int)
    void launchSetFlag(int* flag, cudaStream_t s);
} // namespace elsa_b200
