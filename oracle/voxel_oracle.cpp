// Oracle restatement of elsa's voxel-driven (blob / B-spline) projectors, their lookup tables and
// the modified Bessel functions they use.
//
// TEST INFRASTRUCTURE ONLY: tests/, the smoke check and the benchmark's CPU-baseline arm call it
// as the checker; the product never links it.
//
// Followed files (reference paths inside elsa/):
//   core/Utilities/Bessel.cpp:6-137          bessi0..bessi4, bessi (Abramowitz & Stegun 9.8.1-9.8.4
//                                            polynomial approximations, recurrence 9.6.26)
//   projectors/Blobs.h:67-210               projected blob, its derivative and normalized gradient
//   projectors/BSplines.h:22-99,132-208      B-spline, centred n-d B-spline and its derivative
//   projectors/Luts.hpp:14-83                LUT generation (N samples on [0, support]) and lerp
//   projectors/VoxelComputation.h:20-185     visitDetector, forwardVoxel, backwardVoxel
// Types follow the reference template instantiation for data_t = float (geometry real_t = float,
// some intermediate terms in double exactly where the reference mixes double literals in).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <functional>
#include <vector>

namespace vox
{
    using index_t = int64_t;

    // ---- Bessel.cpp ---------------------------------------------------------------------------
    static double bessi0(double x)
    {
        const double ax = std::abs(x);
        if (ax < 3.75) {
            const double y = std::pow(x / 3.75, 2);
            const double p1 = 0.360768e-1 + y * 0.45813e-2;
            const double p2 = 0.2659732 + y * p1;
            const double p3 = 1.2067492 + y * p2;
            const double p4 = 3.0899424 + y * p3;
            const double p5 = 3.5156229 + y * p4;
            return 1.0 + y * p5;
        }
        const double y = 3.75 / ax;
        const double p1 = -0.1647633e-1 + y * 0.392377e-2;
        const double p2 = 0.2635537e-1 + y * p1;
        const double p3 = -0.2057706e-1 + y * p2;
        const double p4 = 0.916281e-2 + y * p3;
        const double p5 = -0.157565e-2 + y * p4;
        const double p6 = 0.225319e-2 + y * p5;
        const double p7 = 0.1328592e-1 + y * p6;
        const double p8 = 0.39894228 + y * p7;
        return (std::exp(ax) / std::sqrt(ax)) * p8;
    }

    static double bessi1(double x)
    {
        const double ax = std::abs(x);
        double result;
        if (ax < 3.75) {
            const double y = std::pow(x / 3.75, 2);
            const double p1 = 0.301532e-2 + y * 0.32411e-3;
            const double p2 = 0.2658733e-1 + y * p1;
            const double p3 = 0.15084934 + y * p2;
            const double p4 = 0.51498869 + y * p3;
            const double p5 = 0.87890594 + y * p4;
            const double p6 = 0.5 + y * p5;
            result = ax * p6;
        } else {
            const double y = 3.75 / ax;
            const double p1 = 0.1787654e-1 - y * 0.420059e-2;
            const double p2 = -0.2895312e-1 + y * p1;
            const double p3 = 0.2282967e-1 + y * p2;
            const double p4 = -0.1031555e-1 + y * p3;
            const double p5 = 0.163801e-2 + y * p4;
            const double p6 = -0.362018e-2 + y * p5;
            const double p7 = -0.3988024e-1 + y * p6;
            const double p8 = 0.39894228 + y * p7;
            result = p8 * (std::exp(ax) / std::sqrt(ax));
        }
        return x < 0.0 ? -result : result;
    }

    static double bessi2(double x) { return x == 0 ? 0 : bessi0(x) - ((2 * 1) / x) * bessi1(x); }
    static double bessi3(double x) { return x == 0 ? 0 : bessi1(x) - ((2 * 2) / x) * bessi2(x); }
    static double bessi4(double x) { return x == 0 ? 0 : bessi2(x) - ((2 * 3) / x) * bessi3(x); }

    // Miller's downward recurrence for m > 4 (Bessel.cpp:99-135)
    static double bessi(index_t m, double x)
    {
        switch (m) {
        case 0:
            return bessi0(x);
        case 1:
            return bessi1(x);
        case 2:
            return bessi2(x);
        case 3:
            return bessi3(x);
        case 4:
            return bessi4(x);
        default:
            break;
        }
        if (x == 0.0)
            return 0.0;
        const double tox = 2.0 / std::abs(x);
        double result = 0.0, bip = 0.0, bi = 1.0;
        for (index_t j = 2 * (m + static_cast<index_t>(std::sqrt(40.0 * static_cast<double>(m))));
             j > 0; --j) {
            const double bim = bip + static_cast<double>(j) * tox * bi;
            bip = bi;
            bi = bim;
            if (std::abs(bi) > 1.0e10) {
                result *= 1.0e-10;
                bi *= 1.0e-10;
                bip *= 1.0e-10;
            }
            if (j == m)
                result = bip;
        }
        result *= bessi0(x) / bi;
        return (x < 0.0 && (m % 2) == 0) ? -result : result;
    }

    // ---- Blobs.h (data_t = float) -------------------------------------------------------------
    static float blobProjected(float s, float a, float alpha, index_t m)
    {
        const float sda = s / a;
        const float sdas = std::pow(sda, 2.f);
        const float w = 1.f - sdas;
        if (w > 1.0e-10) {
            const float arg = alpha * std::sqrt(w);
            if (m == 0)
                return (2.f * a / alpha) * std::sinh(arg) / static_cast<float>(bessi0(alpha));
            if (m == 1)
                return (2.f * a / alpha) * std::sqrt(w) * (std::cosh(arg) - std::sinh(arg) / arg) /
                       static_cast<float>(bessi1(alpha));
            if (m == 2)
                return (2.f * a / alpha) * w *
                       ((3.f / (arg * arg) + 1.f) * std::sinh(arg) - (3.f / arg) * std::cosh(arg)) /
                       static_cast<float>(bessi2(alpha));
            return std::nanf("");
        }
        return 0.0f;
    }

    static float blobDerivativeProjected(float s, float a, float alpha, int m)
    {
        const float sda = s / a;
        const float sdas = static_cast<float>(std::pow(sda, 2));
        const float w = static_cast<float>(1.0 - sdas);
        if (w > 1.0e-10) {
            const float arg = alpha * std::sqrt(w);
            if (m == 1)
                return static_cast<float>((-2.0 * s / a) * std::sinh(arg) / bessi1(alpha));
            if (m == 2)
                return static_cast<float>((-2.0 * s / alpha / a) *
                                          (std::cosh(arg) * arg - std::sinh(arg)) / bessi2(alpha));
            return std::nanf("");
        }
        return 0.0f;
    }

    static float blobNormalizedGradient(float s, float a, float alpha, int m)
    {
        const float sda = s / a;
        const float sdas = static_cast<float>(std::pow(sda, 2));
        const float w = static_cast<float>(1.0 - sdas);
        if (w > 1.0e-10) {
            const float arg = alpha * std::sqrt(w);
            if (m == 1)
                return static_cast<float>((-2.0 / a) * std::sinh(arg) / bessi1(alpha));
            if (m == 2)
                return static_cast<float>((-2.0 / alpha / a) *
                                          (std::cosh(arg) * arg - std::sinh(arg)) / bessi2(alpha));
            return std::nanf("");
        }
        return 0.0f;
    }

    // ---- BSplines.h ---------------------------------------------------------------------------
    static index_t factorial(index_t n) { return (n == 1 || n == 0) ? 1 : factorial(n - 1) * n; }

    static index_t binom(index_t n, index_t k)
    {
        return (k > n)                  ? 0
               : (k == 0 || k == n)     ? 1
               : (k == 1 || k == n - 1) ? n
               : (k + k < n)            ? (binom(n - 1, k - 1) * n) / k
                                        : (binom(n - 1, k) * n) / (n - k);
    }

    template <typename T>
    static T heaviside(T x, T c)
    {
        return x == 0 ? c : (x < 0 ? T(0) : T(1));
    }

    // bspline1d_evaluate<T>: std::pow<T>(., integer) promotes to double (libstdc++).
    template <typename T>
    static T bspline1d(T x, index_t m)
    {
        const T xs = x + static_cast<T>(m + 1) / T{2};
        T res = 0;
        for (int n = 0; n <= m + 1; ++n) {
            const T nf = static_cast<T>(n);
            const T tmp1 = heaviside<T>(xs - nf, 0);
            const double tmp2 = std::pow(static_cast<double>(xs - nf), static_cast<double>(m));
            const T tmp3 = static_cast<T>(binom(m + 1, n));
            const double tmp4 = std::pow(static_cast<double>(static_cast<T>(-1)),
                                         static_cast<double>(n)) /
                                static_cast<double>(static_cast<T>(factorial(m)));
            res += static_cast<T>(tmp1 * tmp2 * tmp3 * tmp4);
        }
        return res;
    }

    static float ndBsplineCentered(float x, index_t m, index_t dim)
    {
        float res = bspline1d<float>(x, m);
        for (int i = 1; i < dim; ++i)
            res *= bspline1d<float>(0.f, m);
        return res;
    }

    // bsplineDerivative1d_evaluate<float>: x +- 0.5 is double, so both terms run in double
    static float bsplineDerivative1d(float x, index_t m)
    {
        return static_cast<float>(bspline1d<double>(x + 0.5, m - 1) -
                                  bspline1d<double>(x - 0.5, m - 1));
    }

    static float ndBsplineDerivativeCentered(float x, int m, int dim)
    {
        float res = bsplineDerivative1d(x, m);
        for (int i = 1; i < dim; ++i) {
            const double inc = bspline1d<double>(0., m);
            res = static_cast<float>(res * inc);
        }
        return res;
    }

    // ---- Luts.hpp -----------------------------------------------------------------------------
    static void generateLut(const std::function<float(float)>& gen, float support, index_t N,
                            float* out)
    {
        const float step = support / static_cast<float>(N - 1);
        for (index_t i = 0; i < N; ++i)
            out[i] = gen(step * static_cast<float>(i));
    }

    // which: 0 value, 1 derivative, 2 normalized gradient (ProjectedBlob, Blobs.h:233-245)
    static void blobLut(float radius, float alpha, index_t order, int which, index_t N, float* out)
    {
        generateLut(
            [&](float s) -> float {
                if (which == 0)
                    return blobProjected(s, radius, alpha, order);
                if (order <= 0)
                    return 0.0f;
                if (which == 1)
                    return blobDerivativeProjected(s, radius, alpha, static_cast<int>(order));
                return blobNormalizedGradient(s, radius, alpha, static_cast<int>(order));
            },
            radius, N, out);
    }

    // ProjectedBSpline(dim, order), BSplines.h:132-186; support (order + 1) / 2
    static float bsplineSupport(index_t order) { return static_cast<float>((order + 1) * 0.5); }

    static void bsplineLut(index_t dim, index_t order, int which, index_t N, float* out)
    {
        generateLut(
            [&](float x) -> float {
                if (which == 0)
                    return ndBsplineCentered(x, order, dim - 1);
                if (order <= 0)
                    return 0.0f;
                if (which == 1)
                    return ndBsplineDerivativeCentered(x, static_cast<int>(order),
                                                       static_cast<int>(dim - 1));
                if (x == 0)
                    x = 1e-10f;
                return ndBsplineDerivativeCentered(x, static_cast<int>(order),
                                                   static_cast<int>(dim - 1)) /
                       x;
            },
            bsplineSupport(order), N, out);
    }

    // Lut::operator()(float distance), Luts.hpp:61-80 (also used by the ray-driven LutProjector
    // restatement in oracle.cpp)
    float lutLerp(const float* lut, index_t N, float support, float distance)
    {
        const float index = (distance / support) * static_cast<float>(N - 1);
        if (index < 0 || index > static_cast<float>(N - 1))
            return 0;
        const auto a = static_cast<size_t>(std::floor(index));
        const auto b = static_cast<size_t>(std::ceil(index));
        const float fa = lut[a], fb = lut[b];
        const float t = index - static_cast<float>(a);
        return t * fb + (1 - t) * fa;
    }

    // ---- VoxelComputation.h -------------------------------------------------------------------
    struct Pose {
        int dim;
        const float* p; // pose record: P at 0, ext at 27, sdd at 39
        float P(int i, int j) const { return p[i * (dim + 1) + j]; }
        float ext(int i, int j) const { return p[27 + i * (dim + 1) + j]; }
        float sdd() const { return p[39]; }
    };

    struct Footprint {
        float center[2];
        float scaling;
        index_t lo[2], hi[2];
    };

    // Projected centre, scaling and clamped footprint of voxel `coord` (VoxelComputation.h:55-86).
    static Footprint footprint(const Pose& g, const index_t* coord, float radius,
                               const index_t* detDims)
    {
        const int dim = g.dim;
        float h[4];
        for (int i = 0; i < dim; ++i)
            h[i] = static_cast<float>(coord[i]) + 0.5f;
        h[dim] = 1.0f;
        float proj[3], cam[3];
        for (int i = 0; i < dim; ++i) { // P * h and ext * h, sequential sums
            float s = 0.0f, e = 0.0f;
            for (int k = 0; k <= dim; ++k) {
                s = s + g.P(i, k) * h[k];
                e = e + g.ext(i, k) * h[k];
            }
            proj[i] = s;
            cam[i] = e;
        }
        Footprint f{};
        for (int i = 0; i < dim - 1; ++i)
            f.center[i] = proj[i] / proj[dim - 1] - 0.5f;
        float n2 = cam[0] * cam[0];
        for (int i = 1; i < dim; ++i)
            n2 = n2 + cam[i] * cam[i];
        f.scaling = g.sdd() / std::sqrt(n2);
        const float r = f.scaling * radius;
        for (int i = 0; i < dim - 1; ++i) {
            const index_t mn = static_cast<index_t>(std::ceil(f.center[i] - r));
            const index_t mx = static_cast<index_t>(std::floor(f.center[i] + r));
            f.lo[i] = std::max<index_t>(mn, 0);
            f.hi[i] = std::min<index_t>(mx, detDims[i] - 1);
        }
        return f;
    }

    // Weight of one (voxel, pixel) pair: classic lut(|d|), differential 2D lut(|d|) sgn(d0),
    // differential 3D lut(|d|) d0 (VoxelComputation.h:20-38), d = (center - pixel) / scaling.
    static float weight(const float* lut, index_t N, float support, int kind, int dim,
                        const float* d)
    {
        float nrm;
        if (dim == 2)
            nrm = std::sqrt(d[0] * d[0]);
        else
            nrm = std::sqrt(d[0] * d[0] + d[1] * d[1]);
        const float v = lutLerp(lut, N, support, nrm);
        if (kind == 0)
            return v;
        if (dim == 2)
            return v * static_cast<float>((0.0f < d[0]) - (d[0] < 0.0f));
        return v * d[0];
    }

    // Visits the footprint pixels of one voxel in the reference's order.
    // loopMode 1: rows v = lo1..hi1, u = lo0..hi0 (the footprint rectangle).
    // loopMode 0: the reference's CPU loop as written (VoxelComputation.h:88-113): the outer loop
    //   runs hi0-lo0+1 times over rows, the inner one hi1-lo1+1 times along u, and every row
    //   start moves by the difference of the two extents (linear pixel index += nu - ext0); it
    //   equals mode 1 whenever the two extents agree. Pixels it would address outside the view
    //   are skipped here.
    template <class Fn>
    static void visitDetector(const Footprint& f, int dim, const index_t* detDims, int loopMode,
                              Fn apply)
    {
        if (dim == 2) {
            for (index_t i = f.lo[0]; i <= f.hi[0]; ++i) {
                const float d[1] = {(f.center[0] - static_cast<float>(i)) / f.scaling};
                apply(i, d);
            }
            return;
        }
        const index_t nu = detDims[0], nv = detDims[1];
        const index_t ext0 = f.hi[0] - f.lo[0] + 1, ext1 = f.hi[1] - f.lo[1] + 1;
        const index_t rows = loopMode == 0 ? ext0 : ext1;
        const index_t cols = loopMode == 0 ? ext1 : ext0;
        float cur0 = static_cast<float>(f.lo[0]), cur1 = static_cast<float>(f.lo[1]);
        index_t lin = f.lo[1] * nu + f.lo[0]; // linear pixel index inside the view
        for (index_t r = 0; r < rows; ++r) {
            for (index_t c = 0; c < cols; ++c) {
                const float d[2] = {(f.center[0] - cur0) / f.scaling,
                                    (f.center[1] - cur1) / f.scaling};
                if (lin >= 0 && lin < nu * nv)
                    apply(lin, d);
                lin += 1;
                cur0 += 1;
            }
            lin += nu - ext0;
            cur0 -= static_cast<float>(ext0);
            cur1 += 1;
        }
    }

    // forwardVoxel / backwardVoxel (VoxelComputation.h:116-184): the forward sums each pixel over
    // voxels in index order (one pose per thread), the backward sums each voxel over poses and
    // footprint pixels in order.
    template <typename data_t, bool adjoint>
    static void project(int dim, const index_t* volDims, const index_t* detDims, index_t np,
                        const float* poses, const float* lut, index_t N, float support, int kind,
                        int loopMode, const data_t* in, data_t* out)
    {
        index_t nvox = 1;
        for (int i = 0; i < dim; ++i)
            nvox *= volDims[i];
        const index_t npix = dim == 2 ? detDims[0] : detDims[0] * detDims[1];
        auto coordOf = [&](index_t idx, index_t* c) {
            c[0] = idx % volDims[0];
            c[1] = (idx / volDims[0]) % volDims[1];
            if (dim == 3)
                c[2] = idx / (volDims[0] * volDims[1]);
        };
        if (!adjoint) {
            std::fill(out, out + npix * np, data_t(0));
#pragma omp parallel for schedule(dynamic, 1)
            for (index_t p = 0; p < np; ++p) {
                const Pose g{dim, poses + p * 40};
                data_t* view = out + p * npix;
                for (index_t v = 0; v < nvox; ++v) {
                    index_t c[3] = {0, 0, 0};
                    coordOf(v, c);
                    const Footprint f = footprint(g, c, support, detDims);
                    const data_t xv = in[v];
                    visitDetector(f, dim, detDims, loopMode, [&](index_t pix, const float* d) {
                        const data_t w = static_cast<data_t>(weight(lut, N, support, kind, dim, d));
                        view[pix] += xv * w;
                    });
                }
            }
        } else {
            std::fill(out, out + nvox, data_t(0));
#pragma omp parallel for schedule(static)
            for (index_t v = 0; v < nvox; ++v) {
                index_t c[3] = {0, 0, 0};
                coordOf(v, c);
                data_t acc = 0;
                for (index_t p = 0; p < np; ++p) {
                    const Pose g{dim, poses + p * 40};
                    const Footprint f = footprint(g, c, support, detDims);
                    const data_t* view = in + p * npix;
                    visitDetector(f, dim, detDims, loopMode, [&](index_t pix, const float* d) {
                        const data_t w = static_cast<data_t>(weight(lut, N, support, kind, dim, d));
                        acc += w * view[pix];
                    });
                }
                out[v] = acc;
            }
        }
    }
} // namespace vox

extern "C" {

double oracle_bessel(int m, double x) { return vox::bessi(m, x); }

float oracle_blob_projected(float s, float a, float alpha, int m, int which)
{
    if (which == 0)
        return vox::blobProjected(s, a, alpha, m);
    if (which == 1)
        return vox::blobDerivativeProjected(s, a, alpha, m);
    return vox::blobNormalizedGradient(s, a, alpha, m);
}

float oracle_bspline1d(float x, int m) { return vox::bspline1d<float>(x, m); }

void oracle_blob_lut(float radius, float alpha, int order, int which, int64_t n, float* out)
{
    vox::blobLut(radius, alpha, order, which, n, out);
}

void oracle_bspline_lut(int dim, int order, int which, int64_t n, float* out)
{
    vox::bsplineLut(dim, order, which, n, out);
}

float oracle_lut_lerp(const float* lut, int64_t n, float support, float distance)
{
    return vox::lutLerp(lut, n, support, distance);
}

// kind 0 classic, 1 differential; loopMode as in vox::visitDetector
void oracle_voxel_f32(int adjoint, int dim, const int64_t* volDims, const int64_t* detDims,
                      const float* poses, const float* lut, int64_t n, float support, int kind,
                      int loopMode, const float* in, float* out)
{
    const int64_t np = detDims[dim - 1];
    if (adjoint)
        vox::project<float, true>(dim, volDims, detDims, np, poses, lut, n, support, kind,
                                  loopMode, in, out);
    else
        vox::project<float, false>(dim, volDims, detDims, np, poses, lut, n, support, kind,
                                   loopMode, in, out);
}

void oracle_voxel_f64(int adjoint, int dim, const int64_t* volDims, const int64_t* detDims,
                      const float* poses, const float* lut, int64_t n, float support, int kind,
                      int loopMode, const double* in, double* out)
{
    const int64_t np = detDims[dim - 1];
    if (adjoint)
        vox::project<double, true>(dim, volDims, detDims, np, poses, lut, n, support, kind,
                                   loopMode, in, out);
    else
        vox::project<double, false>(dim, volDims, detDims, np, poses, lut, n, support, kind,
                                    loopMode, in, out);
}

} // extern "C"
