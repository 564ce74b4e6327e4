// Host lookup tables of the voxel-driven projectors, see luts.hpp. Compiled with
// -ffp-contract=off: every operation rounds like elsa's host code.
#include "luts.hpp"

#include <cmath>
#include <functional>

#include "internal.cuh"

namespace elsa_b200
{
    namespace
    {
        // Polynomial approximations of I_0 and I_1 (Abramowitz & Stegun 9.8.1-9.8.4), evaluated
        // in Horner form with the coefficient order of core/Utilities/Bessel.cpp:8-72.
        double horner(const double* c, int n, double y)
        {
            double p = c[n - 1];
            for (int i = n - 2; i >= 0; --i)
                p = c[i] + y * p;
            return p;
        }

        double besselI0(double x)
        {
            const double ax = std::abs(x);
            if (ax < 3.75) {
                static const double c[] = {1.0,       3.5156229, 3.0899424, 1.2067492,
                                           0.2659732, 0.360768e-1, 0.45813e-2};
                return horner(c, 7, std::pow(x / 3.75, 2));
            }
            static const double c[] = {0.39894228,   0.1328592e-1, 0.225319e-2,
                                       -0.157565e-2, 0.916281e-2,  -0.2057706e-1,
                                       0.2635537e-1, -0.1647633e-1, 0.392377e-2};
            return (std::exp(ax) / std::sqrt(ax)) * horner(c, 9, 3.75 / ax);
        }

        double besselI1(double x)
        {
            const double ax = std::abs(x);
            double r;
            if (ax < 3.75) {
                static const double c[] = {0.5,        0.87890594, 0.51498869, 0.15084934,
                                           0.2658733e-1, 0.301532e-2, 0.32411e-3};
                r = ax * horner(c, 7, std::pow(x / 3.75, 2));
            } else {
                // the reference's innermost step subtracts y * c8 (Bessel.cpp:60-61)
                const double y = 3.75 / ax;
                double p = 0.1787654e-1 - y * 0.420059e-2;
                static const double c[] = {0.39894228,   -0.3988024e-1, -0.362018e-2,
                                           0.163801e-2,  -0.1031555e-1, 0.2282967e-1,
                                           -0.2895312e-1};
                for (int i = 6; i >= 0; --i)
                    p = c[i] + y * p;
                r = p * (std::exp(ax) / std::sqrt(ax));
            }
            return x < 0.0 ? -r : r;
        }

        // ---- projected blob (data_t = float), projectors/Blobs.h ------------------------------
        float blobValue(float s, float a, float alpha, int m)
        {
            const float sda = s / a;
            const float w = 1.f - std::pow(sda, 2.f);
            if (!(w > 1.0e-10))
                return 0.0f;
            const float arg = alpha * std::sqrt(w);
            switch (m) {
            case 0:
                return (2.f * a / alpha) * std::sinh(arg) / static_cast<float>(besselI(0, alpha));
            case 1:
                return (2.f * a / alpha) * std::sqrt(w) * (std::cosh(arg) - std::sinh(arg) / arg) /
                       static_cast<float>(besselI(1, alpha));
            case 2:
                return (2.f * a / alpha) * w *
                       ((3.f / (arg * arg) + 1.f) * std::sinh(arg) - (3.f / arg) * std::cosh(arg)) /
                       static_cast<float>(besselI(2, alpha));
            default:
                throw Error(ELSA_ERROR_INVALID_ARGUMENT, "blob order must be 0, 1 or 2");
            }
        }

        // derivative (normalized = false) or derivative / s (normalized = true); the reference
        // mixes double literals in, so the outer products run in double
        float blobDerivative(float s, float a, float alpha, int m, bool normalized)
        {
            const float sda = s / a;
            const float sdas = static_cast<float>(std::pow(sda, 2));
            const float w = static_cast<float>(1.0 - sdas);
            if (!(w > 1.0e-10))
                return 0.0f;
            const float arg = alpha * std::sqrt(w);
            if (m == 1) {
                const double f = normalized ? (-2.0 / a) : (-2.0 * s / a);
                return static_cast<float>(f * std::sinh(arg) / besselI(1, alpha));
            }
            if (m == 2) {
                const double f = normalized ? (-2.0 / alpha / a) : (-2.0 * s / alpha / a);
                return static_cast<float>(f * (std::cosh(arg) * arg - std::sinh(arg)) /
                                          besselI(2, alpha));
            }
            throw Error(ELSA_ERROR_INVALID_ARGUMENT, "blob derivative needs order 1 or 2");
        }

        // ---- B-splines, projectors/BSplines.h -------------------------------------------------
        int64_t factorialOf(int64_t n) { return n <= 1 ? 1 : n * factorialOf(n - 1); }

        int64_t binomial(int64_t n, int64_t k)
        {
            if (k > n)
                return 0;
            if (k == 0 || k == n)
                return 1;
            if (k == 1 || k == n - 1)
                return n;
            return (k + k < n) ? (binomial(n - 1, k - 1) * n) / k
                               : (binomial(n - 1, k) * n) / (n - k);
        }

        // Unser's explicit form: sum_n (-1)^n C(m+1, n) (x + (m+1)/2 - n)_+^m / m!, with the
        // reference's promotions (integer powers in double, T accumulator).
        template <typename T>
        T bspline(T x, int m)
        {
            const T xs = x + static_cast<T>(m + 1) / T{2};
            T acc = 0;
            for (int n = 0; n <= m + 1; ++n) {
                const T d = xs - static_cast<T>(n);
                const T step = d == 0 ? T(0) : (d < 0 ? T(0) : T(1));
                const double power = std::pow(static_cast<double>(d), static_cast<double>(m));
                const T coeff = static_cast<T>(binomial(m + 1, n));
                const double sign = std::pow(static_cast<double>(static_cast<T>(-1)),
                                             static_cast<double>(n)) /
                                    static_cast<double>(static_cast<T>(factorialOf(m)));
                acc += static_cast<T>(step * power * coeff * sign);
            }
            return acc;
        }

        float bsplineCentered(float x, int m, int dim)
        {
            float v = bspline<float>(x, m);
            for (int i = 1; i < dim; ++i)
                v *= bspline<float>(0.f, m);
            return v;
        }

        float bsplineDerivativeCentered(float x, int m, int dim)
        {
            float v = static_cast<float>(bspline<double>(x + 0.5, m - 1) -
                                         bspline<double>(x - 0.5, m - 1));
            for (int i = 1; i < dim; ++i)
                v = static_cast<float>(v * bspline<double>(0., m));
            return v;
        }

        VoxelLut tabulate(const std::function<float(float)>& f, float support, int samples)
        {
            VoxelLut lut;
            lut.support = support;
            lut.values.resize(static_cast<size_t>(samples));
            const float step = support / static_cast<float>(samples - 1);
            for (int i = 0; i < samples; ++i)
                lut.values[static_cast<size_t>(i)] = f(step * static_cast<float>(i));
            return lut;
        }
    } // namespace

    double besselI(int m, double x)
    {
        switch (m) {
        case 0:
            return besselI0(x);
        case 1:
            return besselI1(x);
        case 2:
            return x == 0 ? 0 : besselI0(x) - (2.0 / x) * besselI1(x);
        case 3:
            return x == 0 ? 0 : besselI1(x) - (4.0 / x) * besselI(2, x);
        case 4:
            return x == 0 ? 0 : besselI(2, x) - (6.0 / x) * besselI(3, x);
        default:
            break;
        }
        if (x == 0.0)
            return 0.0;
        // Miller's algorithm: recur downwards from an order well above m, renormalise with I_0
        const double tox = 2.0 / std::abs(x);
        double result = 0.0, bip = 0.0, bi = 1.0;
        const int64_t start = 2 * (m + static_cast<int64_t>(std::sqrt(40.0 * m)));
        for (int64_t j = start; j > 0; --j) {
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
        result *= besselI0(x) / bi;
        return (x < 0.0 && (m % 2) == 0) ? -result : result;
    }

    VoxelLut blobLut(float radius, float alpha, int order, LutProfile profile, int samples)
    {
        if (!(radius > 0.0f) || !(alpha > 0.0f) || order < 0 || order > 2 || samples < 2)
            throw Error(ELSA_ERROR_INVALID_ARGUMENT,
                        "blob: need radius > 0, alpha > 0 and order in {0, 1, 2}");
        if (profile == LutProfile::Value)
            return tabulate([=](float s) { return blobValue(s, radius, alpha, order); }, radius,
                            samples);
        const bool normalized = profile == LutProfile::NormalizedGradient;
        return tabulate(
            [=](float s) {
                return order > 0 ? blobDerivative(s, radius, alpha, order, normalized) : 0.0f;
            },
            radius, samples);
    }

    VoxelLut bsplineLut(int dim, int order, LutProfile profile, int samples)
    {
        if (dim < 2 || dim > 3 || order < 0 || order > 10 || samples < 2)
            throw Error(ELSA_ERROR_INVALID_ARGUMENT,
                        "B-spline: need dim in {2, 3} and order in [0, 10]");
        const float support = static_cast<float>((order + 1) * 0.5);
        const int d = dim - 1;
        switch (profile) {
        case LutProfile::Value:
            return tabulate([=](float x) { return bsplineCentered(x, order, d); }, support,
                            samples);
        case LutProfile::Derivative:
            return tabulate(
                [=](float x) { return order > 0 ? bsplineDerivativeCentered(x, order, d) : 0.0f; },
                support, samples);
        default:
            return tabulate(
                [=](float x) {
                    if (order <= 0)
                        return 0.0f;
                    if (x == 0)
                        x = 1e-10f;
                    return bsplineDerivativeCentered(x, order, d) / x;
                },
                support, samples);
        }
    }
} // namespace elsa_b200
