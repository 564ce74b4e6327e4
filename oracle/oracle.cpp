// Oracle: a CPU restatement of elsa's reference algorithms for the projector + solver hot path.
//
// TEST INFRASTRUCTURE ONLY. Nothing in the product (the elsa_b200 package, its CUDA kernels or
// its C ABI) may include, link or call this file. Tests, __graft_entry__.smoke() and the CPU
// baseline leg of bench.py use it as the checker.
//
// Every function cites the reference file:line it follows (paths relative to the elsa source
// tree). Eigen 3.4.0, which the reference uses for all small vector/matrix math, is not available
// here, so its evaluation order is restated: small products are coefficient-wise sequential dot
// products with separate multiply and add (no FMA), reductions of <4 elements are sequential.
// Built with -ffp-contract=off so the compiler does not fuse what the reference keeps separate.
//
// Parity is pinned against the reference's own known-answer tests (projectors/tests/*.cpp,
// core/tests/test_Geometry.cpp) re-expressed in tests/test_oracle_kat.py.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include <omp.h>

namespace vox
{
    // Lut::operator() (voxel_oracle.cpp)
    float lutLerp(const float* lut, int64_t N, float support, float distance);
} // namespace vox

namespace orc
{
    using real_t = float;
    using index_t = int64_t;

    // pi as real_t, core/elsaDefines.h:61-66
    constexpr float pi_f() { return static_cast<float>(3.14159265358979323846); }

    // ------------------------------------------------------------------------------------------
    // Small dense matrices, row-major, with Eigen's coefficient-based product order.
    // ------------------------------------------------------------------------------------------
    struct Mat {
        int r = 0, c = 0;
        float a[16] = {0};
        float& operator()(int i, int j) { return a[i * c + j]; }
        float operator()(int i, int j) const { return a[i * c + j]; }
    };

    static Mat zeros(int r, int c)
    {
        Mat m;
        m.r = r;
        m.c = c;
        return m;
    }

    static Mat identity(int r, int c)
    {
        Mat m = zeros(r, c);
        for (int i = 0; i < std::min(r, c); ++i)
            m(i, i) = 1.0f;
        return m;
    }

    // Coefficient-based lazy product (Eigen 3.4 for rows+cols+depth < 20): every coefficient is
    // the sequential sum of lhs(i,k)*rhs(k,j), k = 0..depth-1.
    static Mat mul(const Mat& A, const Mat& B)
    {
        Mat C = zeros(A.r, B.c);
        for (int i = 0; i < A.r; ++i)
            for (int j = 0; j < B.c; ++j) {
                float s = A(i, 0) * B(0, j);
                for (int k = 1; k < A.c; ++k)
                    s = s + A(i, k) * B(k, j);
                C(i, j) = s;
            }
        return C;
    }

    // Matrix-vector product (Eigen GEMV for tiny sizes): per row ((0 + a0*x0) + a1*x1) + ...
    static void matvec(const Mat& A, const float* x, float* y)
    {
        for (int i = 0; i < A.r; ++i) {
            float s = 0.0f;
            for (int k = 0; k < A.c; ++k)
                s = s + A(i, k) * x[k];
            y[i] = s;
        }
    }

    static float seqSqNorm(const float* v, int n)
    {
        float s = v[0] * v[0];
        for (int i = 1; i < n; ++i)
            s = s + v[i] * v[i];
        return s;
    }

    // ------------------------------------------------------------------------------------------
    // Column-pivoting Householder QR solve in float, restating Eigen 3.4's ColPivHouseholderQR
    // (computeInPlace + _solve_impl), used for the camera centre at core/Geometry.cpp:244-246.
    // ------------------------------------------------------------------------------------------
    static void colPivQrSolve(const Mat& Ain, const float* b, float* x)
    {
        const int n = Ain.r; // square
        Mat qr = Ain;
        float hCoeffs[4] = {0};
        int transp[4] = {0};
        float normsUpd[4], normsDir[4];
        for (int k = 0; k < n; ++k) {
            float col[4];
            for (int i = 0; i < n; ++i)
                col[i] = qr(i, k);
            normsDir[k] = std::sqrt(seqSqNorm(col, n));
            normsUpd[k] = normsDir[k];
        }
        const float eps = std::numeric_limits<float>::epsilon();
        float maxNorm = normsUpd[0];
        for (int k = 1; k < n; ++k)
            if (normsUpd[k] > maxNorm)
                maxNorm = normsUpd[k];
        const float thresholdHelper = (maxNorm * eps) * (maxNorm * eps) / float(n);
        const float downdateThreshold = std::sqrt(eps);
        int nonzeroPivots = n;
        for (int k = 0; k < n; ++k) {
            int big = k;
            float bigNorm = normsUpd[k];
            for (int j = k + 1; j < n; ++j)
                if (normsUpd[j] > bigNorm) {
                    bigNorm = normsUpd[j];
                    big = j;
                }
            const float bigSq = bigNorm * bigNorm;
            if (nonzeroPivots == n && bigSq < thresholdHelper * float(n - k))
                nonzeroPivots = k;
            transp[k] = big;
            if (k != big) {
                for (int i = 0; i < n; ++i)
                    std::swap(qr(i, k), qr(i, big));
                std::swap(normsUpd[k], normsUpd[big]);
                std::swap(normsDir[k], normsDir[big]);
            }
            // makeHouseholderInPlace on qr.col(k).tail(n-k)
            const int len = n - k;
            float tailSq = 0.0f;
            if (len > 1) {
                tailSq = qr(k + 1, k) * qr(k + 1, k);
                for (int i = k + 2; i < n; ++i)
                    tailSq = tailSq + qr(i, k) * qr(i, k);
            }
            const float c0 = qr(k, k);
            float tau, beta;
            const float tol = std::numeric_limits<float>::min();
            if (tailSq <= tol) {
                tau = 0.0f;
                beta = c0;
                for (int i = k + 1; i < n; ++i)
                    qr(i, k) = 0.0f;
            } else {
                beta = std::sqrt(c0 * c0 + tailSq);
                if (c0 >= 0.0f)
                    beta = -beta;
                const float denom = c0 - beta;
                for (int i = k + 1; i < n; ++i)
                    qr(i, k) = qr(i, k) / denom;
                tau = (beta - c0) / beta;
            }
            hCoeffs[k] = tau;
            qr(k, k) = beta;
            // applyHouseholderOnTheLeft to bottomRightCorner(n-k, n-k-1)
            const int cols = n - k - 1;
            if (cols > 0) {
                if (len == 1) {
                    for (int j = k + 1; j < n; ++j)
                        qr(k, j) = qr(k, j) * (1.0f - tau);
                } else if (tau != 0.0f) {
                    float tmp[4];
                    for (int j = k + 1; j < n; ++j) {
                        float s = 0.0f;
                        for (int i = k + 1; i < n; ++i)
                            s = s + qr(i, k) * qr(i, j);
                        tmp[j] = s + qr(k, j);
                    }
                    for (int j = k + 1; j < n; ++j)
                        qr(k, j) = qr(k, j) - tau * tmp[j];
                    float tauEss[4];
                    for (int i = k + 1; i < n; ++i)
                        tauEss[i] = tau * qr(i, k);
                    for (int j = k + 1; j < n; ++j)
                        for (int i = k + 1; i < n; ++i)
                            qr(i, j) = qr(i, j) - tmp[j] * tauEss[i];
                }
            }
            // norm downdate (LAPACK xGEQP3 style)
            for (int j = k + 1; j < n; ++j) {
                if (normsUpd[j] != 0.0f) {
                    float temp = std::fabs(qr(k, j)) / normsUpd[j];
                    temp = (1.0f + temp) * (1.0f - temp);
                    temp = temp < 0.0f ? 0.0f : temp;
                    const float ratio = normsUpd[j] / normsDir[j];
                    const float temp2 = temp * (ratio * ratio);
                    if (temp2 <= downdateThreshold) {
                        float s = 0.0f;
                        if (n - k - 1 > 0) {
                            s = qr(k + 1, j) * qr(k + 1, j);
                            for (int i = k + 2; i < n; ++i)
                                s = s + qr(i, j) * qr(i, j);
                        }
                        normsDir[j] = std::sqrt(s);
                        normsUpd[j] = normsDir[j];
                    } else {
                        normsUpd[j] = normsUpd[j] * std::sqrt(temp);
                    }
                }
            }
        }
        int perm[4];
        for (int i = 0; i < n; ++i)
            perm[i] = i;
        for (int k = 0; k < n; ++k)
            std::swap(perm[k], perm[transp[k]]);
        if (nonzeroPivots == 0) {
            for (int i = 0; i < n; ++i)
                x[i] = 0.0f;
            return;
        }
        float c[4];
        for (int i = 0; i < n; ++i)
            c[i] = b[i];
        // apply Q^T = H_{p-1} ... H_0
        for (int k = 0; k < nonzeroPivots; ++k) {
            const int len = n - k;
            const float tau = hCoeffs[k];
            if (len == 1) {
                c[k] = c[k] * (1.0f - tau);
            } else if (tau != 0.0f) {
                float s = 0.0f;
                for (int i = k + 1; i < n; ++i)
                    s = s + qr(i, k) * c[i];
                s = s + c[k];
                c[k] = c[k] - tau * s;
                for (int i = k + 1; i < n; ++i)
                    c[i] = c[i] - s * (tau * qr(i, k));
            }
        }
        // upper-triangular back substitution, column-major order
        const int p = nonzeroPivots;
        for (int kk = 0; kk < p; ++kk) {
            const int i = p - kk - 1;
            if (c[i] != 0.0f) {
                c[i] = c[i] / qr(i, i);
                for (int s = 0; s < i; ++s)
                    c[s] = c[s] - c[i] * qr(s, i);
            }
        }
        for (int i = 0; i < n; ++i)
            x[i] = 0.0f;
        for (int i = 0; i < p; ++i)
            x[perm[i]] = c[i];
    }

    // ------------------------------------------------------------------------------------------
    // Geometry, core/Geometry.cpp:12-51 (2D), :53-109 (3D), :225-270 (buildMatrices)
    // ------------------------------------------------------------------------------------------
    struct Geom {
        int dim = 3;
        Mat P, Pinv, ext, K, R, S;
        float t[3] = {0, 0, 0};
        float C[3] = {0, 0, 0};
        float sdd = 0;
    };

    static void buildMatrices(Geom& g)
    {
        const int d = g.dim;
        Mat tmpRt = zeros(d + 1, d + 1);
        for (int i = 0; i < d; ++i) {
            for (int j = 0; j < d; ++j)
                tmpRt(i, j) = g.R(i, j);
            tmpRt(i, d) = g.t[i];
        }
        tmpRt(d, d) = 1.0f;
        Mat tmpId = identity(d, d + 1);
        Mat extFull = mul(tmpRt, g.S);
        g.ext = zeros(d, d + 1);
        for (int i = 0; i < d; ++i)
            for (int j = 0; j <= d; ++j)
                g.ext(i, j) = extFull(i, j);
        g.P = mul(mul(g.K, tmpId), extFull);
        // camera centre C = -(P(0:d,0:d)^-1 P(:,d)) by column-pivoting QR
        Mat P33 = zeros(d, d);
        float p4[3];
        for (int i = 0; i < d; ++i) {
            for (int j = 0; j < d; ++j)
                P33(i, j) = g.P(i, j);
            p4[i] = g.P(i, d);
        }
        float sol[3];
        colPivQrSolve(P33, p4, sol);
        for (int i = 0; i < d; ++i)
            g.C[i] = -sol[i];
        // Pinv = Sinv * Rtinv * tmpIdinv * Kinv
        Mat Sinv = zeros(d + 1, d + 1);
        for (int i = 0; i <= d; ++i)
            Sinv(i, i) = 1.0f / g.S(i, i);
        Mat Kinv = identity(d, d);
        Kinv(0, 0) = 1.0f / g.K(0, 0);
        Kinv(0, d - 1) = -g.K(0, d - 1) / g.K(0, 0);
        if (d == 3) {
            Kinv(1, 1) = 1.0f / g.K(1, 1);
            Kinv(1, d - 1) = -g.K(1, d - 1) / g.K(1, 1);
        }
        Mat Rtinv = zeros(d + 1, d + 1);
        for (int i = 0; i < d; ++i)
            for (int j = 0; j < d; ++j)
                Rtinv(i, j) = g.R(j, i);
        // -R^T * t (GEMV with the negation folded into alpha)
        for (int i = 0; i < d; ++i) {
            float s = 0.0f;
            for (int k = 0; k < d; ++k)
                s = s + g.R(k, i) * g.t[k];
            Rtinv(i, d) = -s;
        }
        Rtinv(d, d) = 1.0f;
        Mat tmpIdinv = identity(d + 1, d);
        g.Pinv = mul(mul(mul(Sinv, Rtinv), tmpIdinv), Kinv);
    }

    // Geometry.cpp:12-51
    static Geom geometry2d(float s2c, float c2d, float angle, const float* volSpacing,
                           const float* volOrigin, const float* sinoSpacing,
                           const float* sinoOrigin, float ppOffset, const float* corOffset)
    {
        Geom g;
        g.dim = 2;
        g.sdd = s2c + c2d;
        const float c = std::cos(angle);
        const float s = std::sin(angle);
        g.R = zeros(2, 2);
        g.R(0, 0) = c;
        g.R(0, 1) = -s;
        g.R(1, 0) = s;
        g.R(1, 1) = c;
        g.S = identity(3, 3);
        g.S(0, 0) = volSpacing[0];
        g.S(1, 1) = volSpacing[1];
        float v[2] = {-corOffset[0] - volOrigin[0], -corOffset[1] - volOrigin[1]};
        matvec(g.R, v, g.t);
        g.t[1] = g.t[1] + s2c;
        const float alpha = sinoSpacing[0];
        g.K = identity(2, 2);
        g.K(0, 0) = (s2c + c2d) / alpha;
        g.K(0, 1) = sinoOrigin[0] / alpha + ppOffset;
        buildMatrices(g);
        return g;
    }

    // Geometry.cpp:53-109 (YZY convention, angles gamma, beta, alpha)
    static Geom geometry3d(float s2c, float c2d, const float* volSpacing, const float* volOrigin,
                           const float* sinoSpacing, const float* sinoOrigin, float gamma,
                           float beta, float alpha, const float* ppOffset, const float* corOffset)
    {
        Geom g;
        g.dim = 3;
        g.sdd = s2c + c2d;
        const float ca = std::cos(alpha), sa = std::sin(alpha);
        const float cb = std::cos(beta), sb = std::sin(beta);
        const float cg = std::cos(gamma), sg = std::sin(gamma);
        Mat A = zeros(3, 3), B = zeros(3, 3), Cm = zeros(3, 3);
        A(0, 0) = cg; A(0, 1) = 0; A(0, 2) = sg;
        A(1, 0) = 0;  A(1, 1) = 1; A(1, 2) = 0;
        A(2, 0) = -sg; A(2, 1) = 0; A(2, 2) = cg;
        B(0, 0) = cb; B(0, 1) = -sb; B(0, 2) = 0;
        B(1, 0) = sb; B(1, 1) = cb; B(1, 2) = 0;
        B(2, 0) = 0;  B(2, 1) = 0;  B(2, 2) = 1;
        Cm(0, 0) = ca; Cm(0, 1) = 0; Cm(0, 2) = sa;
        Cm(1, 0) = 0;  Cm(1, 1) = 1; Cm(1, 2) = 0;
        Cm(2, 0) = -sa; Cm(2, 1) = 0; Cm(2, 2) = ca;
        g.R = mul(mul(A, B), Cm);
        g.S = identity(4, 4);
        for (int i = 0; i < 3; ++i)
            g.S(i, i) = volSpacing[i];
        float v[3] = {-corOffset[0] - volOrigin[0], -corOffset[1] - volOrigin[1],
                      -corOffset[2] - volOrigin[2]};
        matvec(g.R, v, g.t);
        g.t[2] = g.t[2] + s2c;
        const float a1 = sinoSpacing[0], a2 = sinoSpacing[1];
        g.K = identity(3, 3);
        g.K(0, 0) = (s2c + c2d) / a1;
        g.K(0, 2) = sinoOrigin[0] / a1 + ppOffset[0];
        g.K(1, 1) = (s2c + c2d) / a2;
        g.K(1, 2) = sinoOrigin[1] / a2 + ppOffset[1];
        buildMatrices(g);
        return g;
    }

    // Pose record exchanged with the tests (same layout as the product's C ABI):
    // P at 0 (d x d+1, row-major), Pinv at 12 (d+1 x d), C at 24, ext at 27 (d x d+1), sdd at 39.
    constexpr int POSE_FLOATS = 40;

    static void packPose(const Geom& g, float* out)
    {
        std::memset(out, 0, sizeof(float) * POSE_FLOATS);
        const int d = g.dim;
        for (int i = 0; i < d * (d + 1); ++i) {
            out[i] = g.P.a[i];
            out[12 + i] = g.Pinv.a[i];
            out[27 + i] = g.ext.a[i];
        }
        for (int i = 0; i < d; ++i)
            out[24 + i] = g.C[i];
        out[39] = g.sdd;
    }

    struct PoseView {
        int dim;
        const float* p;
        float P(int i, int j) const { return p[i * (dim + 1) + j]; }
        float Pinv(int i, int j) const { return p[12 + i * dim + j]; }
        float C(int i) const { return p[24 + i]; }
        float ext(int i, int j) const { return p[27 + i * (dim + 1) + j]; }
        float sdd() const { return p[39]; }
    };

    // ------------------------------------------------------------------------------------------
    // Rays: core/Descriptors/DetectorDescriptor.cpp:20-52,90-128
    // ------------------------------------------------------------------------------------------
    struct Ray {
        float o[3];
        float d[3];
    };

    static Ray rayFromDetector(const PoseView& pv, const float* detCoord)
    {
        const int d = pv.dim;
        float h[3] = {detCoord[0], d == 3 ? detCoord[1] : 1.0f, 1.0f};
        Ray r{};
        float dir[4];
        for (int i = 0; i <= d; ++i) {
            float s = 0.0f;
            for (int k = 0; k < d; ++k)
                s = s + pv.Pinv(i, k) * h[k];
            dir[i] = s;
        }
        const float z = seqSqNorm(dir, d);
        const float nrm = std::sqrt(z);
        for (int i = 0; i < d; ++i) {
            r.d[i] = z > 0.0f ? dir[i] / nrm : dir[i];
            r.o[i] = pv.C(i);
        }
        return r;
    }

    // coords (optional): a curved detector's planar coordinate per pixel (2 floats, u fastest),
    // used in place of the pixel centre (CurvedDetectorDescriptor.cpp:93-120)
    static Ray rayForIndex(const PoseView* poses, int dim, const index_t* detDims, index_t ir,
                           const float* coords = nullptr)
    {
        // detector coordinate from index, x (u) fastest, pose last
        float dc[2] = {0, 0};
        index_t pose;
        index_t pixel;
        if (dim == 2) {
            const index_t u = ir % detDims[0];
            pose = ir / detDims[0];
            pixel = u;
            dc[0] = static_cast<float>(u) + 0.5f;
        } else {
            const index_t u = ir % detDims[0];
            const index_t v = (ir / detDims[0]) % detDims[1];
            pose = ir / (detDims[0] * detDims[1]);
            pixel = u + detDims[0] * v;
            dc[0] = static_cast<float>(u) + 0.5f;
            dc[1] = static_cast<float>(v) + 0.5f;
        }
        if (coords) {
            dc[0] = coords[2 * pixel];
            if (dim == 3)
                dc[1] = coords[2 * pixel + 1];
        }
        return rayFromDetector(poses[pose], dc);
    }

    // CurvedDetectorDescriptor::setup / mapCurvedCoordToPlanarCoord
    // (core/Descriptors/CurvedDetectorDescriptor.cpp:33-91): planar coordinates of the pixel
    // centres, 2 floats per pixel (v' = 0 in 2D)
    static void curvedCoords(int dim, index_t nu, index_t nv, float angle, float s2d, float* out)
    {
        const index_t height = dim == 3 ? nv : 1;
        const float radius = static_cast<float>(nu) / angle;
        const float angleDelta = angle / static_cast<float>(nu);
        const float centre[2] = {static_cast<float>(nu) / 2.0f, static_cast<float>(height) / 2.0f};
        const float circle[2] = {centre[0], s2d - radius};
        for (index_t h = 0; h < height; ++h)
            for (index_t l = 0; l < nu; ++l) {
                const float coord0 = static_cast<float>(l) + 0.5f;
                const float coord1 = static_cast<float>(h) + 0.5f;
                const float rayAngle = (coord0 - centre[0]) * angleDelta;
                // the reference's unqualified sin / cos of a float: evaluated in double here
                const float deltaX =
                    static_cast<float>(std::sin(static_cast<double>(rayAngle))) * radius;
                const float deltaDepth =
                    static_cast<float>(std::cos(static_cast<double>(rayAngle))) * radius;
                const float onCurved[2] = {circle[0] + deltaX, circle[1] + deltaDepth};
                const float factor = onCurved[1] == 0 ? 1.0f : s2d / onCurved[1];
                float* o = out + 2 * (h * nu + l);
                o[0] = (onCurved[0] - centre[0]) * factor + centre[0];
                o[1] = dim == 3 ? (coord1 - centre[1]) * factor + centre[1] : 0.0f;
            }
    }

    // projectors/Intersection.h:179-198
    template <typename T1, typename T2>
    static T1 minNum(T1 x, T2 y)
    {
        return (y != y) ? x : (x < y ? x : static_cast<T1>(y));
    }
    template <typename T1, typename T2>
    static T1 maxNum(T1 x, T2 y)
    {
        return (y != y) ? x : (x > y ? x : static_cast<T1>(y));
    }

    // projectors/Intersection.cpp:7-46; box is [0, dims]
    static bool intersectRay(const float* boxMax, int dim, const Ray& r, float& tmin, float& tmax)
    {
        float invDir = 1 / r.d[0];
        float t1 = (0.0f - r.o[0]) * invDir;
        float t2 = (boxMax[0] - r.o[0]) * invDir;
        tmin = invDir >= 0 ? t1 : t2;
        tmax = invDir >= 0 ? t2 : t1;
        for (int i = 1; i < dim; ++i) {
            invDir = 1 / r.d[i];
            t1 = (0.0f - r.o[i]) * invDir;
            t2 = (boxMax[i] - r.o[i]) * invDir;
            tmin = maxNum(tmin, invDir >= 0 ? t1 : t2);
            tmax = minNum(tmax, invDir >= 0 ? t2 : t1);
        }
        if (tmax == 0.0f && tmin == 0.0f)
            return false;
        return tmax >= maxNum(tmin, 0.0f);
    }

    // ------------------------------------------------------------------------------------------
    // Joseph: projectors/DrivingDirectionTraversal.cpp:6-106 + JosephsMethod.cpp:37-198
    // ------------------------------------------------------------------------------------------
    struct DDTraversal {
        float pos[3], step[3];
        float length = 0;
        int driving = 0;
        index_t numSteps = 0;
    };

    static DDTraversal ddSetup(const float* boxMax, int dim, const Ray& r)
    {
        DDTraversal t;
        float tmin, tmax;
        const bool hit = intersectRay(boxMax, dim, r, tmin, tmax);
        // argmax |d| (first occurrence)
        int drv = 0;
        float best = std::fabs(r.d[0]);
        for (int i = 1; i < dim; ++i)
            if (std::fabs(r.d[i]) > best) {
                best = std::fabs(r.d[i]);
                drv = i;
            }
        t.driving = drv;
        if (!hit) {
            t.numSteps = 0;
            return t;
        }
        float exitp[3] = {0, 0, 0};
        for (int i = 0; i < dim; ++i) {
            t.pos[i] = r.o[i] + r.d[i] * tmin;
            exitp[i] = r.o[i] + r.d[i] * tmax;
            if (t.pos[i] < 0.0f)
                t.pos[i] = 0.0f;
            if (t.pos[i] > boxMax[i])
                t.pos[i] = boxMax[i];
            if (exitp[i] < 0.0f)
                exitp[i] = 0.0f;
            if (exitp[i] > boxMax[i])
                exitp[i] = boxMax[i];
        }
        const float absd = std::fabs(r.d[drv]);
        for (int i = 0; i < dim; ++i)
            t.step[i] = r.d[i] / absd;
        const float dist = t.pos[drv] - std::floor(t.pos[drv]);
        const float sgn = (t.step[drv] > 0.0f) ? 1.0f : ((t.step[drv] < 0.0f) ? -1.0f : 0.0f);
        const float shift = 0.5f - dist;
        for (int i = 0; i < dim; ++i)
            t.pos[i] = t.pos[i] + (t.step[i] * shift) * sgn;
        t.pos[drv] = std::floor(t.pos[drv]) + 0.5f;
        t.numSteps = static_cast<index_t>(std::ceil(std::fabs(exitp[drv] - t.pos[drv])));
        // fixed-size Eigen array norm: the unrolled reduction adds s0^2 + (s1^2 + s2^2)
        t.length = dim == 3 ? std::sqrt(t.step[0] * t.step[0]
                                        + (t.step[1] * t.step[1] + t.step[2] * t.step[2]))
                            : std::sqrt(t.step[0] * t.step[0] + t.step[1] * t.step[1]);
        return t;
    }

    // Visit the taps of one Joseph sample exactly as JosephsMethod.cpp:37-97 does: weights from
    // the position, masked (weight 0) and clipped taps, in the reference's tap order.
    template <class Fn>
    static void josephTaps(const float* pos, int drv, int dim, const index_t* volDims, Fn fn)
    {
        index_t fl[3], ce[3];
        float w[3], cw[3];
        for (int i = 0; i < dim; ++i) {
            const float p5 = pos[i] - 0.5f;
            fl[i] = static_cast<index_t>(std::floor(p5));
            ce[i] = static_cast<index_t>(std::ceil(p5));
            cw[i] = (pos[i] - static_cast<float>(fl[i])) - 0.5f;
            w[i] = 1.0f - cw[i];
        }
        w[drv] = 1.0f;
        cw[drv] = 1.0f;
        auto tap = [&](index_t i0, index_t i1, index_t i2, float w0, float w1, float w2) {
            index_t c[3] = {i0, i1, i2};
            bool in = true;
            for (int k = 0; k < dim; ++k)
                in = in && c[k] >= 0 && c[k] < volDims[k];
            for (int k = 0; k < dim; ++k)
                c[k] = std::max<index_t>(0, std::min<index_t>(c[k], volDims[k] - 1));
            float wt = static_cast<float>(in) * w0;
            wt = wt * w1;
            if (dim == 3)
                wt = wt * w2;
            const index_t idx =
                dim == 2 ? c[0] + c[1] * volDims[0] : c[0] + volDims[0] * (c[1] + volDims[1] * c[2]);
            fn(idx, wt);
        };
        if (dim == 2) {
            tap(fl[0], ce[1], 0, w[0], cw[1], 1.0f);
            tap(ce[0], fl[1], 0, cw[0], w[1], 1.0f);
        } else {
            tap(fl[0], fl[1], fl[2], w[0], w[1], w[2]);
            tap(fl[0], ce[1], ce[2], w[0], cw[1], cw[2]);
            tap(ce[0], fl[1], ce[2], cw[0], w[1], cw[2]);
            tap(ce[0], ce[1], fl[2], cw[0], cw[1], w[2]);
        }
    }

    // ------------------------------------------------------------------------------------------
    // Adjoint accumulation in a fixed order. The reference adds every contribution with
    // `omp atomic` (JosephsMethod.cpp:180-186, SiddonsMethod.cpp:119), so its float sums change
    // from run to run. Here the rays are split into `chunks` contiguous ranges, a number that
    // depends on the problem size only; one thread scatters each range, in ray order, into a
    // partial volume of its own, and the partial volumes are added in range order. The result is
    // the same for every thread count and every run.
    // ------------------------------------------------------------------------------------------
    // When set (oracle_set_adjoint_atomic), the adjoints add with `omp atomic` straight into the
    // output as the reference does: the reference's speed, not its order. Only the CPU-baseline
    // timing uses it; parity checks use the fixed order.
    static bool gAtomicAdjoint = false;

    template <typename data_t, class RayFn>
    static void orderedScatter(index_t nrays, index_t nvol, data_t* out, RayFn rayFn)
    {
        if (gAtomicAdjoint) {
            std::fill(out, out + nvol, data_t(0));
            auto add = [out](index_t idx, data_t v) {
#pragma omp atomic
                out[idx] += v;
            };
#pragma omp parallel for schedule(dynamic, 256)
            for (index_t ir = 0; ir < nrays; ++ir)
                rayFn(ir, add);
            return;
        }
        const index_t bytes = std::max<index_t>(1, nvol * static_cast<index_t>(sizeof(data_t)));
        index_t chunks = std::min<index_t>(32, std::max<index_t>(1, (index_t(1) << 31) / bytes));
        chunks = std::min<index_t>(chunks, std::max<index_t>(1, nrays));
        std::fill(out, out + nvol, data_t(0));
        std::vector<data_t> partial(static_cast<size_t>((chunks - 1) * nvol), data_t(0));
#pragma omp parallel for schedule(dynamic, 1)
        for (index_t c = 0; c < chunks; ++c) {
            data_t* dst = c == 0 ? out : partial.data() + (c - 1) * nvol;
            auto add = [dst](index_t idx, data_t v) { dst[idx] += v; };
            const index_t lo = nrays * c / chunks, hi = nrays * (c + 1) / chunks;
            for (index_t ir = lo; ir < hi; ++ir)
                rayFn(ir, add);
        }
        if (chunks > 1) {
#pragma omp parallel for schedule(static)
            for (index_t v = 0; v < nvol; ++v) {
                data_t s = out[v];
                for (index_t c = 1; c < chunks; ++c)
                    s += partial[static_cast<size_t>((c - 1) * nvol + v)];
                out[v] = s;
            }
        }
    }

    // mode 0: reference position update (pos += step each step, DrivingDirectionTraversal.cpp:265)
    // mode 1: pos_j = fma(j, step, pos_0) (one rounding; used to isolate the accumulation drift)
    template <typename data_t, bool adjoint>
    static void josephTraverse(int dim, const index_t* volDims, const index_t* detDims,
                               index_t numPoses, const float* poseData, const data_t* in,
                               data_t* out, int mode, const float* coords = nullptr)
    {
        std::vector<PoseView> poses(numPoses);
        for (index_t p = 0; p < numPoses; ++p)
            poses[p] = PoseView{dim, poseData + p * POSE_FLOATS};
        float boxMax[3] = {0, 0, 0};
        index_t nvol = 1;
        for (int i = 0; i < dim; ++i) {
            boxMax[i] = static_cast<float>(volDims[i]);
            nvol *= volDims[i];
        }
        const index_t nrays = (dim == 2 ? detDims[0] : detDims[0] * detDims[1]) * numPoses;
        // one ray; the adjoint adds through add(index, value) (orderedScatter)
        auto ray = [&](index_t ir, auto& add) {
            const Ray r = rayForIndex(poses.data(), dim, detDims, ir, coords);
            DDTraversal tr = ddSetup(boxMax, dim, r);
            const data_t L = static_cast<data_t>(tr.length);
            data_t acc = 0;
            float pos[3] = {tr.pos[0], tr.pos[1], tr.pos[2]};
            for (index_t s = 0; s < tr.numSteps; ++s) {
                if (mode == 1) {
                    for (int i = 0; i < dim; ++i)
                        pos[i] = std::fma(static_cast<float>(s), tr.step[i], tr.pos[i]);
                }
                if (adjoint) {
                    const data_t y = in[ir];
                    josephTaps(pos, tr.driving, dim, volDims, [&](index_t idx, float wt) {
                        add(idx, y * L * static_cast<data_t>(wt));
                    });
                } else {
                    josephTaps(pos, tr.driving, dim, volDims, [&](index_t idx, float wt) {
                        acc += in[idx] * L * static_cast<data_t>(wt);
                    });
                }
                if (mode == 0)
                    for (int i = 0; i < dim; ++i)
                        pos[i] = pos[i] + tr.step[i];
            }
            if (!adjoint)
                out[ir] = acc;
        };
        if (adjoint) {
            orderedScatter<data_t>(nrays, nvol, out, ray);
            return;
        }
        auto none = [](index_t, data_t) {};
#pragma omp parallel for schedule(dynamic, 256)
        for (index_t ir = 0; ir < nrays; ++ir)
            ray(ir, none);
    }

    // ------------------------------------------------------------------------------------------
    // Siddon: projectors/TraverseAABB.cpp:6-184 + SiddonsMethod.cpp:76-124
    // ------------------------------------------------------------------------------------------
    // visits (optional): per-ray number of visited voxels. binary: BinaryMethod
    // (projectors/BinaryMethod.cpp:66-111), the same TraverseAABB visits with weight 1.
    template <typename data_t, bool adjoint>
    static void siddonTraverse(int dim, const index_t* volDims, const index_t* detDims,
                               index_t numPoses, const float* poseData, const data_t* in,
                               data_t* out, index_t* visits = nullptr, bool binary = false,
                               const float* coords = nullptr)
    {
        std::vector<PoseView> poses(numPoses);
        for (index_t p = 0; p < numPoses; ++p)
            poses[p] = PoseView{dim, poseData + p * POSE_FLOATS};
        float boxMax[3] = {0, 0, 0};
        index_t nvol = 1;
        index_t strides[3] = {1, volDims[0], dim == 3 ? volDims[0] * volDims[1] : 0};
        for (int i = 0; i < dim; ++i) {
            boxMax[i] = static_cast<float>(volDims[i]);
            nvol *= volDims[i];
        }
        const index_t nrays = (dim == 2 ? detDims[0] : detDims[0] * detDims[1]) * numPoses;
        const float EPS = std::numeric_limits<float>::epsilon();
        const float MAXF = std::numeric_limits<float>::max();
        // one ray; the adjoint adds through add(index, value) (orderedScatter)
        auto ray = [&](index_t ir, auto& add) {
            const Ray r = rayForIndex(poses.data(), dim, detDims, ir, coords);
            data_t acc = 0;
            float tmin, tmax;
            bool inBox = intersectRay(boxMax, dim, r, tmin, tmax);
            if (inBox) {
                float entry[3], cur[3], T[3], tDelta[3];
                int stepDir[3];
                for (int i = 0; i < dim; ++i) {
                    entry[i] = r.o[i] + r.d[i] * tmin;
                    if (entry[i] < 0.0f)
                        entry[i] = 0.0f;
                    if (entry[i] > boxMax[i])
                        entry[i] = boxMax[i];
                }
                for (int i = 0; i < dim; ++i)
                    stepDir[i] = (r.d[i] > 0.0f) ? 1 : ((r.d[i] < 0.0f) ? -1 : 0);
                for (int i = 0; i < dim; ++i) {
                    float lc = std::floor(entry[i]);
                    if (lc == entry[i] && stepDir[i] < 0)
                        lc = lc - 1.0f;
                    cur[i] = lc;
                }
                for (int i = 0; i < dim; ++i)
                    if (cur[i] >= boxMax[i] || cur[i] < 0.0f)
                        inBox = false;
                if (inBox) {
                    for (int i = 0; i < dim; ++i) {
                        const float td = static_cast<float>(stepDir[i]) / r.d[i];
                        tDelta[i] = std::fabs(r.d[i]) > EPS ? td : MAXF;
                        const float tt =
                            ((r.d[i] > 0.0f ? cur[i] + 1.0f : cur[i]) - entry[i]) / r.d[i];
                        T[i] = std::fabs(r.d[i]) > EPS ? tt : MAXF;
                    }
                    index_t idx = 0;
                    for (int i = 0; i < dim; ++i)
                        idx += strides[i] * static_cast<index_t>(cur[i]);
                    float tExit = 0.0f;
                    while (inBox) {
                        const float tEntry = tExit;
                        float tm = T[0];
                        for (int i = 1; i < dim; ++i)
                            tm = (T[i] < tm) ? T[i] : tm;
                        tExit = tm;
                        bool mask[3];
                        for (int i = 0; i < dim; ++i) {
                            bool m = true;
                            for (int j = 0; j < dim; ++j)
                                if (j != i)
                                    m = m && (T[i] <= T[j]);
                            mask[i] = m;
                        }
                        for (int i = 0; i < dim; ++i) {
                            if (mask[i]) {
                                cur[i] = cur[i] + static_cast<float>(stepDir[i]);
                                T[i] = T[i] + tDelta[i];
                            }
                        }
                        for (int i = 0; i < dim; ++i)
                            if (!(cur[i] < boxMax[i] && cur[i] >= 0.0f))
                                inBox = false;
                        const float weight = tExit - tEntry;
                        if (visits)
                            ++visits[ir];
                        if (binary) {
                            if (adjoint) {
                                add(idx, in[ir]);
                            } else {
                                acc += in[idx];
                            }
                        } else if (adjoint) {
                            add(idx, in[ir] * static_cast<data_t>(weight));
                        } else {
                            acc += in[idx] * static_cast<data_t>(weight);
                        }
                        for (int i = 0; i < dim; ++i)
                            if (mask[i])
                                idx += stepDir[i] * strides[i];
                    }
                }
            }
            if (!adjoint)
                out[ir] = acc;
        };
        if (adjoint) {
            orderedScatter<data_t>(nrays, nvol, out, ray);
            return;
        }
        auto none = [](index_t, data_t) {};
#pragma omp parallel for schedule(dynamic, 256)
        for (index_t ir = 0; ir < nrays; ++ir)
            ray(ir, none);
    }

    // ------------------------------------------------------------------------------------------
    // Ray-driven blob / B-spline projector: projectors/LutProjector.h:85-163 with
    // SliceTraversal.cpp:7-200 (traversal coordinates: the leading axis of the ray rotated onto
    // +x about the box centre), Intersection.cpp:47-119 (intersectXPlanes) and
    // core/Utilities/CartesianIndices.cpp:341-356 (neighbours_in_slice, last axis fastest).
    // ------------------------------------------------------------------------------------------
    struct SliceWalk {
        bool hit = false;
        float start[3] = {0, 0, 0}; // ray.pointAt(t) of the first slice, original coordinates
        float step[3] = {0, 0, 0};  // direction * tDelta
        index_t count = 0;          // endIndex
        int lead = 0;
    };

    // rotation of TransformToTraversal::create2DRotation / create3DRotation
    static void traversalRotation(int dim, int lead, float coeff, float R[3][3])
    {
        const float pi = static_cast<float>(3.14159265358979323846);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                R[i][j] = i == j ? 1.0f : 0.0f;
        if (dim == 2) {
            float rad = 0.0f;
            if (lead == 0 && coeff >= 0)
                rad = 0.0f;
            else if (lead == 0 && coeff < 0)
                rad = pi;
            else if (lead == 1 && coeff >= 0)
                rad = 3 * pi / 2;
            else if (lead == 1 && coeff <= 0)
                rad = pi / 2;
            const float c = std::cos(rad), sn = std::sin(rad);
            R[0][0] = c, R[0][1] = -sn, R[1][0] = sn, R[1][1] = c;
            return;
        }
        auto rotY = [&](float rad) {
            const float c = std::cos(rad), sn = std::sin(rad);
            R[0][0] = c, R[0][1] = 0, R[0][2] = sn;
            R[1][0] = 0, R[1][1] = 1, R[1][2] = 0;
            R[2][0] = -sn, R[2][1] = 0, R[2][2] = c;
        };
        auto rotZ = [&](float rad) {
            const float c = std::cos(rad), sn = std::sin(rad);
            R[0][0] = c, R[0][1] = -sn, R[0][2] = 0;
            R[1][0] = sn, R[1][1] = c, R[1][2] = 0;
            R[2][0] = 0, R[2][1] = 0, R[2][2] = 1;
        };
        const float half = static_cast<float>(0.5 * static_cast<double>(pi));
        if (lead == 0 && coeff >= 0)
            return;
        else if (lead == 0 && coeff < 0)
            rotY(pi);
        else if (lead == 1 && coeff >= 0)
            rotZ(-half);
        else if (lead == 1 && coeff <= 0)
            rotZ(half);
        else if (lead == 2 && coeff >= 0)
            rotY(half);
        else if (lead == 2 && coeff <= 0)
            rotY(-half);
    }

    // SliceTraversal(aabb, ray) for the box [bmin, bmax]
    static SliceWalk sliceWalk(int dim, const float* bmin, const float* bmax, const Ray& r)
    {
        SliceWalk w;
        int lead = 0;
        float best = std::fabs(r.d[0]);
        for (int i = 1; i < dim; ++i)
            if (std::fabs(r.d[i]) > best) {
                best = std::fabs(r.d[i]);
                lead = i;
            }
        w.lead = lead;
        float R[3][3];
        traversalRotation(dim, lead, r.d[lead], R);
        // T = rotation * translation(-centre): columns 0..dim-1 are R, column dim is R (-centre)
        float centre[3] = {0, 0, 0}, tcol[3] = {0, 0, 0};
        for (int i = 0; i < dim; ++i)
            centre[i] = bmax[i] / 2;
        for (int i = 0; i < dim; ++i) {
            float acc = 0.0f;
            for (int k = 0; k < dim; ++k)
                acc = acc + R[i][k] * (-centre[k]);
            tcol[i] = acc + 0.0f;
        }
        auto point = [&](const float* p, float* out) {
            for (int i = 0; i < dim; ++i) {
                float acc = 0.0f;
                for (int k = 0; k < dim; ++k)
                    acc = acc + R[i][k] * p[k];
                out[i] = acc + tcol[i];
            }
        };
        float o[3], d[3], lo[3], hi[3];
        point(r.o, o);
        for (int i = 0; i < dim; ++i) {
            float acc = 0.0f;
            for (int k = 0; k < dim; ++k)
                acc = acc + R[i][k] * r.d[k];
            d[i] = acc;
        }
        point(bmin, lo);
        point(bmax, hi);
        for (int i = 0; i < dim; ++i)
            if (lo[i] > hi[i])
                std::swap(lo[i], hi[i]);
        // intersectXPlanes
        lo[0] += 0.5f;
        hi[0] -= 0.5f;
        float invDir = 1 / d[0];
        float t1 = (lo[0] - o[0]) * invDir, t2 = (hi[0] - o[0]) * invDir;
        float tmin = invDir >= 0 ? t1 : t2, tmax = invDir >= 0 ? t2 : t1;
        const float txmin = tmin, txmax = tmax;
        for (int i = 1; i < dim; ++i) {
            invDir = 1 / d[i];
            t1 = (lo[i] - o[i]) * invDir;
            t2 = (hi[i] - o[i]) * invDir;
            tmin = maxNum(tmin, invDir >= 0 ? t1 : t2);
            tmax = minNum(tmax, invDir >= 0 ? t2 : t1);
        }
        const float xcentre = std::fabs(lo[0] - static_cast<float>(static_cast<int>(std::round(lo[0]))));
        auto fractional = [](float v) {
            float trash = 0;
            return std::modf(v, &trash);
        };
        if (txmin < tmin) {
            const float e = o[0] + tmin * d[0];
            const float tmp = std::fabs(fractional(e - xcentre));
            const float frac = e < xcentre ? tmp : 1 - tmp;
            tmin += (tmp > 0.00001 && frac > 0.00001) ? frac / d[0] : 0;
        }
        if (txmax > tmax) {
            const float e = o[0] + tmax * d[0];
            const float tmp = std::fabs(fractional(e - xcentre));
            const float frac = e < xcentre ? 1 - tmp : tmp;
            tmax -= (tmp > 0.00001 && frac > 0.00001) ? frac / d[0] : 0;
        }
        if (tmax == 0.0 && tmin == 0.0)
            return w;
        if (!(tmax - maxNum(tmin, 0.0f) > -0.000001))
            return w;
        const float first = o[0] + tmin * d[0], last = o[0] + tmax * d[0];
        w.count = std::max<index_t>(1, static_cast<index_t>(std::ceil(last - first + 0.5f)));
        const float tDelta = 1 / d[0];
        for (int i = 0; i < dim; ++i) {
            w.start[i] = r.o[i] + tmin * r.d[i];
            w.step[i] = r.d[i] * tDelta;
        }
        w.hit = true;
        return w;
    }

    // Visit the neighbourhood of every slice voxel: f(linear index, weight). backward: the walk
    // uses the box grown by `support` in the non-leading axes (LutProjector.h:135-147).
    template <class F>
    static void lutRay(int dim, const index_t* volDims, const Ray& r, const float* lut,
                       index_t lutN, float radius, int support, bool backward, F&& f)
    {
        float bmin[3] = {0, 0, 0}, bmax[3] = {0, 0, 0};
        for (int i = 0; i < dim; ++i)
            bmax[i] = static_cast<float>(volDims[i]);
        int lead = 0;
        {
            float best = std::fabs(r.d[0]);
            for (int i = 1; i < dim; ++i)
                if (std::fabs(r.d[i]) > best) {
                    best = std::fabs(r.d[i]);
                    lead = i;
                }
        }
        float wmin[3], wmax[3];
        for (int i = 0; i < dim; ++i) {
            wmin[i] = bmin[i], wmax[i] = bmax[i];
            if (backward && i != lead) {
                wmin[i] -= static_cast<float>(support);
                wmax[i] += static_cast<float>(support);
            }
        }
        const SliceWalk w = sliceWalk(dim, wmin, wmax, r);
        if (!w.hit)
            return;
        float cur[3] = {w.start[0], w.start[1], w.start[2]};
        for (index_t it = 0; it < w.count; ++it) {
            index_t from[3] = {0, 0, 0}, to[3] = {1, 1, 1};
            for (int i = 0; i < dim; ++i) {
                const index_t pos = static_cast<index_t>(cur[i]);
                const index_t dist = i == lead ? 0 : support;
                from[i] = std::max<index_t>(pos - dist, 0);
                to[i] = std::min<index_t>(pos + dist + 1, volDims[i]);
                if (to[i] == from[i])
                    from[i] -= 1;
            }
            for (index_t a = from[0]; a < to[0]; ++a)
                for (index_t b = from[1]; b < to[1]; ++b)
                    for (index_t c = from[2]; c < (dim == 3 ? to[2] : from[2] + 1); ++c) {
                        const index_t nb[3] = {a, b, c};
                        float diff[3], dot = 0.0f;
                        for (int i = 0; i < dim; ++i)
                            diff[i] = (static_cast<float>(nb[i]) + 0.5f) - r.o[i];
                        for (int i = 0; i < dim; ++i)
                            dot = dot + r.d[i] * diff[i];
                        float sq = 0.0f;
                        for (int i = 0; i < dim; ++i) {
                            const float v = diff[i] - dot * r.d[i];
                            sq = sq + v * v;
                        }
                        const float distance = std::sqrt(sq);
                        const float wt = vox::lutLerp(lut, lutN, radius, distance);
                        const index_t idx = a + volDims[0] * (b + (dim == 3 ? volDims[1] * c : 0));
                        if (a >= 0 && b >= 0 && c >= 0)
                            f(idx, wt);
                    }
            for (int i = 0; i < dim; ++i)
                cur[i] = cur[i] + w.step[i];
        }
    }

    template <typename data_t, bool adjoint>
    static void lutTraverse(int dim, const index_t* volDims, const index_t* detDims,
                            index_t numPoses, const float* poseData, const float* lut,
                            index_t lutN, float radius, int support, const data_t* in,
                            data_t* out)
    {
        std::vector<PoseView> poses(numPoses);
        for (index_t p = 0; p < numPoses; ++p)
            poses[p] = PoseView{dim, poseData + p * POSE_FLOATS};
        index_t nvol = 1;
        for (int i = 0; i < dim; ++i)
            nvol *= volDims[i];
        const index_t nrays = (dim == 2 ? detDims[0] : detDims[0] * detDims[1]) * numPoses;
        // one ray; the adjoint adds through add(index, value) (orderedScatter)
        auto ray = [&](index_t ir, auto& add) {
            const Ray r = rayForIndex(poses.data(), dim, detDims, ir);
            if (adjoint) {
                const data_t y = in[ir];
                lutRay(dim, volDims, r, lut, lutN, radius, support, true,
                       [&](index_t idx, float wt) {
                           if (idx < 0 || idx >= nvol)
                               return;
                           add(idx, static_cast<data_t>(wt) * y);
                       });
            } else {
                data_t acc = 0;
                lutRay(dim, volDims, r, lut, lutN, radius, support, false,
                       [&](index_t idx, float wt) {
                           if (idx < 0 || idx >= nvol)
                               return;
                           acc += static_cast<data_t>(wt) * in[idx];
                       });
                out[ir] = acc;
            }
        };
        if (adjoint) {
            orderedScatter<data_t>(nrays, nvol, out, ray);
            return;
        }
        auto none = [](index_t, data_t) {};
#pragma omp parallel for schedule(dynamic, 64)
        for (index_t ir = 0; ir < nrays; ++ir)
            ray(ir, none);
    }

    // ------------------------------------------------------------------------------------------
    // Vector operations (storage/reductions/DotProduct.h:24-47, L2.h:15-49,
    // transforms/Lincomb.h:28-33): reductions accumulate in data_t, in 64 fixed blocks combined
    // sequentially (a deterministic stand-in for Thrust's blocked reduction).
    // ------------------------------------------------------------------------------------------
    template <typename data_t>
    static data_t blockedDot(const data_t* a, const data_t* b, index_t n)
    {
        const int NB = 64;
        data_t part[NB];
#pragma omp parallel for
        for (int blk = 0; blk < NB; ++blk) {
            const index_t lo = n * blk / NB, hi = n * (blk + 1) / NB;
            data_t s = 0;
            for (index_t i = lo; i < hi; ++i)
                s += a[i] * b[i];
            part[blk] = s;
        }
        data_t s = 0;
        for (int blk = 0; blk < NB; ++blk)
            s += part[blk];
        return s;
    }

} // namespace orc

// ----------------------------------------------------------------------------------------------
// C ABI for the Python test harness (ctypes)
// ----------------------------------------------------------------------------------------------
using orc::index_t;

extern "C" {

int oracle_num_threads(void)
{
    return omp_get_max_threads();
}

void oracle_set_adjoint_atomic(int on)
{
    orc::gAtomicAdjoint = on != 0;
}

void oracle_set_num_threads(int n)
{
    omp_set_num_threads(n);
}

// Single 2D pose (Geometry.cpp:12-51) packed into a 40-float pose record.
void oracle_geometry2d(float s2c, float c2d, float angleRad, const float* volSpacing,
                       const float* volOrigin, const float* sinoSpacing, const float* sinoOrigin,
                       float ppOffset, const float* corOffset, float* out)
{
    orc::packPose(orc::geometry2d(s2c, c2d, angleRad, volSpacing, volOrigin, sinoSpacing,
                                  sinoOrigin, ppOffset, corOffset),
                  out);
}

// Single 3D pose (Geometry.cpp:53-109).
void oracle_geometry3d(float s2c, float c2d, const float* volSpacing, const float* volOrigin,
                       const float* sinoSpacing, const float* sinoOrigin, float gamma, float beta,
                       float alpha, const float* ppOffset, const float* corOffset, float* out)
{
    orc::packPose(orc::geometry3d(s2c, c2d, volSpacing, volOrigin, sinoSpacing, sinoOrigin, gamma,
                                  beta, alpha, ppOffset, corOffset),
                  out);
}

// Circular trajectory: generators/CircleTrajectoryGenerator.cpp:9-24,
// BaseCircleTrajectoryGenerator.cpp:12-74, TrajectoryGenerator.cpp:9-47.
// volDims/volSpacing: dim entries; detSize: dim-1 entries (or NULL -> floor(N*sqrt(2)));
// detSpacing: dim-1 entries (or NULL -> volume spacing). Writes numPoses pose records and the
// detector coefficient counts (dim entries, last = numPoses).
void oracle_circle_trajectory(int dim, const int64_t* volDims, const float* volSpacing,
                              int64_t numPoses, float arcDegrees, float s2c, float c2d,
                              const int64_t* detSize, const float* detSpacing, float* outPoses,
                              int64_t* outDetDims)
{
    float volOrigin[3], spacing[3], coeffsF[3];
    int64_t coeffs[3];
    for (int i = 0; i < dim; ++i)
        volOrigin[i] = 0.5f * (static_cast<float>(volDims[i]) * volSpacing[i]);
    if (detSize) {
        for (int i = 0; i < dim - 1; ++i)
            coeffs[i] = detSize[i];
    } else {
        const float sqrt2 = std::sqrt(2.f);
        for (int i = 0; i < dim - 1; ++i)
            coeffs[i] = static_cast<int64_t>(static_cast<float>(volDims[i]) * sqrt2);
    }
    coeffs[dim - 1] = numPoses;
    for (int i = 0; i < dim - 1; ++i)
        spacing[i] = detSpacing ? detSpacing[i] : volSpacing[i];
    spacing[dim - 1] = 1.0f;
    for (int i = 0; i < dim; ++i) {
        coeffsF[i] = static_cast<float>(coeffs[i]);
        outDetDims[i] = coeffs[i];
    }
    float sinoOrigin[3];
    for (int i = 0; i < dim; ++i)
        sinoOrigin[i] = 0.5f * (coeffsF[i] * spacing[i]);
    // Eigen LinSpaced(n, 0, arc) for float: low + i*step, last = high
    const float arc = static_cast<float>(arcDegrees);
    const float stepDeg = numPoses == 1 ? 0.0f : (arc - 0.0f) / static_cast<float>(numPoses - 1);
    const float zero3[3] = {0, 0, 0};
    for (int64_t p = 0; p < numPoses; ++p) {
        float deg = (p == numPoses - 1) ? arc : 0.0f + static_cast<float>(p) * stepDeg;
        if (numPoses == 1)
            deg = arc;
        const float rad = deg * orc::pi_f() / 180;
        float* out = outPoses + p * orc::POSE_FLOATS;
        if (dim == 2)
            orc::packPose(orc::geometry2d(s2c, c2d, rad, volSpacing, volOrigin, spacing,
                                          sinoOrigin, 0.0f, zero3),
                          out);
        else
            orc::packPose(orc::geometry3d(s2c, c2d, volSpacing, volOrigin, spacing, sinoOrigin,
                                          rad, 0.0f, 0.0f, zero3, zero3),
                          out);
    }
}

// Ray for one detector index: writes origin (dim) and direction (dim).
void oracle_ray(int dim, const int64_t* detDims, const float* poses, int64_t ir, float* origin,
                float* direction)
{
    std::vector<orc::PoseView> pv(detDims[dim - 1]);
    for (int64_t p = 0; p < detDims[dim - 1]; ++p)
        pv[p] = orc::PoseView{dim, poses + p * orc::POSE_FLOATS};
    const orc::Ray r = orc::rayForIndex(pv.data(), dim, detDims, ir);
    for (int i = 0; i < dim; ++i) {
        origin[i] = r.o[i];
        direction[i] = r.d[i];
    }
}

// Driving-direction traversal setup for one ray: pos (dim), step (dim), length, driving axis,
// number of steps.
void oracle_dd_setup(int dim, const int64_t* volDims, const float* origin, const float* direction,
                     float* pos, float* step, float* length, int* driving, int64_t* numSteps)
{
    float boxMax[3] = {0, 0, 0};
    for (int i = 0; i < dim; ++i)
        boxMax[i] = static_cast<float>(volDims[i]);
    orc::Ray r{};
    for (int i = 0; i < dim; ++i) {
        r.o[i] = origin[i];
        r.d[i] = direction[i];
    }
    const orc::DDTraversal t = orc::ddSetup(boxMax, dim, r);
    for (int i = 0; i < dim; ++i) {
        pos[i] = t.pos[i];
        step[i] = t.step[i];
    }
    *length = t.length;
    *driving = t.driving;
    *numSteps = t.numSteps;
}

void oracle_joseph_f32(int adjoint, int dim, const int64_t* volDims, const int64_t* detDims,
                       const float* poses, const float* in, float* out, int mode, const float* coords)
{
    const int64_t np = detDims[dim - 1];
    if (adjoint)
        orc::josephTraverse<float, true>(dim, volDims, detDims, np, poses, in, out, mode, coords);
    else
        orc::josephTraverse<float, false>(dim, volDims, detDims, np, poses, in, out, mode, coords);
}

void oracle_joseph_f64(int adjoint, int dim, const int64_t* volDims, const int64_t* detDims,
                       const float* poses, const double* in, double* out, int mode, const float* coords)
{
    const int64_t np = detDims[dim - 1];
    if (adjoint)
        orc::josephTraverse<double, true>(dim, volDims, detDims, np, poses, in, out, mode, coords);
    else
        orc::josephTraverse<double, false>(dim, volDims, detDims, np, poses, in, out, mode, coords);
}

void oracle_siddon_f32(int adjoint, int dim, const int64_t* volDims, const int64_t* detDims,
                       const float* poses, const float* in, float* out, const float* coords)
{
    const int64_t np = detDims[dim - 1];
    if (adjoint)
        orc::siddonTraverse<float, true>(dim, volDims, detDims, np, poses, in, out, nullptr, false, coords);
    else
        orc::siddonTraverse<float, false>(dim, volDims, detDims, np, poses, in, out, nullptr, false, coords);
}

void oracle_siddon_f64(int adjoint, int dim, const int64_t* volDims, const int64_t* detDims,
                       const float* poses, const double* in, double* out, const float* coords)
{
    const int64_t np = detDims[dim - 1];
    if (adjoint)
        orc::siddonTraverse<double, true>(dim, volDims, detDims, np, poses, in, out, nullptr, false, coords);
    else
        orc::siddonTraverse<double, false>(dim, volDims, detDims, np, poses, in, out, nullptr, false, coords);
}

void oracle_binary_f32(int adjoint, int dim, const int64_t* volDims, const int64_t* detDims,
                       const float* poses, const float* in, float* out, const float* coords)
{
    const int64_t np = detDims[dim - 1];
    if (adjoint)
        orc::siddonTraverse<float, true>(dim, volDims, detDims, np, poses, in, out, nullptr, true, coords);
    else
        orc::siddonTraverse<float, false>(dim, volDims, detDims, np, poses, in, out, nullptr,
                                          true, coords);
}

void oracle_binary_f64(int adjoint, int dim, const int64_t* volDims, const int64_t* detDims,
                       const float* poses, const double* in, double* out, const float* coords)
{
    const int64_t np = detDims[dim - 1];
    if (adjoint)
        orc::siddonTraverse<double, true>(dim, volDims, detDims, np, poses, in, out, nullptr,
                                          true, coords);
    else
        orc::siddonTraverse<double, false>(dim, volDims, detDims, np, poses, in, out, nullptr,
                                           true, coords);
}

void oracle_lut_f32(int adjoint, int dim, const int64_t* volDims, const int64_t* detDims,
                    const float* poses, const float* lut, int64_t lutN, float radius, int support,
                    const float* in, float* out)
{
    const int64_t np = detDims[dim - 1];
    if (adjoint)
        orc::lutTraverse<float, true>(dim, volDims, detDims, np, poses, lut, lutN, radius,
                                      support, in, out);
    else
        orc::lutTraverse<float, false>(dim, volDims, detDims, np, poses, lut, lutN, radius,
                                       support, in, out);
}

void oracle_lut_f64(int adjoint, int dim, const int64_t* volDims, const int64_t* detDims,
                    const float* poses, const float* lut, int64_t lutN, float radius, int support,
                    const double* in, double* out)
{
    const int64_t np = detDims[dim - 1];
    if (adjoint)
        orc::lutTraverse<double, true>(dim, volDims, detDims, np, poses, lut, lutN, radius,
                                       support, in, out);
    else
        orc::lutTraverse<double, false>(dim, volDims, detDims, np, poses, lut, lutN, radius,
                                        support, in, out);
}

void oracle_curved_coords(int dim, int64_t nu, int64_t nv, float angle, float s2d, float* out)
{
    orc::curvedCoords(dim, nu, nv, angle, s2d, out);
}

// Number of Joseph samples (sum over rays of numSteps) and Siddon voxel crossings, used for the
// algorithmic-bytes figure of the roofline.
int64_t oracle_joseph_sample_count(int dim, const int64_t* volDims, const int64_t* detDims,
                                   const float* poseData)
{
    const int64_t np = detDims[dim - 1];
    std::vector<orc::PoseView> poses(np);
    for (int64_t p = 0; p < np; ++p)
        poses[p] = orc::PoseView{dim, poseData + p * orc::POSE_FLOATS};
    float boxMax[3] = {0, 0, 0};
    for (int i = 0; i < dim; ++i)
        boxMax[i] = static_cast<float>(volDims[i]);
    const int64_t nrays = (dim == 2 ? detDims[0] : detDims[0] * detDims[1]) * np;
    int64_t total = 0;
#pragma omp parallel for reduction(+ : total)
    for (int64_t ir = 0; ir < nrays; ++ir) {
        const orc::Ray r = orc::rayForIndex(poses.data(), dim, detDims, ir);
        total += orc::ddSetup(boxMax, dim, r).numSteps;
    }
    return total;
}

int64_t oracle_siddon_visit_count(int dim, const int64_t* volDims, const int64_t* detDims,
                                  const float* poseData)
{
    const int64_t np = detDims[dim - 1];
    const int64_t nrays = (dim == 2 ? detDims[0] : detDims[0] * detDims[1]) * np;
    int64_t nvol = 1;
    for (int i = 0; i < dim; ++i)
        nvol *= volDims[i];
    std::vector<float> x(static_cast<size_t>(nvol), 0.0f), y(static_cast<size_t>(nrays));
    std::vector<int64_t> visits(static_cast<size_t>(nrays), 0);
    orc::siddonTraverse<float, false>(dim, volDims, detDims, np, poseData, x.data(), y.data(),
                                      visits.data());
    int64_t total = 0;
    for (int64_t v : visits)
        total += v;
    return total;
}

double oracle_dot_f32(const float* a, const float* b, int64_t n)
{
    return static_cast<double>(orc::blockedDot(a, b, n));
}

double oracle_dot_f64(const double* a, const double* b, int64_t n)
{
    return orc::blockedDot(a, b, n);
}

} // extern "C"
