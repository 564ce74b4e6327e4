// Host-side projection geometry, see geometry.hpp.
//
// Reference: core/Geometry.cpp:12-51 (2D ctor), :53-109 (3D ctor), :225-270 (buildMatrices);
// generators/CircleTrajectoryGenerator.cpp:9-24, BaseCircleTrajectoryGenerator.cpp:12-74,
// TrajectoryGenerator.cpp:9-47. Evaluation order mirrors Eigen 3.4's coefficient-based products
// for tiny dynamic matrices (sequential k-sum, multiply then add, never fused); this file must be
// compiled without floating-point contraction (-ffp-contract=off).
#include "geometry.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <utility>

namespace elsa_b200
{
    namespace
    {
        // Row-major matrix up to 4x4.
        struct M4 {
            int rows = 0, cols = 0;
            float e[4][4] = {};
            M4() = default;
            M4(int r, int c, bool eye = false) : rows(r), cols(c)
            {
                if (eye)
                    for (int i = 0; i < r && i < c; ++i)
                        e[i][i] = 1.0f;
            }
        };

        M4 prod(const M4& a, const M4& b)
        {
            M4 out(a.rows, b.cols);
            for (int i = 0; i < a.rows; ++i)
                for (int j = 0; j < b.cols; ++j) {
                    float acc = a.e[i][0] * b.e[0][j];
                    for (int k = 1; k < a.cols; ++k)
                        acc = acc + a.e[i][k] * b.e[k][j];
                    out.e[i][j] = acc;
                }
            return out;
        }

        float sumSquares(const float* v, int n)
        {
            float acc = v[0] * v[0];
            for (int i = 1; i < n; ++i)
                acc = acc + v[i] * v[i];
            return acc;
        }

        // Solve A x = b (n <= 3) with column-pivoting Householder QR in float, the algorithm of
        // Eigen's ColPivHouseholderQR (LAPACK xGEQP3 with the norm-downdate safeguard).
        void solveColPivQr(M4 a, const float* b, float* x)
        {
            const int n = a.rows;
            float tau[4] = {}, nrmU[4] = {}, nrmD[4] = {};
            int swapWith[4] = {};
            for (int j = 0; j < n; ++j) {
                float col[4];
                for (int i = 0; i < n; ++i)
                    col[i] = a.e[i][j];
                nrmD[j] = nrmU[j] = std::sqrt(sumSquares(col, n));
            }
            const float eps = std::numeric_limits<float>::epsilon();
            float biggest = nrmU[0];
            for (int j = 1; j < n; ++j)
                biggest = nrmU[j] > biggest ? nrmU[j] : biggest;
            const float thr = (biggest * eps) * (biggest * eps) / float(n);
            const float downdateThr = std::sqrt(eps);
            int rank = n;
            for (int k = 0; k < n; ++k) {
                int piv = k;
                for (int j = k + 1; j < n; ++j)
                    if (nrmU[j] > nrmU[piv])
                        piv = j;
                if (rank == n && nrmU[piv] * nrmU[piv] < thr * float(n - k))
                    rank = k;
                swapWith[k] = piv;
                if (piv != k) {
                    for (int i = 0; i < n; ++i)
                        std::swap(a.e[i][k], a.e[i][piv]);
                    std::swap(nrmU[k], nrmU[piv]);
                    std::swap(nrmD[k], nrmD[piv]);
                }
                // Householder reflector for column k, rows k..n-1
                float tail = 0.0f;
                if (n - k > 1) {
                    tail = a.e[k + 1][k] * a.e[k + 1][k];
                    for (int i = k + 2; i < n; ++i)
                        tail = tail + a.e[i][k] * a.e[i][k];
                }
                const float head = a.e[k][k];
                float beta;
                if (tail <= std::numeric_limits<float>::min()) {
                    tau[k] = 0.0f;
                    beta = head;
                    for (int i = k + 1; i < n; ++i)
                        a.e[i][k] = 0.0f;
                } else {
                    beta = std::sqrt(head * head + tail);
                    if (head >= 0.0f)
                        beta = -beta;
                    const float d = head - beta;
                    for (int i = k + 1; i < n; ++i)
                        a.e[i][k] = a.e[i][k] / d;
                    tau[k] = (beta - head) / beta;
                }
                a.e[k][k] = beta;
                // reflect the trailing columns
                if (k + 1 < n) {
                    if (n - k == 1) {
                        for (int j = k + 1; j < n; ++j)
                            a.e[k][j] = a.e[k][j] * (1.0f - tau[k]);
                    } else if (tau[k] != 0.0f) {
                        float w[4];
                        for (int j = k + 1; j < n; ++j) {
                            float acc = 0.0f;
                            for (int i = k + 1; i < n; ++i)
                                acc = acc + a.e[i][k] * a.e[i][j];
                            w[j] = acc + a.e[k][j];
                        }
                        for (int j = k + 1; j < n; ++j)
                            a.e[k][j] = a.e[k][j] - tau[k] * w[j];
                        float tv[4];
                        for (int i = k + 1; i < n; ++i)
                            tv[i] = tau[k] * a.e[i][k];
                        for (int j = k + 1; j < n; ++j)
                            for (int i = k + 1; i < n; ++i)
                                a.e[i][j] = a.e[i][j] - w[j] * tv[i];
                    }
                }
                for (int j = k + 1; j < n; ++j) {
                    if (nrmU[j] == 0.0f)
                        continue;
                    float r = std::fabs(a.e[k][j]) / nrmU[j];
                    r = (1.0f + r) * (1.0f - r);
                    if (r < 0.0f)
                        r = 0.0f;
                    const float q = nrmU[j] / nrmD[j];
                    if (r * (q * q) <= downdateThr) {
                        float acc = 0.0f;
                        if (k + 1 < n) {
                            acc = a.e[k + 1][j] * a.e[k + 1][j];
                            for (int i = k + 2; i < n; ++i)
                                acc = acc + a.e[i][j] * a.e[i][j];
                        }
                        nrmD[j] = nrmU[j] = std::sqrt(acc);
                    } else {
                        nrmU[j] = nrmU[j] * std::sqrt(r);
                    }
                }
            }
            int order[4];
            for (int i = 0; i < n; ++i)
                order[i] = i;
            for (int k = 0; k < n; ++k)
                std::swap(order[k], order[swapWith[k]]);
            for (int i = 0; i < n; ++i)
                x[i] = 0.0f;
            if (rank == 0)
                return;
            float c[4];
            for (int i = 0; i < n; ++i)
                c[i] = b[i];
            for (int k = 0; k < rank; ++k) {
                if (n - k == 1) {
                    c[k] = c[k] * (1.0f - tau[k]);
                } else if (tau[k] != 0.0f) {
                    float acc = 0.0f;
                    for (int i = k + 1; i < n; ++i)
                        acc = acc + a.e[i][k] * c[i];
                    acc = acc + c[k];
                    c[k] = c[k] - tau[k] * acc;
                    for (int i = k + 1; i < n; ++i)
                        c[i] = c[i] - acc * (tau[k] * a.e[i][k]);
                }
            }
            for (int i = rank - 1; i >= 0; --i) {
                if (c[i] == 0.0f)
                    continue;
                c[i] = c[i] / a.e[i][i];
                for (int s = 0; s < i; ++s)
                    c[s] = c[s] - c[i] * a.e[s][i];
            }
            for (int i = 0; i < rank; ++i)
                x[order[i]] = c[i];
        }

        struct Pose {
            int dim;
            M4 K, R, S;
            float t[3] = {};
            float sdd = 0;
        };

        PoseRecord finish(const Pose& g)
        {
            const int d = g.dim;
            M4 Rt(d + 1, d + 1);
            for (int i = 0; i < d; ++i) {
                for (int j = 0; j < d; ++j)
                    Rt.e[i][j] = g.R.e[i][j];
                Rt.e[i][d] = g.t[i];
            }
            Rt.e[d][d] = 1.0f;
            const M4 extFull = prod(Rt, g.S);
            const M4 P = prod(prod(g.K, M4(d, d + 1, true)), extFull);

            M4 P3(d, d);
            float p4[3];
            for (int i = 0; i < d; ++i) {
                for (int j = 0; j < d; ++j)
                    P3.e[i][j] = P.e[i][j];
                p4[i] = P.e[i][d];
            }
            float centre[3] = {};
            solveColPivQr(P3, p4, centre);

            M4 Sinv(d + 1, d + 1);
            for (int i = 0; i <= d; ++i)
                Sinv.e[i][i] = 1.0f / g.S.e[i][i];
            M4 Kinv(d, d, true);
            Kinv.e[0][0] = 1.0f / g.K.e[0][0];
            Kinv.e[0][d - 1] = -g.K.e[0][d - 1] / g.K.e[0][0];
            if (d == 3) {
                Kinv.e[1][1] = 1.0f / g.K.e[1][1];
                Kinv.e[1][d - 1] = -g.K.e[1][d - 1] / g.K.e[1][1];
            }
            M4 RtInv(d + 1, d + 1);
            for (int i = 0; i < d; ++i) {
                float acc = 0.0f;
                for (int k = 0; k < d; ++k) {
                    RtInv.e[i][k] = g.R.e[k][i];
                    acc = acc + g.R.e[k][i] * g.t[k];
                }
                RtInv.e[i][d] = -acc;
            }
            RtInv.e[d][d] = 1.0f;
            const M4 Pinv = prod(prod(prod(Sinv, RtInv), M4(d + 1, d, true)), Kinv);

            PoseRecord rec;
            std::memset(rec.v, 0, sizeof(rec.v));
            for (int i = 0; i < d; ++i)
                for (int j = 0; j <= d; ++j) {
                    rec.v[kPoseOffP + i * (d + 1) + j] = P.e[i][j];
                    rec.v[kPoseOffExt + i * (d + 1) + j] = extFull.e[i][j];
                }
            for (int i = 0; i <= d; ++i)
                for (int j = 0; j < d; ++j)
                    rec.v[kPoseOffPinv + i * d + j] = Pinv.e[i][j];
            for (int i = 0; i < d; ++i)
                rec.v[kPoseOffC + i] = -centre[i];
            rec.v[kPoseOffSdd] = g.sdd;
            return rec;
        }

        // _t = R * (-corOffset - origin), computed as a GEMV row by row
        void translation(Pose& g, const float* volOrigin, const float* corOffset)
        {
            float v[3];
            for (int i = 0; i < g.dim; ++i)
                v[i] = -corOffset[i] - volOrigin[i];
            for (int i = 0; i < g.dim; ++i) {
                float acc = 0.0f;
                for (int k = 0; k < g.dim; ++k)
                    acc = acc + g.R.e[i][k] * v[k];
                g.t[i] = acc;
            }
        }
    } // namespace

    PoseRecord makePose2d(float s2c, float c2d, float angle, const float* volSpacing,
                          const float* volOrigin, const float* sinoSpacing,
                          const float* sinoOrigin, float ppOffset, const float* corOffset)
    {
        Pose g;
        g.dim = 2;
        g.sdd = s2c + c2d;
        const float c = std::cos(angle), s = std::sin(angle);
        g.R = M4(2, 2);
        g.R.e[0][0] = c;
        g.R.e[0][1] = -s;
        g.R.e[1][0] = s;
        g.R.e[1][1] = c;
        g.S = M4(3, 3, true);
        g.S.e[0][0] = volSpacing[0];
        g.S.e[1][1] = volSpacing[1];
        translation(g, volOrigin, corOffset);
        g.t[1] = g.t[1] + s2c;
        g.K = M4(2, 2, true);
        g.K.e[0][0] = (s2c + c2d) / sinoSpacing[0];
        g.K.e[0][1] = sinoOrigin[0] / sinoSpacing[0] + ppOffset;
        return finish(g);
    }

    PoseRecord makePose3d(float s2c, float c2d, const float* volSpacing, const float* volOrigin,
                          const float* sinoSpacing, const float* sinoOrigin, float gamma,
                          float beta, float alpha, const float* ppOffset, const float* corOffset)
    {
        Pose g;
        g.dim = 3;
        g.sdd = s2c + c2d;
        const float ca = std::cos(alpha), sa = std::sin(alpha);
        const float cb = std::cos(beta), sb = std::sin(beta);
        const float cg = std::cos(gamma), sg = std::sin(gamma);
        M4 ry1(3, 3), rz(3, 3), ry2(3, 3);
        ry1.e[0][0] = cg, ry1.e[0][2] = sg, ry1.e[1][1] = 1, ry1.e[2][0] = -sg, ry1.e[2][2] = cg;
        rz.e[0][0] = cb, rz.e[0][1] = -sb, rz.e[1][0] = sb, rz.e[1][1] = cb, rz.e[2][2] = 1;
        ry2.e[0][0] = ca, ry2.e[0][2] = sa, ry2.e[1][1] = 1, ry2.e[2][0] = -sa, ry2.e[2][2] = ca;
        g.R = prod(prod(ry1, rz), ry2);
        g.S = M4(4, 4, true);
        for (int i = 0; i < 3; ++i)
            g.S.e[i][i] = volSpacing[i];
        translation(g, volOrigin, corOffset);
        g.t[2] = g.t[2] + s2c;
        g.K = M4(3, 3, true);
        g.K.e[0][0] = (s2c + c2d) / sinoSpacing[0];
        g.K.e[0][2] = sinoOrigin[0] / sinoSpacing[0] + ppOffset[0];
        g.K.e[1][1] = (s2c + c2d) / sinoSpacing[1];
        g.K.e[1][2] = sinoOrigin[1] / sinoSpacing[1] + ppOffset[1];
        return finish(g);
    }

    std::vector<PoseRecord> circleTrajectory(int dim, const int64_t* volDims,
                                             const float* volSpacing, int64_t numPoses,
                                             float arcDegrees, float s2c, float c2d,
                                             const int64_t* detSize, const float* detSpacing,
                                             int64_t* detDims)
    {
        float volOrigin[3] = {}, spacing[3] = {}, sinoOrigin[3] = {};
        for (int i = 0; i < dim; ++i)
            volOrigin[i] = 0.5f * (static_cast<float>(volDims[i]) * volSpacing[i]);
        for (int i = 0; i < dim - 1; ++i) {
            detDims[i] = detSize ? detSize[i]
                                 : static_cast<int64_t>(static_cast<float>(volDims[i])
                                                        * std::sqrt(2.f));
            spacing[i] = detSpacing ? detSpacing[i] : volSpacing[i];
        }
        detDims[dim - 1] = numPoses;
        spacing[dim - 1] = 1.0f;
        for (int i = 0; i < dim; ++i)
            sinoOrigin[i] = 0.5f * (static_cast<float>(detDims[i]) * spacing[i]);

        const float pi = static_cast<float>(3.14159265358979323846);
        const float step = numPoses > 1 ? arcDegrees / static_cast<float>(numPoses - 1) : 0.0f;
        const float zero[3] = {0.0f, 0.0f, 0.0f};
        std::vector<PoseRecord> poses;
        poses.reserve(static_cast<size_t>(numPoses));
        for (int64_t p = 0; p < numPoses; ++p) {
            // LinSpaced(n, 0, arc): i*step, the last entry exactly arc (arc alone when n == 1)
            const float deg = (p == numPoses - 1) ? arcDegrees : static_cast<float>(p) * step;
            const float rad = deg * pi / 180;
            if (dim == 2)
                poses.push_back(makePose2d(s2c, c2d, rad, volSpacing, volOrigin, spacing,
                                           sinoOrigin, 0.0f, zero));
            else
                poses.push_back(makePose3d(s2c, c2d, volSpacing, volOrigin, spacing, sinoOrigin,
                                           rad, 0.0f, 0.0f, zero, zero));
        }
        return poses;
    }

    std::vector<std::vector<int>> splitRoundRobin(const std::vector<int>& indices, int nSubsets)
    {
        std::vector<std::vector<int>> out(static_cast<size_t>(nSubsets));
        for (size_t i = 0; i < indices.size(); ++i)
            out[i % static_cast<size_t>(nSubsets)].push_back(indices[i]);
        return out;
    }

    std::vector<std::vector<int>> splitRotationalClustering(int dim,
                                                            const std::vector<PoseRecord>& poses,
                                                            int nSubsets)
    {
        // rotation block of the extrinsic matrix [R | t] (row stride dim + 1)
        auto rot = [dim](const PoseRecord& r, int i, int j) {
            return r.v[kPoseOffExt + i * (dim + 1) + j];
        };
        // R1 R2^T coefficient (i, j): k-sum in sequence, as a coefficient-based small product
        auto prod = [&](const PoseRecord& a, const PoseRecord& b, int i, int j) {
            float acc = rot(a, i, 0) * rot(b, j, 0);
            for (int k = 1; k < dim; ++k)
                acc = acc + rot(a, i, k) * rot(b, j, k);
            return acc;
        };
        const PoseRecord first = poses.front();
        auto dist = [&](const PoseRecord& g) {
            if (dim == 2)
                return static_cast<double>(std::atan2(prod(first, g, 1, 0), prod(first, g, 0, 0)));
            float trace = prod(first, g, 0, 0) + prod(first, g, 1, 1);
            trace = trace + prod(first, g, 2, 2);
            return std::acos((trace - 1.0) / 2.0);
        };
        std::vector<int> idx(poses.size());
        for (size_t i = 0; i < idx.size(); ++i)
            idx[i] = static_cast<int>(i);
        std::sort(idx.begin(), idx.end(), [&](int lhs, int rhs) {
            return dist(poses[static_cast<size_t>(lhs)]) < dist(poses[static_cast<size_t>(rhs)]);
        });
        return splitRoundRobin(idx, nSubsets);
    }

    std::vector<float> curvedPlanarCoords(int dim, int nu, int nv, float angle, float s2d,
                                          std::vector<float>* columnFactor)
    {
        if (columnFactor)
            columnFactor->assign(static_cast<size_t>(nu), 1.0f);
        const int height = dim == 3 ? nv : 1;
        const float radius = static_cast<float>(nu) / angle;
        const float angleDelta = angle / static_cast<float>(nu);
        const float cx = static_cast<float>(nu) / 2.0f;
        const float cy = static_cast<float>(height) / 2.0f;
        const float circleX = cx, circleY = s2d - radius;
        std::vector<float> out(static_cast<size_t>(nu) * height * 2, 0.0f);
        for (int h = 0; h < height; ++h)
            for (int l = 0; l < nu; ++l) {
                const float c0 = static_cast<float>(l) + 0.5f;
                const float c1 = static_cast<float>(h) + 0.5f;
                const float rayAngle = (c0 - cx) * angleDelta;
                // sin / cos of the float angle evaluated in double, as the unqualified calls on
                // a float argument in the reference resolve
                const float dx = static_cast<float>(std::sin(static_cast<double>(rayAngle))) *
                                 radius;
                const float dd = static_cast<float>(std::cos(static_cast<double>(rayAngle))) *
                                 radius;
                const float px = circleX + dx, py = circleY + dd;
                const float factor = py == 0.0f ? 1.0f : s2d / py;
                if (columnFactor)
                    (*columnFactor)[static_cast<size_t>(l)] = factor;
                const size_t i = (static_cast<size_t>(h) * nu + l) * 2;
                out[i] = (px - cx) * factor + cx;
                out[i + 1] = dim == 3 ? (c1 - cy) * factor + cy : 0.0f;
            }
        return out;
    }
} // namespace elsa_b200
