/*
 * elsa_b200.hpp: a header-only C++17 layer over the C ABI (elsa_b200.h) with elsa's class names
 * and signatures, so that C++ code written against elsa's operator and solver API ports with a
 * namespace change:
 *
 *   using namespace elsa_b200::elsa;
 *   VolumeDescriptor vol({256, 256, 256});
 *   auto sino = CircleTrajectoryGenerator::createTrajectory(360, vol, 360, 2560, 640,
 *                                                           IndexVector{384, 384});
 *   JosephsMethodCUDA<float> A(vol, *sino);
 *   DataContainer<float> b = A.apply(x);
 *   DataContainer<float> rec = CGNE<float>(A, b).solve(30);
 *
 * Reference interfaces: core/LinearOperator.h:38-195 (apply / applyAdjoint),
 * core/Descriptors/VolumeDescriptor.h, PlanarDetectorDescriptor.h,
 * CurvedDetectorDescriptor.h, generators/CircleTrajectoryGenerator.h,
 * CurvedCircleTrajectoryGenerator.h, the projectors_cuda headers, projectors/BinaryMethod.h,
 * LutProjector.h, SubsetSampler.h, solvers/CGNE.h, CGLS.h, Landweber.h, APGD.h, SIRT.h, FGM.h,
 * OGM.h, SQS.h, the proximal_operators headers and io/EDFHandler.h, MHDHandler.h, PGMHandler.h.
 * DataContainer<float> here owns device
 * memory (elsa's is a thrust::universal_vector); its data is float32, x fastest, like elsa's.
 */
#ifndef ELSA_B200_HPP
#define ELSA_B200_HPP

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <memory>
#include <optional>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "elsa_b200.h"

namespace elsa_b200
{
    class Error : public std::runtime_error
    {
    public:
        Error(elsa_status s, const std::string& msg) : std::runtime_error(msg), status(s) {}
        elsa_status status;
    };

    inline void check(elsa_status s)
    {
        if (s != ELSA_SUCCESS)
            throw Error(s, elsa_last_error());
    }

    inline void checkCuda(cudaError_t e, const char* what)
    {
        if (e != cudaSuccess)
            throw Error(ELSA_ERROR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }

    namespace elsa
    {
        using IndexVector = std::vector<int64_t>;
        using RealVector = std::vector<float>;

        // core/Descriptors/DataDescriptor.h
        class DataDescriptor
        {
        public:
            explicit DataDescriptor(IndexVector size, RealVector spacing = {})
                : size_(std::move(size)), spacing_(std::move(spacing))
            {
                if (size_.empty())
                    throw Error(ELSA_ERROR_INVALID_ARGUMENT, "DataDescriptor: empty size");
                for (auto n : size_)
                    if (n <= 0)
                        throw Error(ELSA_ERROR_INVALID_ARGUMENT, "DataDescriptor: invalid size");
                if (spacing_.empty())
                    spacing_.assign(size_.size(), 1.0f);
                if (spacing_.size() != size_.size())
                    throw Error(ELSA_ERROR_INVALID_ARGUMENT, "DataDescriptor: spacing size");
            }
            virtual ~DataDescriptor() = default;
            int64_t getNumberOfDimensions() const { return static_cast<int64_t>(size_.size()); }
            const IndexVector& getNumberOfCoefficientsPerDimension() const { return size_; }
            const RealVector& getSpacingPerDimension() const { return spacing_; }
            int64_t getNumberOfCoefficients() const
            {
                int64_t n = 1;
                for (auto v : size_)
                    n *= v;
                return n;
            }

        private:
            IndexVector size_;
            RealVector spacing_;
        };

        class VolumeDescriptor : public DataDescriptor
        {
        public:
            using DataDescriptor::DataDescriptor;
        };

        // core/Descriptors/PlanarDetectorDescriptor.h: one pose record (elsa_b200.h layout)
        // per projection; the last dimension counts the poses.
        class PlanarDetectorDescriptor : public DataDescriptor
        {
        public:
            PlanarDetectorDescriptor(IndexVector size, std::vector<float> poses,
                                     RealVector spacing = {})
                : DataDescriptor(std::move(size), std::move(spacing)), poses_(std::move(poses))
            {
                const auto n = getNumberOfCoefficientsPerDimension().back();
                if (static_cast<int64_t>(poses_.size()) != n * ELSA_POSE_FLOATS)
                    throw Error(ELSA_ERROR_INVALID_ARGUMENT,
                                "PlanarDetectorDescriptor: poses do not match the last dimension");
            }
            int64_t getNumberOfGeometryPoses() const
            {
                return getNumberOfCoefficientsPerDimension().back();
            }
            const std::vector<float>& poses() const { return poses_; }

        private:
            std::vector<float> poses_;
        };

        // generators/CircleTrajectoryGenerator.h
        struct CircleTrajectoryGenerator {
            static std::unique_ptr<PlanarDetectorDescriptor>
                createTrajectory(int64_t numberOfPoses, const DataDescriptor& volumeDescriptor,
                                 int64_t arcDegrees, float sourceToCenter, float centerToDetector,
                                 std::optional<IndexVector> detectorSize = std::nullopt,
                                 std::optional<RealVector> detectorSpacing = std::nullopt)
            {
                const int32_t dim = static_cast<int32_t>(volumeDescriptor.getNumberOfDimensions());
                std::vector<float> poses(static_cast<size_t>(numberOfPoses) * ELSA_POSE_FLOATS);
                IndexVector det(static_cast<size_t>(dim));
                check(elsa_circle_trajectory(
                    dim, volumeDescriptor.getNumberOfCoefficientsPerDimension().data(),
                    volumeDescriptor.getSpacingPerDimension().data(), numberOfPoses,
                    static_cast<float>(arcDegrees), sourceToCenter, centerToDetector,
                    detectorSize ? detectorSize->data() : nullptr,
                    detectorSpacing ? detectorSpacing->data() : nullptr, poses.data(),
                    det.data()));
                RealVector spacing = detectorSpacing
                                         ? *detectorSpacing
                                         : RealVector(volumeDescriptor.getSpacingPerDimension().begin(),
                                                      volumeDescriptor.getSpacingPerDimension().end() - 1);
                spacing.push_back(1.0f);
                return std::make_unique<PlanarDetectorDescriptor>(det, std::move(poses), spacing);
            }
        };

        // core/Descriptors/CurvedDetectorDescriptor.h: the poses of a flat detector plus the
        // opening angle (radian) and the source-to-detector distance
        class CurvedDetectorDescriptor : public PlanarDetectorDescriptor
        {
        public:
            CurvedDetectorDescriptor(IndexVector size, std::vector<float> poses, float angle,
                                     float s2d, RealVector spacing = {})
                : PlanarDetectorDescriptor(std::move(size), std::move(poses), std::move(spacing)),
                  angle_(angle), s2d_(s2d)
            {
            }
            float angle() const { return angle_; }
            float sourceToDetector() const { return s2d_; }
            float getRadius() const
            {
                return static_cast<float>(getNumberOfCoefficientsPerDimension()[0]) / angle_;
            }
            // planar (u', v') per pixel centre, u fastest (CurvedDetectorDescriptor::
            // getPlanarCoords)
            std::vector<float> getPlanarCoords() const
            {
                const auto& n = getNumberOfCoefficientsPerDimension();
                const int32_t dim = static_cast<int32_t>(n.size());
                const int32_t nv = dim == 3 ? static_cast<int32_t>(n[1]) : 1;
                std::vector<float> out(2 * static_cast<size_t>(n[0]) * nv);
                check(elsa_curved_detector_coords(dim, static_cast<int32_t>(n[0]), nv, angle_,
                                                  s2d_, out.data()));
                return out;
            }

        private:
            float angle_, s2d_;
        };

        // generators/CurvedCircleTrajectoryGenerator.cpp:8-30
        struct CurvedCircleTrajectoryGenerator {
            static std::unique_ptr<CurvedDetectorDescriptor>
                createTrajectory(int64_t numberOfPoses, const DataDescriptor& volumeDescriptor,
                                 int64_t arcDegrees, float sourceToCenter, float centerToDetector,
                                 float angle, std::optional<IndexVector> detectorSize = std::nullopt,
                                 std::optional<RealVector> detectorSpacing = std::nullopt)
            {
                auto flat = CircleTrajectoryGenerator::createTrajectory(
                    numberOfPoses, volumeDescriptor, arcDegrees, sourceToCenter, centerToDetector,
                    detectorSize, detectorSpacing);
                return std::make_unique<CurvedDetectorDescriptor>(
                    flat->getNumberOfCoefficientsPerDimension(), flat->poses(), angle,
                    sourceToCenter + centerToDetector, flat->getSpacingPerDimension());
            }
        };

        // core/DataContainer.h, float32 on the device (x fastest). Copyable (deep copy).
        template <typename data_t>
        class DataContainer
        {
            static_assert(sizeof(data_t) == 4, "elsa_b200 computes in float32");

        public:
            explicit DataContainer(std::shared_ptr<const DataDescriptor> desc) : desc_(std::move(desc))
            {
                allocate();
                checkCuda(cudaMemset(ptr_, 0, bytes()), "cudaMemset");
            }
            DataContainer(std::shared_ptr<const DataDescriptor> desc, const std::vector<data_t>& host)
                : desc_(std::move(desc))
            {
                if (static_cast<int64_t>(host.size()) != getSize())
                    throw Error(ELSA_ERROR_INVALID_ARGUMENT, "DataContainer: size mismatch");
                allocate();
                checkCuda(cudaMemcpy(ptr_, host.data(), bytes(), cudaMemcpyHostToDevice),
                          "cudaMemcpy");
            }
            DataContainer(const DataContainer& o) : desc_(o.desc_)
            {
                allocate();
                checkCuda(cudaMemcpy(ptr_, o.ptr_, bytes(), cudaMemcpyDeviceToDevice), "cudaMemcpy");
            }
            DataContainer(DataContainer&& o) noexcept : desc_(std::move(o.desc_)), ptr_(o.ptr_)
            {
                o.ptr_ = nullptr;
            }
            DataContainer& operator=(DataContainer o)
            {
                std::swap(desc_, o.desc_);
                std::swap(ptr_, o.ptr_);
                return *this;
            }
            ~DataContainer()
            {
                if (ptr_)
                    cudaFree(ptr_);
            }

            const DataDescriptor& getDataDescriptor() const { return *desc_; }
            std::shared_ptr<const DataDescriptor> descriptor() const { return desc_; }
            int64_t getSize() const { return desc_->getNumberOfCoefficients(); }
            data_t* data() { return ptr_; }
            const data_t* data() const { return ptr_; }

            std::vector<data_t> toHost() const
            {
                std::vector<data_t> h(static_cast<size_t>(getSize()));
                checkCuda(cudaMemcpy(h.data(), ptr_, bytes(), cudaMemcpyDeviceToHost), "cudaMemcpy");
                return h;
            }

            // float64-accumulated reductions (storage/reductions) and lincomb on the device
            double dot(const DataContainer& o) const
            {
                double* d = nullptr;
                checkCuda(cudaMalloc(&d, sizeof(double)), "cudaMalloc");
                const elsa_status st = elsa_dot(ptr_, o.ptr_, getSize(), d, nullptr);
                double h = 0;
                cudaMemcpy(&h, d, sizeof(double), cudaMemcpyDeviceToHost);
                cudaFree(d);
                check(st);
                return h;
            }
            double squaredL2Norm() const { return dot(*this); }
            double l2Norm() const { return std::sqrt(squaredL2Norm()); }

        private:
            size_t bytes() const { return sizeof(data_t) * static_cast<size_t>(getSize()); }
            void allocate()
            {
                checkCuda(cudaMalloc(reinterpret_cast<void**>(&ptr_), bytes() ? bytes() : 4),
                          "cudaMalloc");
            }
            std::shared_ptr<const DataDescriptor> desc_;
            data_t* ptr_ = nullptr;
        };

        // out = a x + b y (core/DataContainer.cpp:1075-1108)
        template <typename data_t>
        void lincomb(data_t a, const DataContainer<data_t>& x, data_t b,
                     const DataContainer<data_t>& y, DataContainer<data_t>& out)
        {
            check(elsa_lincomb(a, x.data(), b, y.data(), out.data(), x.getSize(), nullptr));
        }

        // core/LinearOperator.h: apply / applyAdjoint on device containers
        template <typename data_t>
        class LinearOperator
        {
        public:
            LinearOperator(const DataDescriptor& domain, const PlanarDetectorDescriptor& range,
                           int32_t kind, std::vector<float> params = {})
                : domain_(std::make_shared<VolumeDescriptor>(
                      domain.getNumberOfCoefficientsPerDimension(),
                      domain.getSpacingPerDimension())),
                  range_(copyRange(range))
            {
                if (domain.getNumberOfDimensions() != range.getNumberOfDimensions())
                    throw Error(ELSA_ERROR_INVALID_ARGUMENT,
                                "domain and range dimension need to match");
                elsa_projector* h = nullptr;
                const auto* curved = dynamic_cast<const CurvedDetectorDescriptor*>(&range);
                if (curved)
                    check(elsa_projector_create_curved(
                        kind, static_cast<int32_t>(domain.getNumberOfDimensions()),
                        domain.getNumberOfCoefficientsPerDimension().data(),
                        range.getNumberOfCoefficientsPerDimension().data(), range.poses().data(),
                        params.empty() ? nullptr : params.data(),
                        static_cast<int32_t>(params.size()), curved->angle(),
                        curved->sourceToDetector(), &h));
                else
                    check(elsa_projector_create(
                        kind, static_cast<int32_t>(domain.getNumberOfDimensions()),
                        domain.getNumberOfCoefficientsPerDimension().data(),
                        range.getNumberOfCoefficientsPerDimension().data(), range.poses().data(),
                        params.empty() ? nullptr : params.data(),
                        static_cast<int32_t>(params.size()), &h));
                handle_.reset(h, [](elsa_projector* p) { elsa_projector_destroy(p); });
            }
            virtual ~LinearOperator() = default;

            static std::shared_ptr<const PlanarDetectorDescriptor>
                copyRange(const PlanarDetectorDescriptor& r)
            {
                if (const auto* c = dynamic_cast<const CurvedDetectorDescriptor*>(&r))
                    return std::make_shared<CurvedDetectorDescriptor>(*c);
                return std::make_shared<PlanarDetectorDescriptor>(r);
            }

            // autotune the launch parameters for this geometry (elsa_projector_autotune); returns
            // true when the tuning cache supplied them
            bool autotune(bool force = false)
            {
                int32_t hit = 0;
                check(elsa_projector_autotune(handle_.get(), nullptr, force ? 1 : 0, nullptr,
                                              &hit));
                return hit != 0;
            }

            // launch knobs (ELSA_KNOB_*, elsa_projector_get_knob / _set_knob): e.g.
            // setKnob(ELSA_KNOB_ADJOINT_SCATTER, 1) selects Siddon's atomic scatter adjoint
            // instead of the bit-reproducible brick owner
            int32_t getKnob(int32_t knob) const
            {
                int32_t v = -1;
                check(elsa_projector_get_knob(handle_.get(), knob, &v));
                return v;
            }
            void setKnob(int32_t knob, int32_t value)
            {
                check(elsa_projector_set_knob(handle_.get(), knob, value));
            }

            const DataDescriptor& getDomainDescriptor() const { return *domain_; }
            const DataDescriptor& getRangeDescriptor() const { return *range_; }
            elsa_projector* handle() const { return handle_.get(); }

            void apply(const DataContainer<data_t>& x, DataContainer<data_t>& Ax) const
            {
                check(elsa_projector_apply(handle_.get(), x.data(), Ax.data(), nullptr));
            }
            DataContainer<data_t> apply(const DataContainer<data_t>& x) const
            {
                DataContainer<data_t> Ax(range_);
                apply(x, Ax);
                return Ax;
            }
            void applyAdjoint(const DataContainer<data_t>& y, DataContainer<data_t>& Aty) const
            {
                check(elsa_projector_apply_adjoint(handle_.get(), y.data(), Aty.data(), nullptr));
            }
            DataContainer<data_t> applyAdjoint(const DataContainer<data_t>& y) const
            {
                DataContainer<data_t> Aty(domain_);
                applyAdjoint(y, Aty);
                return Aty;
            }
            std::shared_ptr<const DataDescriptor> domain() const { return domain_; }
            std::shared_ptr<const DataDescriptor> range() const { return range_; }

        private:
            std::shared_ptr<const DataDescriptor> domain_, range_;
            std::shared_ptr<elsa_projector> handle_;
        };

        template <typename data_t>
        struct JosephsMethodCUDA : LinearOperator<data_t> {
            // fast: elsa's unmatched `fast` adjoint (JosephsMethodCUDA.h:60-67). elsa defaults to
            // it; here the matched adjoint (the transpose, as the CPU JosephsMethod) is the
            // default, since the solvers assume a transpose.
            JosephsMethodCUDA(const VolumeDescriptor& v, const PlanarDetectorDescriptor& d,
                              bool fast = false)
                : LinearOperator<data_t>(v, d, ELSA_PROJECTOR_JOSEPH,
                                         fast ? std::vector<float>{1.0f} : std::vector<float>{})
            {
            }
        };

        // projectors/JosephsMethod.h: the matched Joseph projector
        template <typename data_t>
        struct JosephsMethod : LinearOperator<data_t> {
            JosephsMethod(const VolumeDescriptor& v, const PlanarDetectorDescriptor& d)
                : LinearOperator<data_t>(v, d, ELSA_PROJECTOR_JOSEPH)
            {
            }
        };

        template <typename data_t>
        struct SiddonsMethodCUDA : LinearOperator<data_t> {
            SiddonsMethodCUDA(const VolumeDescriptor& v, const PlanarDetectorDescriptor& d)
                : LinearOperator<data_t>(v, d, ELSA_PROJECTOR_SIDDON)
            {
            }
        };

        template <typename data_t>
        struct BlobVoxelProjectorCUDA : LinearOperator<data_t> {
            BlobVoxelProjectorCUDA(const VolumeDescriptor& v, const PlanarDetectorDescriptor& d,
                                   float radius = 2.0f, float alpha = 10.83f, int order = 2)
                : LinearOperator<data_t>(v, d, ELSA_PROJECTOR_BLOB,
                                         {radius, alpha, static_cast<float>(order)})
            {
            }
        };

        template <typename data_t>
        struct BSplineVoxelProjectorCUDA : LinearOperator<data_t> {
            BSplineVoxelProjectorCUDA(const VolumeDescriptor& v, const PlanarDetectorDescriptor& d,
                                      int order = 2)
                : LinearOperator<data_t>(v, d, ELSA_PROJECTOR_BSPLINE, {static_cast<float>(order)})
            {
            }
        };

        template <typename data_t>
        struct PhaseContrastBlobVoxelProjectorCUDA : LinearOperator<data_t> {
            PhaseContrastBlobVoxelProjectorCUDA(const VolumeDescriptor& v,
                                                const PlanarDetectorDescriptor& d,
                                                float radius = 2.0f, float alpha = 10.83f,
                                                int order = 2)
                : LinearOperator<data_t>(v, d, ELSA_PROJECTOR_PHASE_CONTRAST_BLOB,
                                         {radius, alpha, static_cast<float>(order)})
            {
            }
        };

        template <typename data_t>
        struct PhaseContrastBSplineVoxelProjectorCUDA : LinearOperator<data_t> {
            PhaseContrastBSplineVoxelProjectorCUDA(const VolumeDescriptor& v,
                                                   const PlanarDetectorDescriptor& d,
                                                   int order = 2)
                : LinearOperator<data_t>(v, d, ELSA_PROJECTOR_PHASE_CONTRAST_BSPLINE,
                                         {static_cast<float>(order)})
            {
            }
        };

        // projectors/BinaryMethod.h: Siddon's traversal with weight 1 per visited voxel
        template <typename data_t>
        struct BinaryMethod : LinearOperator<data_t> {
            BinaryMethod(const VolumeDescriptor& v, const PlanarDetectorDescriptor& d)
                : LinearOperator<data_t>(v, d, ELSA_PROJECTOR_BINARY)
            {
            }
        };

        // projectors/LutProjector.h: ray-driven projectors with a blob / B-spline look-up table
        template <typename data_t>
        struct BlobProjector : LinearOperator<data_t> {
            BlobProjector(const VolumeDescriptor& v, const PlanarDetectorDescriptor& d,
                          float radius = 2.0f, float alpha = 10.83f, int order = 2)
                : LinearOperator<data_t>(v, d, ELSA_PROJECTOR_RAY_BLOB,
                                         {radius, alpha, static_cast<float>(order)})
            {
            }
        };

        template <typename data_t>
        struct BSplineProjector : LinearOperator<data_t> {
            BSplineProjector(const VolumeDescriptor& v, const PlanarDetectorDescriptor& d,
                             int order = 2)
                : LinearOperator<data_t>(v, d, ELSA_PROJECTOR_RAY_BSPLINE,
                                         {static_cast<float>(order)})
            {
            }
        };

        // proximal_operators/*: the APGD parameters (elsa_b200.h, ELSA_SOLVER_APGD)
        struct ProximalIdentity {
            std::vector<double> params() const { return {0.0, NAN, NAN, 1.0}; }
        };
        struct ProximalBoxConstraint {
            std::optional<float> lower, upper;
            std::vector<double> params() const
            {
                return {1.0, lower ? double(*lower) : NAN, upper ? double(*upper) : NAN, 1.0};
            }
        };
        struct ProximalL1 {
            float sigma = 1.0f;
            std::vector<double> params() const { return {2.0, NAN, NAN, double(sigma)}; }
        };

        // solvers/Solver.h: solve(iterations, x0) on a device session (elsa_solver_*)
        template <typename data_t>
        class Solver
        {
        public:
            Solver(const LinearOperator<data_t>& A, const DataContainer<data_t>& b, int32_t kind,
                   std::vector<double> params)
                : A_(A), b_(b), kind_(kind), params_(std::move(params))
            {
            }
            virtual ~Solver() = default;

            DataContainer<data_t> solve(int64_t iterations,
                                        std::optional<DataContainer<data_t>> x0 = std::nullopt)
            {
                DataContainer<data_t> x = x0 ? *x0 : DataContainer<data_t>(A_.domain());
                elsa_solver* s = open(x, x0.has_value());
                std::unique_ptr<elsa_solver, elsa_status (*)(elsa_solver*)> guard(
                    s, elsa_solver_destroy);
                check(elsa_solver_iterate(s, static_cast<int32_t>(iterations), nullptr));
                double res = 0;
                check(elsa_solver_squared_residual(s, nullptr, &res)); // synchronizes
                lastResidual_ = res;
                return x;
            }
            double lastSquaredResidual() const { return lastResidual_; }

        protected:
            // elsa_solver_create on the iterate x; SQS with subsets overrides it
            virtual elsa_solver* open(DataContainer<data_t>& x, bool useX0)
            {
                elsa_solver* s = nullptr;
                check(elsa_solver_create(kind_, A_.handle(), b_.data(), x.data(), useX0 ? 1 : 0,
                                         params_.empty() ? nullptr : params_.data(),
                                         static_cast<int32_t>(params_.size()), nullptr, &s));
                return s;
            }
            const LinearOperator<data_t>& A_;
            const DataContainer<data_t>& b_;
            int32_t kind_;
            std::vector<double> params_;
            double lastResidual_ = 0.0;
        };

        template <typename data_t>
        struct CGNE : Solver<data_t> {
            CGNE(const LinearOperator<data_t>& A, const DataContainer<data_t>& b)
                : Solver<data_t>(A, b, ELSA_SOLVER_CGNE, {})
            {
            }
        };

        template <typename data_t>
        struct CGLS : Solver<data_t> {
            CGLS(const LinearOperator<data_t>& A, const DataContainer<data_t>& b, data_t eps = 0,
                 data_t tol = 1e-4)
                : Solver<data_t>(A, b, ELSA_SOLVER_CGLS, {double(eps), double(tol)})
            {
            }
        };

        template <typename data_t>
        struct Landweber : Solver<data_t> {
            Landweber(const LinearOperator<data_t>& A, const DataContainer<data_t>& b)
                : Solver<data_t>(A, b, ELSA_SOLVER_LANDWEBER, {})
            {
            }
            Landweber(const LinearOperator<data_t>& A, const DataContainer<data_t>& b,
                      data_t stepSize)
                : Solver<data_t>(A, b, ELSA_SOLVER_LANDWEBER, {double(stepSize)})
            {
            }
        };

        template <typename data_t>
        struct APGD : Solver<data_t> {
            template <class Prox>
            APGD(const LinearOperator<data_t>& A, const DataContainer<data_t>& b, Prox prox,
                 std::optional<data_t> mu = std::nullopt,
                 data_t epsilon = static_cast<data_t>(1.1920928955078125e-07))
                : Solver<data_t>(A, b, ELSA_SOLVER_APGD, params(prox, mu, epsilon))
            {
            }

        private:
            template <class Prox>
            static std::vector<double> params(const Prox& prox, std::optional<data_t> mu,
                                              data_t epsilon)
            {
                const auto p = prox.params();
                return {mu ? double(*mu) : 0.0, double(epsilon), p[0], p[1], p[2], p[3]};
            }
        };

        template <typename data_t>
        using FISTA = APGD<data_t>;

        // solvers/SIRT.cpp:8-45
        template <typename data_t>
        struct SIRT : Solver<data_t> {
            SIRT(const LinearOperator<data_t>& A, const DataContainer<data_t>& b,
                 std::optional<data_t> stepSize = std::nullopt)
                : Solver<data_t>(A, b, ELSA_SOLVER_SIRT,
                                 {stepSize ? double(*stepSize) : 0.0})
            {
            }
        };

        // problems/LeastSquares.h: 0.5 |A x - b|^2 (the operator and data are borrowed)
        template <typename data_t>
        struct LeastSquares {
            const LinearOperator<data_t>& A;
            const DataContainer<data_t>& b;
        };

        // solvers/FGM.cpp:33-78 and solvers/OGM.cpp:40-95 on LeastSquares(A, b)
        template <typename data_t>
        struct FGM : Solver<data_t> {
            explicit FGM(const LeastSquares<data_t>& problem,
                         data_t epsilon = static_cast<data_t>(1.1920928955078125e-07))
                : Solver<data_t>(problem.A, problem.b, ELSA_SOLVER_FGM, {double(epsilon)})
            {
            }
        };

        template <typename data_t>
        struct OGM : Solver<data_t> {
            explicit OGM(const LeastSquares<data_t>& problem,
                         data_t epsilon = static_cast<data_t>(1.1920928955078125e-07))
                : Solver<data_t>(problem.A, problem.b, ELSA_SOLVER_OGM, {double(epsilon)})
            {
            }
        };

        // operators/Scaling.h used as a diagonal preconditioner: x -> s .* x
        template <typename data_t>
        struct Scaling {
            const DataContainer<data_t>& scaleFactors;
            const DataContainer<data_t>& getScaleFactors() const { return scaleFactors; }
        };

        // solvers/SQS.cpp:10-22,87-170: SQS(problem[, subsets][, preconditioner],
        // momentumAcceleration, epsilon). The problems and the preconditioner are borrowed and
        // must outlive solve().
        template <typename data_t>
        class SQS : public Solver<data_t>
        {
        public:
            explicit SQS(const LeastSquares<data_t>& problem, bool momentumAcceleration = true,
                         data_t epsilon = static_cast<data_t>(1.1920928955078125e-07))
                : SQS(problem, {}, nullptr, momentumAcceleration, epsilon)
            {
            }
            SQS(const LeastSquares<data_t>& problem,
                std::vector<LeastSquares<data_t>> subsets, bool momentumAcceleration = true,
                data_t epsilon = static_cast<data_t>(1.1920928955078125e-07))
                : SQS(problem, std::move(subsets), nullptr, momentumAcceleration, epsilon)
            {
            }
            SQS(const LeastSquares<data_t>& problem, std::vector<LeastSquares<data_t>> subsets,
                const Scaling<data_t>& preconditioner, bool momentumAcceleration = true,
                data_t epsilon = static_cast<data_t>(1.1920928955078125e-07))
                : SQS(problem, std::move(subsets), &preconditioner.getScaleFactors(),
                      momentumAcceleration, epsilon)
            {
            }

        protected:
            elsa_solver* open(DataContainer<data_t>& x, bool useX0) override
            {
                std::vector<elsa_projector*> ops;
                std::vector<const float*> data;
                for (const auto& sp : subsets_) {
                    ops.push_back(sp.A.handle());
                    data.push_back(sp.b.data());
                }
                elsa_solver* s = nullptr;
                check(elsa_sqs_create(this->A_.handle(), this->b_.data(),
                                      ops.empty() ? nullptr : ops.data(),
                                      data.empty() ? nullptr : data.data(),
                                      static_cast<int32_t>(ops.size()), x.data(), useX0 ? 1 : 0,
                                      momentum_ ? 1 : 0, double(epsilon_),
                                      preconditioner_ ? preconditioner_->data() : nullptr,
                                      nullptr, &s));
                return s;
            }

        private:
            SQS(const LeastSquares<data_t>& problem, std::vector<LeastSquares<data_t>> subsets,
                const DataContainer<data_t>* preconditioner, bool momentum, data_t epsilon)
                : Solver<data_t>(problem.A, problem.b, ELSA_SOLVER_SQS, {}),
                  subsets_(std::move(subsets)), preconditioner_(preconditioner),
                  momentum_(momentum), epsilon_(epsilon)
            {
            }
            std::vector<LeastSquares<data_t>> subsets_;
            const DataContainer<data_t>* preconditioner_;
            bool momentum_;
            data_t epsilon_;
        };

        // projectors/SubsetSampler.h:22-129: ordered subsets of a detector's poses. The
        // partitioned data are one container per subset (the reference's blocks of one
        // PartitionDescriptor container); the projectors are created with the subset detectors.
        template <typename DetectorDescriptor_t, typename data_t>
        class SubsetSampler
        {
        public:
            enum class SamplingStrategy { ROUND_ROBIN, ROTATIONAL_CLUSTERING };

            SubsetSampler(const VolumeDescriptor& volumeDescriptor,
                          const DetectorDescriptor_t& detectorDescriptor, int64_t nSubsets,
                          SamplingStrategy strategy = SamplingStrategy::ROUND_ROBIN)
                : volume_(volumeDescriptor), full_(detectorDescriptor)
            {
                if (nSubsets <= 1)
                    throw Error(ELSA_ERROR_INVALID_ARGUMENT,
                                "SubsetSampler: nSubsets must be >= 2");
                const int32_t np = static_cast<int32_t>(full_.getNumberOfGeometryPoses());
                std::vector<int32_t> order(np), sizes(static_cast<size_t>(nSubsets));
                check(elsa_subset_split(
                    static_cast<int32_t>(full_.getNumberOfDimensions()), full_.poses().data(), np,
                    static_cast<int32_t>(nSubsets),
                    strategy == SamplingStrategy::ROUND_ROBIN ? ELSA_SUBSET_ROUND_ROBIN
                                                              : ELSA_SUBSET_ROTATIONAL_CLUSTERING,
                    order.data(), sizes.data()));
                size_t at = 0;
                for (int32_t n : sizes) {
                    std::vector<int32_t> idx(order.begin() + at, order.begin() + at + n);
                    at += static_cast<size_t>(n);
                    std::vector<float> poses;
                    for (int32_t i : idx)
                        poses.insert(poses.end(), full_.poses().begin() + i * ELSA_POSE_FLOATS,
                                     full_.poses().begin() + (i + 1) * ELSA_POSE_FLOATS);
                    IndexVector size = full_.getNumberOfCoefficientsPerDimension();
                    size.back() = n;
                    detectors_.push_back(subsetDetector(size, std::move(poses)));
                    mapping_.push_back(std::move(idx));
                }
            }

            const std::vector<std::vector<int32_t>>& getIndexMapping() const { return mapping_; }
            const std::vector<std::shared_ptr<DetectorDescriptor_t>>&
                getSubsetDetectorDescriptors() const
            {
                return detectors_;
            }

            std::vector<DataContainer<data_t>>
                getPartitionedData(const DataContainer<data_t>& sinogram) const
            {
                const auto& n = full_.getNumberOfCoefficientsPerDimension();
                int64_t view = 1;
                for (size_t d = 0; d + 1 < n.size(); ++d)
                    view *= n[d];
                std::vector<DataContainer<data_t>> out;
                for (size_t i = 0; i < mapping_.size(); ++i) {
                    out.emplace_back(detectors_[i]);
                    check(elsa_gather_views(sinogram.data(), view, mapping_[i].data(),
                                            static_cast<int32_t>(mapping_[i].size()),
                                            static_cast<int32_t>(n.back()), out.back().data(),
                                            nullptr));
                }
                checkCuda(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
                return out;
            }

            template <typename Projector_t>
            std::unique_ptr<Projector_t> getProjector() const
            {
                return std::make_unique<Projector_t>(volume_, full_);
            }
            template <typename Projector_t>
            std::vector<std::unique_ptr<Projector_t>> getSubsetProjectors() const
            {
                std::vector<std::unique_ptr<Projector_t>> out;
                for (const auto& d : detectors_)
                    out.push_back(std::make_unique<Projector_t>(volume_, *d));
                return out;
            }

        private:
            std::shared_ptr<DetectorDescriptor_t> subsetDetector(IndexVector size,
                                                                 std::vector<float> poses) const
            {
                if constexpr (std::is_same_v<DetectorDescriptor_t, CurvedDetectorDescriptor>)
                    return std::make_shared<CurvedDetectorDescriptor>(
                        std::move(size), std::move(poses), full_.angle(),
                        full_.sourceToDetector(), full_.getSpacingPerDimension());
                else
                    return std::make_shared<DetectorDescriptor_t>(
                        std::move(size), std::move(poses), full_.getSpacingPerDimension());
            }
            VolumeDescriptor volume_;
            DetectorDescriptor_t full_;
            std::vector<std::vector<int32_t>> mapping_;
            std::vector<std::shared_ptr<DetectorDescriptor_t>> detectors_;
        };

        // io/EDFHandler.h, io/MHDHandler.h, io/PGMHandler.h on device containers (the data
        // pass through host memory)
        namespace detail
        {
            inline std::shared_ptr<VolumeDescriptor> imageDescriptor(const elsa_image_info& info)
            {
                return std::make_shared<VolumeDescriptor>(
                    IndexVector(info.dims, info.dims + info.ndim),
                    RealVector(info.spacing, info.spacing + info.ndim));
            }
        } // namespace detail

        struct EDF {
            template <typename data_t>
            static DataContainer<data_t> read(const std::string& filename)
            {
                elsa_image_info info{};
                check(elsa_edf_info(filename.c_str(), &info));
                auto desc = detail::imageDescriptor(info);
                std::vector<data_t> host(static_cast<size_t>(desc->getNumberOfCoefficients()));
                check(elsa_edf_read(filename.c_str(), host.data(),
                                    static_cast<int64_t>(host.size())));
                return DataContainer<data_t>(desc, host);
            }
            template <typename data_t>
            static void write(const DataContainer<data_t>& data, const std::string& filename)
            {
                const auto& d = data.getDataDescriptor();
                const auto host = data.toHost();
                check(elsa_edf_write(filename.c_str(), host.data(),
                                     static_cast<int32_t>(d.getNumberOfDimensions()),
                                     d.getNumberOfCoefficientsPerDimension().data(),
                                     d.getSpacingPerDimension().data()));
            }
        };

        struct MHD {
            template <typename data_t>
            static DataContainer<data_t> read(const std::string& filename)
            {
                elsa_image_info info{};
                check(elsa_mhd_info(filename.c_str(), &info));
                auto desc = detail::imageDescriptor(info);
                std::vector<data_t> host(static_cast<size_t>(desc->getNumberOfCoefficients()));
                check(elsa_mhd_read(filename.c_str(), host.data(),
                                    static_cast<int64_t>(host.size())));
                return DataContainer<data_t>(desc, host);
            }
            template <typename data_t>
            static void write(const DataContainer<data_t>& data, const std::string& metaFilename,
                              const std::string& rawFilename)
            {
                const auto& d = data.getDataDescriptor();
                const auto host = data.toHost();
                check(elsa_mhd_write(metaFilename.c_str(), rawFilename.c_str(), host.data(),
                                     static_cast<int32_t>(d.getNumberOfDimensions()),
                                     d.getNumberOfCoefficientsPerDimension().data(),
                                     d.getSpacingPerDimension().data()));
            }
        };

        struct PGM {
            template <typename data_t>
            static void write(const DataContainer<data_t>& data, const std::string& filename)
            {
                const auto& d = data.getDataDescriptor();
                const auto host = data.toHost();
                check(elsa_pgm_write(filename.c_str(), host.data(),
                                     static_cast<int32_t>(d.getNumberOfDimensions()),
                                     d.getNumberOfCoefficientsPerDimension().data()));
            }
        };

        // solvers/PowerIterations.cpp:10-27 on adjoint(A) * A
        template <typename data_t>
        double powerIterations(const LinearOperator<data_t>& A, int32_t niters = 5)
        {
            double v = 0;
            check(elsa_power_iterations(A.handle(), niters, nullptr, &v));
            return v;
        }
    } // namespace elsa
} // namespace elsa_b200

#endif /* ELSA_B200_HPP */
