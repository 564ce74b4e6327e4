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
 * generators/CircleTrajectoryGenerator.h, the projectors_cuda headers, solvers/CGNE.h, CGLS.h,
 * Landweber.h, APGD.h and the proximal_operators headers. DataContainer<float> here owns device
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
                  range_(std::make_shared<PlanarDetectorDescriptor>(range))
            {
                if (domain.getNumberOfDimensions() != range.getNumberOfDimensions())
                    throw Error(ELSA_ERROR_INVALID_ARGUMENT,
                                "domain and range dimension need to match");
                elsa_projector* h = nullptr;
                check(elsa_projector_create(
                    kind, static_cast<int32_t>(domain.getNumberOfDimensions()),
                    domain.getNumberOfCoefficientsPerDimension().data(),
                    range.getNumberOfCoefficientsPerDimension().data(), range.poses().data(),
                    params.empty() ? nullptr : params.data(), static_cast<int32_t>(params.size()),
                    &h));
                handle_.reset(h, [](elsa_projector* p) { elsa_projector_destroy(p); });
            }
            virtual ~LinearOperator() = default;

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
            JosephsMethodCUDA(const VolumeDescriptor& v, const PlanarDetectorDescriptor& d,
                              bool /*fast: the matched adjoint is always used*/ = true)
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
                elsa_solver* s = nullptr;
                check(elsa_solver_create(kind_, A_.handle(), b_.data(), x.data(), x0 ? 1 : 0,
                                         params_.empty() ? nullptr : params_.data(),
                                         static_cast<int32_t>(params_.size()), nullptr, &s));
                std::unique_ptr<elsa_solver, elsa_status (*)(elsa_solver*)> guard(
                    s, elsa_solver_destroy);
                check(elsa_solver_iterate(s, static_cast<int32_t>(iterations), nullptr));
                double res = 0;
                check(elsa_solver_squared_residual(s, nullptr, &res)); // synchronizes
                lastResidual_ = res;
                return x;
            }
            double lastSquaredResidual() const { return lastResidual_; }

        private:
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
