// pybind11 module elsa_b200._pyelsa: elsa's Python class and method names
// (pyelsa/pyelsa/bind_core.cpp, bind_generators.cpp, bind_projectors_cuda.cpp, bind_solvers
// in bind_operators.cpp) bound to the header-only C++ layer (include/elsa_b200.hpp), which sits
// on the C ABI. Data containers live in device memory; the buffer protocol hands out a read-only
// host copy in Fortran order (first index x fastest, as core_hints.cpp:126-185 lays out elsa's
// host containers), and containers are built from numpy arrays in the same order.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <memory>
#include <optional>
#include <string>
#include <vector>

#include "elsa_b200.hpp"

namespace py = pybind11;
using namespace elsa_b200::elsa;

namespace
{
    using DC = DataContainer<float>;
    using LinOp = LinearOperator<float>;

    // A device container plus the host copy its buffer protocol exposes.
    struct PyDataContainer {
        std::shared_ptr<DC> dc;
        std::vector<float> mirror;
    };

    std::shared_ptr<const DataDescriptor> copyDescriptor(const DataDescriptor& d)
    {
        if (const auto* c = dynamic_cast<const CurvedDetectorDescriptor*>(&d))
            return std::make_shared<CurvedDetectorDescriptor>(*c);
        if (const auto* p = dynamic_cast<const PlanarDetectorDescriptor*>(&d))
            return std::make_shared<PlanarDetectorDescriptor>(*p);
        return std::make_shared<VolumeDescriptor>(d.getNumberOfCoefficientsPerDimension(),
                                                  d.getSpacingPerDimension());
    }

    // values in x-fastest order from an array of the descriptor's shape (any memory order) or a
    // flat array
    std::vector<float> xFastest(const py::array& a, const DataDescriptor& d)
    {
        py::module_ np = py::module_::import("numpy");
        const int64_t n = d.getNumberOfCoefficients();
        py::array flat = np.attr("ravel")(np.attr("asarray")(a, "float32"), "F");
        if (flat.size() != n)
            throw elsa_b200::Error(ELSA_ERROR_INVALID_ARGUMENT,
                                   "DataContainer: array size does not match the descriptor");
        py::array_t<float, py::array::forcecast> f(flat);
        return std::vector<float>(f.data(), f.data() + n);
    }

    PyDataContainer makeContainer(std::shared_ptr<const DataDescriptor> desc,
                                  std::optional<py::array> values)
    {
        PyDataContainer out;
        if (values)
            out.dc = std::make_shared<DC>(desc, xFastest(*values, *desc));
        else
            out.dc = std::make_shared<DC>(desc);
        return out;
    }

    PyDataContainer wrap(DC&& d)
    {
        PyDataContainer out;
        out.dc = std::make_shared<DC>(std::move(d));
        return out;
    }

    PyDataContainer combine(const PyDataContainer& x, float a, const PyDataContainer* y, float b)
    {
        PyDataContainer out;
        out.dc = std::make_shared<DC>(x.dc->descriptor());
        if (y && y->dc->getSize() != x.dc->getSize())
            throw elsa_b200::Error(ELSA_ERROR_INVALID_ARGUMENT, "DataContainer: size mismatch");
        lincomb(a, *x.dc, b, y ? *y->dc : *x.dc, *out.dc);
        return out;
    }

    // a projector constructed from (volume, detector) only
    template <class Op>
    void bindProjector(py::module_& m, const char* name, const char* alias)
    {
        py::class_<Op, LinOp, std::shared_ptr<Op>> cls(m, name);
        cls.def(py::init<const VolumeDescriptor&, const PlanarDetectorDescriptor&>(),
                py::arg("domainDescriptor"), py::arg("rangeDescriptor"));
        m.attr(alias) = cls;
    }
} // namespace

PYBIND11_MODULE(_pyelsa, m)
{
    m.doc() = "elsa's pyelsa names on the B200 projector and solver library (pybind11)";
    py::register_exception<elsa_b200::Error>(m, "ElsaError", PyExc_RuntimeError);

    // ---- descriptors (core/Descriptors) ----
    py::class_<DataDescriptor, std::shared_ptr<DataDescriptor>>(m, "DataDescriptor")
        .def("getNumberOfDimensions", &DataDescriptor::getNumberOfDimensions)
        .def("getNumberOfCoefficients", &DataDescriptor::getNumberOfCoefficients)
        .def("getNumberOfCoefficientsPerDimension",
             &DataDescriptor::getNumberOfCoefficientsPerDimension)
        .def("getSpacingPerDimension", &DataDescriptor::getSpacingPerDimension)
        .def_property_readonly("shape", &DataDescriptor::getNumberOfCoefficientsPerDimension);
    py::class_<VolumeDescriptor, DataDescriptor, std::shared_ptr<VolumeDescriptor>>(
        m, "VolumeDescriptor")
        .def(py::init<IndexVector, RealVector>(), py::arg("numberOfCoefficientsPerDimension"),
             py::arg("spacingPerDimension") = RealVector{});
    py::class_<PlanarDetectorDescriptor, DataDescriptor,
               std::shared_ptr<PlanarDetectorDescriptor>>(m, "PlanarDetectorDescriptor")
        .def("getNumberOfGeometryPoses", &PlanarDetectorDescriptor::getNumberOfGeometryPoses)
        .def("poses", &PlanarDetectorDescriptor::poses);
    py::class_<CurvedDetectorDescriptor, PlanarDetectorDescriptor,
               std::shared_ptr<CurvedDetectorDescriptor>>(m, "CurvedDetectorDescriptor")
        .def("getRadius", &CurvedDetectorDescriptor::getRadius)
        .def("getPlanarCoords", &CurvedDetectorDescriptor::getPlanarCoords);

    // ---- trajectories (generators/CircleTrajectoryGenerator.h) ----
    py::class_<CircleTrajectoryGenerator>(m, "CircleTrajectoryGenerator")
        .def_static(
            "createTrajectory",
            [](int64_t numberOfPoses, const DataDescriptor& volume, int64_t arcDegrees,
               float sourceToCenter, float centerToDetector, std::optional<IndexVector> detSize,
               std::optional<RealVector> detSpacing) {
                return std::shared_ptr<PlanarDetectorDescriptor>(
                    CircleTrajectoryGenerator::createTrajectory(numberOfPoses, volume, arcDegrees,
                                                                sourceToCenter, centerToDetector,
                                                                detSize, detSpacing));
            },
            py::arg("numberOfPoses"), py::arg("volumeDescriptor"), py::arg("arcDegrees"),
            py::arg("sourceToCenter"), py::arg("centerToDetector"),
            py::arg("detectorSize") = py::none(), py::arg("detectorSpacing") = py::none());
    py::class_<CurvedCircleTrajectoryGenerator>(m, "CurvedCircleTrajectoryGenerator")
        .def_static(
            "createTrajectory",
            [](int64_t numberOfPoses, const DataDescriptor& volume, int64_t arcDegrees,
               float sourceToCenter, float centerToDetector, float angle,
               std::optional<IndexVector> detSize, std::optional<RealVector> detSpacing) {
                return std::shared_ptr<CurvedDetectorDescriptor>(
                    CurvedCircleTrajectoryGenerator::createTrajectory(
                        numberOfPoses, volume, arcDegrees, sourceToCenter, centerToDetector,
                        angle, detSize, detSpacing));
            },
            py::arg("numberOfPoses"), py::arg("volumeDescriptor"), py::arg("arcDegrees"),
            py::arg("sourceToCenter"), py::arg("centerToDetector"), py::arg("angle"),
            py::arg("detectorSize") = py::none(), py::arg("detectorSpacing") = py::none());

    // ---- DataContainer (core/DataContainer.h), float32 on the device ----
    py::class_<PyDataContainer>(m, "DataContainerf", py::buffer_protocol())
        .def(py::init([](const DataDescriptor& d) { return makeContainer(copyDescriptor(d), {}); }),
             py::arg("dataDescriptor"))
        .def(py::init([](py::array values, const DataDescriptor& d) {
                 return makeContainer(copyDescriptor(d), values);
             }),
             py::arg("values"), py::arg("dataDescriptor"))
        .def_buffer([](PyDataContainer& self) {
            // a fresh read-only host copy, first index fastest (Fortran order)
            self.mirror = self.dc->toHost();
            const auto& n = self.dc->getDataDescriptor().getNumberOfCoefficientsPerDimension();
            std::vector<py::ssize_t> shape(n.begin(), n.end()), strides(n.size());
            py::ssize_t st = sizeof(float);
            for (size_t i = 0; i < n.size(); ++i) {
                strides[i] = st;
                st *= static_cast<py::ssize_t>(n[i]);
            }
            return py::buffer_info(self.mirror.data(), sizeof(float),
                                   py::format_descriptor<float>::format(),
                                   static_cast<py::ssize_t>(n.size()), shape, strides, true);
        })
        .def("getDataDescriptor",
             [](const PyDataContainer& self) { return copyDescriptor(self.dc->getDataDescriptor()); })
        .def("getSize", [](const PyDataContainer& self) { return self.dc->getSize(); })
        .def("dot", [](const PyDataContainer& a, const PyDataContainer& b) {
            return a.dc->dot(*b.dc);
        })
        .def("squaredL2Norm", [](const PyDataContainer& a) { return a.dc->squaredL2Norm(); })
        .def("l2Norm", [](const PyDataContainer& a) { return a.dc->l2Norm(); })
        .def("data_ptr", [](const PyDataContainer& a) {
            return reinterpret_cast<uintptr_t>(a.dc->data());
        })
        .def("__add__", [](const PyDataContainer& a, const PyDataContainer& b) {
            return combine(a, 1.0f, &b, 1.0f);
        })
        .def("__sub__", [](const PyDataContainer& a, const PyDataContainer& b) {
            return combine(a, 1.0f, &b, -1.0f);
        })
        .def("__mul__", [](const PyDataContainer& a, float s) { return combine(a, s, nullptr, 0.0f); })
        .def("__rmul__", [](const PyDataContainer& a, float s) { return combine(a, s, nullptr, 0.0f); })
        .def("__len__", [](const PyDataContainer& a) { return a.dc->getSize(); });
    m.attr("DataContainer") = m.attr("DataContainerf");

    // ---- operators (core/LinearOperator.h, projectors_cuda/*) ----
    py::class_<LinOp, std::shared_ptr<LinOp>>(m, "LinearOperatorf")
        .def("apply", [](const LinOp& A, const PyDataContainer& x) { return wrap(A.apply(*x.dc)); })
        .def("applyAdjoint",
             [](const LinOp& A, const PyDataContainer& y) { return wrap(A.applyAdjoint(*y.dc)); })
        .def("getDomainDescriptor",
             [](const LinOp& A) { return copyDescriptor(A.getDomainDescriptor()); })
        .def("getRangeDescriptor",
             [](const LinOp& A) { return copyDescriptor(A.getRangeDescriptor()); })
        .def("autotune", &LinOp::autotune, py::arg("force") = false)
        .def("getKnob", &LinOp::getKnob)
        .def("setKnob", &LinOp::setKnob);
    m.attr("LinearOperator") = m.attr("LinearOperatorf");

    py::class_<JosephsMethodCUDA<float>, LinOp, std::shared_ptr<JosephsMethodCUDA<float>>>(
        m, "JosephsMethodCUDAf")
        .def(py::init<const VolumeDescriptor&, const PlanarDetectorDescriptor&, bool>(),
             py::arg("domainDescriptor"), py::arg("rangeDescriptor"), py::arg("fast") = false);
    m.attr("JosephsMethodCUDA") = m.attr("JosephsMethodCUDAf");
    bindProjector<JosephsMethod<float>>(m, "JosephsMethodf", "JosephsMethod");
    bindProjector<SiddonsMethodCUDA<float>>(m, "SiddonsMethodCUDAf", "SiddonsMethodCUDA");
    bindProjector<BinaryMethod<float>>(m, "BinaryMethodf", "BinaryMethod");
    py::class_<BlobVoxelProjectorCUDA<float>, LinOp,
               std::shared_ptr<BlobVoxelProjectorCUDA<float>>>(m, "BlobVoxelProjectorCUDAf")
        .def(py::init<const VolumeDescriptor&, const PlanarDetectorDescriptor&, float, float,
                      int>(),
             py::arg("domainDescriptor"), py::arg("rangeDescriptor"), py::arg("radius") = 2.0f,
             py::arg("alpha") = 10.83f, py::arg("order") = 2);
    m.attr("BlobVoxelProjectorCUDA") = m.attr("BlobVoxelProjectorCUDAf");
    py::class_<BSplineVoxelProjectorCUDA<float>, LinOp,
               std::shared_ptr<BSplineVoxelProjectorCUDA<float>>>(m, "BSplineVoxelProjectorCUDAf")
        .def(py::init<const VolumeDescriptor&, const PlanarDetectorDescriptor&, int>(),
             py::arg("domainDescriptor"), py::arg("rangeDescriptor"), py::arg("order") = 2);
    m.attr("BSplineVoxelProjectorCUDA") = m.attr("BSplineVoxelProjectorCUDAf");
    py::class_<PhaseContrastBlobVoxelProjectorCUDA<float>, LinOp,
               std::shared_ptr<PhaseContrastBlobVoxelProjectorCUDA<float>>>(
        m, "PhaseContrastBlobVoxelProjectorCUDAf")
        .def(py::init<const VolumeDescriptor&, const PlanarDetectorDescriptor&, float, float,
                      int>(),
             py::arg("domainDescriptor"), py::arg("rangeDescriptor"), py::arg("radius") = 2.0f,
             py::arg("alpha") = 10.83f, py::arg("order") = 2);
    m.attr("PhaseContrastBlobVoxelProjectorCUDA") = m.attr("PhaseContrastBlobVoxelProjectorCUDAf");
    py::class_<PhaseContrastBSplineVoxelProjectorCUDA<float>, LinOp,
               std::shared_ptr<PhaseContrastBSplineVoxelProjectorCUDA<float>>>(
        m, "PhaseContrastBSplineVoxelProjectorCUDAf")
        .def(py::init<const VolumeDescriptor&, const PlanarDetectorDescriptor&, int>(),
             py::arg("domainDescriptor"), py::arg("rangeDescriptor"), py::arg("order") = 2);
    m.attr("PhaseContrastBSplineVoxelProjectorCUDA") =
        m.attr("PhaseContrastBSplineVoxelProjectorCUDAf");
    py::class_<BlobProjector<float>, LinOp, std::shared_ptr<BlobProjector<float>>>(
        m, "BlobProjectorf")
        .def(py::init<const VolumeDescriptor&, const PlanarDetectorDescriptor&, float, float,
                      int>(),
             py::arg("domainDescriptor"), py::arg("rangeDescriptor"), py::arg("radius") = 2.0f,
             py::arg("alpha") = 10.83f, py::arg("order") = 2);
    m.attr("BlobProjector") = m.attr("BlobProjectorf");
    py::class_<BSplineProjector<float>, LinOp, std::shared_ptr<BSplineProjector<float>>>(
        m, "BSplineProjectorf")
        .def(py::init<const VolumeDescriptor&, const PlanarDetectorDescriptor&, int>(),
             py::arg("domainDescriptor"), py::arg("rangeDescriptor"), py::arg("order") = 2);
    m.attr("BSplineProjector") = m.attr("BSplineProjectorf");

    // ---- proximal operators and solvers (solvers/*) ----
    py::class_<ProximalIdentity>(m, "ProximalIdentityf").def(py::init<>());
    m.attr("ProximalIdentity") = m.attr("ProximalIdentityf");
    py::class_<ProximalBoxConstraint>(m, "ProximalBoxConstraintf")
        .def(py::init([](std::optional<float> lower, std::optional<float> upper) {
                 return ProximalBoxConstraint{lower, upper};
             }),
             py::arg("lower") = py::none(), py::arg("upper") = py::none());
    m.attr("ProximalBoxConstraint") = m.attr("ProximalBoxConstraintf");
    py::class_<ProximalL1>(m, "ProximalL1f")
        .def(py::init([](float sigma) { return ProximalL1{sigma}; }), py::arg("sigma") = 1.0f);
    m.attr("ProximalL1") = m.attr("ProximalL1f");

    // a solver keeps its operator and data alive (keep_alive) and returns device containers
    using Solv = Solver<float>;
    py::class_<Solv, std::shared_ptr<Solv>>(m, "Solverf")
        .def("solve",
             [](Solv& s, int64_t iterations, std::optional<PyDataContainer> x0) {
                 std::optional<DC> init;
                 if (x0)
                     init = *x0->dc;
                 return wrap(s.solve(iterations, init));
             },
             py::arg("iterations"), py::arg("x0") = py::none())
        .def("lastSquaredResidual", &Solv::lastSquaredResidual);
    py::class_<CGNE<float>, Solv, std::shared_ptr<CGNE<float>>>(m, "CGNEf")
        .def(py::init([](const LinOp& A, const PyDataContainer& b) {
                 return std::make_shared<CGNE<float>>(A, *b.dc);
             }),
             py::keep_alive<1, 2>(), py::keep_alive<1, 3>());
    m.attr("CGNE") = m.attr("CGNEf");
    py::class_<CGLS<float>, Solv, std::shared_ptr<CGLS<float>>>(m, "CGLSf")
        .def(py::init([](const LinOp& A, const PyDataContainer& b, float eps, float tol) {
                 return std::make_shared<CGLS<float>>(A, *b.dc, eps, tol);
             }),
             py::arg("operator"), py::arg("b"), py::arg("eps") = 0.0f, py::arg("tol") = 1e-4f,
             py::keep_alive<1, 2>(), py::keep_alive<1, 3>());
    m.attr("CGLS") = m.attr("CGLSf");
    py::class_<Landweber<float>, Solv, std::shared_ptr<Landweber<float>>>(m, "Landweberf")
        .def(py::init([](const LinOp& A, const PyDataContainer& b, std::optional<float> step) {
                 return step ? std::make_shared<Landweber<float>>(A, *b.dc, *step)
                             : std::make_shared<Landweber<float>>(A, *b.dc);
             }),
             py::arg("operator"), py::arg("b"), py::arg("stepSize") = py::none(),
             py::keep_alive<1, 2>(), py::keep_alive<1, 3>());
    m.attr("Landweber") = m.attr("Landweberf");
    py::class_<APGD<float>, Solv, std::shared_ptr<APGD<float>>>(m, "APGDf")
        .def(py::init([](const LinOp& A, const PyDataContainer& b, py::object prox,
                         std::optional<float> mu, float epsilon) {
                 if (py::isinstance<ProximalBoxConstraint>(prox))
                     return std::make_shared<APGD<float>>(A, *b.dc,
                                                          prox.cast<ProximalBoxConstraint>(), mu,
                                                          epsilon);
                 if (py::isinstance<ProximalL1>(prox))
                     return std::make_shared<APGD<float>>(A, *b.dc, prox.cast<ProximalL1>(), mu,
                                                          epsilon);
                 return std::make_shared<APGD<float>>(A, *b.dc, ProximalIdentity{}, mu, epsilon);
             }),
             py::arg("operator"), py::arg("b"), py::arg("prox") = py::none(),
             py::arg("mu") = py::none(), py::arg("epsilon") = 1.1920928955078125e-07f,
             py::keep_alive<1, 2>(), py::keep_alive<1, 3>());
    m.attr("APGD") = m.attr("APGDf");
    m.attr("FISTA") = m.attr("APGDf");
    py::class_<SIRT<float>, Solv, std::shared_ptr<SIRT<float>>>(m, "SIRTf")
        .def(py::init([](const LinOp& A, const PyDataContainer& b, std::optional<float> step) {
                 return std::make_shared<SIRT<float>>(A, *b.dc, step);
             }),
             py::arg("operator"), py::arg("b"), py::arg("stepSize") = py::none(),
             py::keep_alive<1, 2>(), py::keep_alive<1, 3>());
    m.attr("SIRT") = m.attr("SIRTf");
    // problems/LeastSquares.h with FGM, OGM and SQS on it
    struct PyLeastSquares {
        std::shared_ptr<LinOp> A;
        PyDataContainer b;
    };
    py::class_<PyLeastSquares>(m, "LeastSquaresf")
        .def(py::init([](std::shared_ptr<LinOp> A, const PyDataContainer& b) {
            return PyLeastSquares{std::move(A), b};
        }));
    m.attr("LeastSquares") = m.attr("LeastSquaresf");
    py::class_<FGM<float>, Solv, std::shared_ptr<FGM<float>>>(m, "FGMf")
        .def(py::init([](const PyLeastSquares& p, float epsilon) {
                 return std::make_shared<FGM<float>>(LeastSquares<float>{*p.A, *p.b.dc}, epsilon);
             }),
             py::arg("problem"), py::arg("epsilon") = 1.1920928955078125e-07f,
             py::keep_alive<1, 2>());
    m.attr("FGM") = m.attr("FGMf");
    py::class_<OGM<float>, Solv, std::shared_ptr<OGM<float>>>(m, "OGMf")
        .def(py::init([](const PyLeastSquares& p, float epsilon) {
                 return std::make_shared<OGM<float>>(LeastSquares<float>{*p.A, *p.b.dc}, epsilon);
             }),
             py::arg("problem"), py::arg("epsilon") = 1.1920928955078125e-07f,
             py::keep_alive<1, 2>());
    m.attr("OGM") = m.attr("OGMf");
    py::class_<SQS<float>, Solv, std::shared_ptr<SQS<float>>>(m, "SQSf")
        .def(py::init([](const PyLeastSquares& p, bool momentum, float epsilon) {
                 return std::make_shared<SQS<float>>(LeastSquares<float>{*p.A, *p.b.dc}, momentum,
                                                     epsilon);
             }),
             py::arg("problem"), py::arg("momentumAcceleration") = true,
             py::arg("epsilon") = 1.1920928955078125e-07f, py::keep_alive<1, 2>());
    m.attr("SQS") = m.attr("SQSf");
}
