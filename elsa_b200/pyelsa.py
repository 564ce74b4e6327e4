"""pyelsa-style Python API over the elsa_b200 C ABI.

The names, arguments and defaults follow elsa's Python bindings (pyelsa/pyelsa/bind_core.cpp,
bind_generators.cpp, bind_projectors_cuda.cpp, bind_solvers.cpp, bind_proximal_operators.cpp), so
that a pyelsa script runs with ``import elsa_b200.pyelsa as elsa``:

    vol = elsa.VolumeDescriptor([256, 256, 256])
    sino = elsa.CircleTrajectoryGenerator.createTrajectory(360, vol, 360, 2560, 640,
                                                           detectorSize=[384, 384])
    A = elsa.JosephsMethodCUDA(vol, sino)
    b = A.apply(phantom)                       # numpy (F-order, x fastest) or DataContainer
    x = elsa.CGNE(A, b).solve(30)
    np.asarray(x)                              # back to numpy, shape (256, 256, 256)

Arrays follow elsa's layout: the first index is x (fastest), i.e. Fortran order, as pyelsa's
buffer protocol does. Data lives on the GPU (torch tensors on cuda:0); every projector and solver
call runs the native CUDA kernels. The float64 instantiations (…CUDAd) are not provided: the
device path computes in float32 with float64 inner products.
"""
import math

import numpy as np

from . import _capi


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("elsa_b200.pyelsa needs a CUDA device")
    return torch


# ---- descriptors (core/Descriptors) ----------------------------------------------------------------

class DataDescriptor:
    """Shape and spacing of a data container (core/Descriptors/DataDescriptor.h)."""

    def __init__(self, size, spacing=None):
        self._size = np.asarray(size, np.int64).ravel()
        if self._size.size < 1 or np.any(self._size <= 0):
            raise _capi.InvalidArgumentError(1, "DataDescriptor: invalid size")
        sp = np.ones(self._size.size) if spacing is None else np.asarray(spacing, np.float64)
        if sp.size != self._size.size or np.any(sp <= 0):
            raise _capi.InvalidArgumentError(1, "DataDescriptor: invalid spacing")
        self._spacing = sp.astype(np.float32)

    def getNumberOfDimensions(self):
        return int(self._size.size)

    def getNumberOfCoefficients(self):
        return int(np.prod(self._size))

    def getNumberOfCoefficientsPerDimension(self):
        return self._size.copy()

    def getSpacingPerDimension(self):
        return self._spacing.astype(np.float64)

    def getLocationOfOrigin(self):
        # 0.5 * (size * spacing), DataDescriptor.cpp:21,49
        return (0.5 * (self._size.astype(np.float32) * self._spacing)).astype(np.float64)

    @property
    def shape(self):
        return tuple(int(v) for v in self._size)

    def __eq__(self, other):
        return (isinstance(other, DataDescriptor) and np.array_equal(self._size, other._size)
                and np.array_equal(self._spacing, other._spacing))


class VolumeDescriptor(DataDescriptor):
    """core/Descriptors/VolumeDescriptor.h"""


class PlanarDetectorDescriptor(DataDescriptor):
    """Flat-panel detector with one geometry (pose record) per projection
    (core/Descriptors/PlanarDetectorDescriptor.h). The last dimension counts the poses."""

    def __init__(self, size, poses, spacing=None):
        super().__init__(size, spacing)
        self.poses = np.ascontiguousarray(poses, np.float32).reshape(-1, _capi.POSE_FLOATS)
        if self.poses.shape[0] != self._size[-1]:
            raise _capi.InvalidArgumentError(1, "PlanarDetectorDescriptor: poses != last dim")

    def getNumberOfGeometryPoses(self):
        return int(self.poses.shape[0])


class CurvedDetectorDescriptor(PlanarDetectorDescriptor):
    """Cylindrical detector (core/Descriptors/CurvedDetectorDescriptor.h): the poses of a flat
    detector plus the opening angle (radian) and the source-to-detector distance."""

    def __init__(self, size, poses, angle, s2d, spacing=None):
        super().__init__(size, poses, spacing)
        self.angle = float(angle)
        self.s2d = float(s2d)

    def getPlanarCoords(self):
        dim = self.getNumberOfDimensions()
        nv = int(self._size[1]) if dim == 3 else 1
        c = _capi.curved_detector_coords(dim, int(self._size[0]), nv, self.angle, self.s2d)
        return [c[v, u, :dim - 1].astype(np.float64) for v in range(c.shape[0])
                for u in range(c.shape[1])]

    def getRadius(self):
        return float(np.float32(np.float32(self._size[0]) / np.float32(self.angle)))


class CircleTrajectoryGenerator:
    """generators/CircleTrajectoryGenerator.cpp:9-24."""

    @staticmethod
    def createTrajectory(numberOfPoses, volumeDescriptor, arcDegrees, sourceToCenter,
                         centerToDetector, principalPointOffset=None, centerOfRotOffset=None,
                         detectorSize=None, detectorSpacing=None):
        if principalPointOffset is not None or centerOfRotOffset is not None:
            raise NotImplementedError("createTrajectory: principal point / centre of rotation "
                                      "offsets are not supported; build poses with pose_2d / "
                                      "pose_3d instead")
        vol = volumeDescriptor
        poses, det = _capi.circle_trajectory(vol.shape, int(numberOfPoses), float(arcDegrees),
                                             float(sourceToCenter), float(centerToDetector),
                                             detectorSize, vol.getSpacingPerDimension(),
                                             detectorSpacing)
        dim = vol.getNumberOfDimensions()
        spacing = list(detectorSpacing) if detectorSpacing is not None else \
            list(vol.getSpacingPerDimension()[:dim - 1])
        return PlanarDetectorDescriptor(det, poses, spacing + [1.0])


class CurvedCircleTrajectoryGenerator:
    """generators/CurvedCircleTrajectoryGenerator.cpp:8-30: the circle trajectory's poses with a
    curved detector of opening angle `angle` (radian) at source-to-detector distance
    sourceToCenter + centerToDetector."""

    @staticmethod
    def createTrajectory(numberOfPoses, volumeDescriptor, arcDegrees, sourceToCenter,
                         centerToDetector, angle, principalPointOffset=None,
                         centerOfRotOffset=None, detectorSize=None, detectorSpacing=None):
        flat = CircleTrajectoryGenerator.createTrajectory(
            numberOfPoses, volumeDescriptor, arcDegrees, sourceToCenter, centerToDetector,
            principalPointOffset, centerOfRotOffset, detectorSize, detectorSpacing)
        s2d = float(np.float32(np.float32(sourceToCenter) + np.float32(centerToDetector)))
        return CurvedDetectorDescriptor(flat.shape, flat.poses, angle, s2d,
                                        list(flat.getSpacingPerDimension()))


# ---- DataContainer ---------------------------------------------------------------------------------

class DataContainer:
    """A float32 device buffer with a descriptor (core/DataContainer.h). Built from a numpy array
    (x fastest: Fortran order for an array of shape (nx, ny[, nz])) or a flat torch tensor."""

    def __init__(self, data, descriptor=None):
        torch = _torch()
        if isinstance(data, DataContainer):
            descriptor = descriptor or data.descriptor
            self.tensor = data.tensor.clone()
        elif isinstance(data, torch.Tensor):
            t = data.detach().to(device="cuda", dtype=torch.float32).contiguous().reshape(-1)
            self.tensor = t
            if descriptor is None:
                raise _capi.InvalidArgumentError(1, "DataContainer: a tensor needs a descriptor")
        else:
            arr = np.asarray(data, dtype=np.float32)
            if descriptor is None:
                descriptor = DataDescriptor(arr.shape)
            flat = np.ascontiguousarray(arr.reshape(-1, order="F") if arr.ndim > 1 else
                                        arr.reshape(-1))
            self.tensor = torch.from_numpy(flat).cuda()
        if self.tensor.numel() != descriptor.getNumberOfCoefficients():
            raise _capi.InvalidArgumentError(1, "DataContainer: size does not match descriptor")
        self.descriptor = descriptor

    @classmethod
    def zeros(cls, descriptor):
        torch = _torch()
        obj = cls.__new__(cls)
        obj.tensor = torch.zeros(descriptor.getNumberOfCoefficients(), dtype=torch.float32,
                                 device="cuda")
        obj.descriptor = descriptor
        return obj

    def getDataDescriptor(self):
        return self.descriptor

    def getSize(self):
        return self.tensor.numel()

    def __array__(self, dtype=None, copy=None):
        arr = self.tensor.cpu().numpy().reshape(self.descriptor.shape, order="F")
        return arr.astype(dtype) if dtype is not None else arr

    def _ptr(self):
        return self.tensor.data_ptr()

    def _stream(self):
        return _torch().cuda.current_stream().cuda_stream

    def dot(self, other):
        """<self, other> with float64 accumulation (elsa_dot)."""
        import ctypes
        torch = _torch()
        o = _as_dc(other, self.descriptor)
        res = torch.empty(1, dtype=torch.float64, device="cuda")
        _capi.call("elsa_dot", ctypes.c_void_p(self._ptr()), ctypes.c_void_p(o._ptr()),
                   self.getSize(), ctypes.c_void_p(res.data_ptr()),
                   ctypes.c_void_p(self._stream()))
        return float(res.item())

    def squaredL2Norm(self):
        import ctypes
        torch = _torch()
        res = torch.empty(1, dtype=torch.float64, device="cuda")
        _capi.call("elsa_squared_l2_norm", ctypes.c_void_p(self._ptr()), self.getSize(),
                   ctypes.c_void_p(res.data_ptr()), ctypes.c_void_p(self._stream()))
        return float(res.item())

    def l2Norm(self):
        return math.sqrt(self.squaredL2Norm())

    def _lincomb(self, a, other, b):
        """a * self + b * other (elsa_lincomb, core/DataContainer.cpp:1075-1108)."""
        import ctypes
        o = _as_dc(other, self.descriptor) if other is not None else self
        out = DataContainer.zeros(self.descriptor)
        _capi.call("elsa_lincomb", ctypes.c_float(a), ctypes.c_void_p(self._ptr()),
                   ctypes.c_float(b), ctypes.c_void_p(o._ptr()), ctypes.c_void_p(out._ptr()),
                   self.getSize(), ctypes.c_void_p(self._stream()))
        return out

    def __add__(self, other):
        return self._lincomb(1.0, other, 1.0)

    def __sub__(self, other):
        return self._lincomb(1.0, other, -1.0)

    def __mul__(self, other):
        if isinstance(other, (int, float, np.floating)):
            return self._lincomb(float(other), None, 0.0)
        # element-wise product: a convenience outside the projector / solver path
        obj = DataContainer.__new__(DataContainer)
        obj.tensor = self.tensor * _as_dc(other, self.descriptor).tensor
        obj.descriptor = self.descriptor
        return obj

    __rmul__ = __mul__


def _as_dc(x, descriptor):
    if isinstance(x, DataContainer):
        if x.getSize() != descriptor.getNumberOfCoefficients():
            raise _capi.InvalidArgumentError(1, "size does not match the operator")
        return x
    return DataContainer(x, descriptor)


# ---- operators (core/LinearOperator.h, projectors_cuda/*) -------------------------------------------

class LinearOperator:
    """Base of the projectors: apply / applyAdjoint on DataContainers or numpy arrays."""

    def __init__(self, kind, volumeDescriptor, detectorDescriptor, params=None):
        if volumeDescriptor.getNumberOfDimensions() != \
                detectorDescriptor.getNumberOfDimensions():
            raise _capi.InvalidArgumentError(1, "domain and range dimension need to match")
        if not isinstance(detectorDescriptor, PlanarDetectorDescriptor):
            raise _capi.InvalidArgumentError(1, "range descriptor needs a geometry")
        self._domain = volumeDescriptor
        self._range = detectorDescriptor
        curved = None
        if isinstance(detectorDescriptor, CurvedDetectorDescriptor):
            curved = (detectorDescriptor.angle, detectorDescriptor.s2d)
        self._op = _capi.Projector(kind, volumeDescriptor.shape, detectorDescriptor.shape,
                                   detectorDescriptor.poses, params, curved)

    def getDomainDescriptor(self):
        return self._domain

    def getRangeDescriptor(self):
        return self._range

    @property
    def native(self):
        """The underlying elsa_b200.Projector (C ABI handle)."""
        return self._op

    def _stream(self):
        return _torch().cuda.current_stream().cuda_stream

    def apply(self, x, Ax=None):
        x = _as_dc(x, self._domain)
        out = Ax if Ax is not None else DataContainer.zeros(self._range)
        self._op.apply_ptr(x._ptr(), _as_dc(out, self._range)._ptr(), self._stream())
        return out

    def applyAdjoint(self, y, Aty=None):
        y = _as_dc(y, self._range)
        out = Aty if Aty is not None else DataContainer.zeros(self._domain)
        self._op.apply_adjoint_ptr(y._ptr(), _as_dc(out, self._domain)._ptr(), self._stream())
        return out


class JosephsMethodCUDA(LinearOperator):
    """JosephsMethodCUDA(volume, detector, fast=False). fast=False: the matched, deterministic
    adjoint (the transpose of the forward, as elsa's CPU JosephsMethod). fast=True: elsa's
    `fast` adjoint, a voxel-driven backprojection through a texture that is not the transpose
    (JosephsMethodCUDA.h:60-67). elsa's own default is fast=True; here the matched adjoint is the
    default, since the solvers assume a transpose."""

    def __init__(self, volumeDescriptor, detectorDescriptor, fast=False):
        super().__init__(_capi.PROJECTOR_JOSEPH, volumeDescriptor, detectorDescriptor,
                         [1.0] if fast else [])


class JosephsMethod(LinearOperator):
    """JosephsMethod(volume, detector): elsa's CPU Joseph projector (matched adjoint), on the
    device."""

    def __init__(self, volumeDescriptor, detectorDescriptor):
        super().__init__(_capi.PROJECTOR_JOSEPH, volumeDescriptor, detectorDescriptor)


class SiddonsMethodCUDA(LinearOperator):
    def __init__(self, volumeDescriptor, detectorDescriptor):
        super().__init__(_capi.PROJECTOR_SIDDON, volumeDescriptor, detectorDescriptor)


class BinaryMethod(LinearOperator):
    """BinaryMethod(volume, detector) (projectors/BinaryMethod.h): the voxels a ray visits, each
    with weight 1, on the device (the Siddon traversal kernels)."""

    def __init__(self, volumeDescriptor, detectorDescriptor):
        super().__init__(_capi.PROJECTOR_BINARY, volumeDescriptor, detectorDescriptor)


class BlobProjector(LinearOperator):
    """BlobProjector(volume, detector, radius=2, alpha=10.83, order=2): elsa's ray-driven blob
    projector (projectors/LutProjector.h), on the device."""

    def __init__(self, volumeDescriptor, detectorDescriptor, radius=2.0, alpha=10.83, order=2):
        super().__init__(_capi.PROJECTOR_RAY_BLOB, volumeDescriptor, detectorDescriptor,
                         [radius, alpha, order])


class BSplineProjector(LinearOperator):
    """BSplineProjector(volume, detector, order=2): elsa's ray-driven B-spline projector."""

    def __init__(self, volumeDescriptor, detectorDescriptor, order=2):
        super().__init__(_capi.PROJECTOR_RAY_BSPLINE, volumeDescriptor, detectorDescriptor,
                         [order])


class BlobVoxelProjectorCUDA(LinearOperator):
    def __init__(self, volumeDescriptor, detectorDescriptor, radius=2.0, alpha=10.83, order=2,
                 footprint=_capi.FOOTPRINT_REFERENCE):
        super().__init__(_capi.PROJECTOR_BLOB, volumeDescriptor, detectorDescriptor,
                         [radius, alpha, order, footprint])


class BSplineVoxelProjectorCUDA(LinearOperator):
    def __init__(self, volumeDescriptor, detectorDescriptor, order=2,
                 footprint=_capi.FOOTPRINT_REFERENCE):
        super().__init__(_capi.PROJECTOR_BSPLINE, volumeDescriptor, detectorDescriptor,
                         [order, footprint])


class PhaseContrastBlobVoxelProjectorCUDA(LinearOperator):
    def __init__(self, volumeDescriptor, detectorDescriptor, radius=2.0, alpha=10.83, order=2,
                 footprint=_capi.FOOTPRINT_REFERENCE):
        super().__init__(_capi.PROJECTOR_PHASE_CONTRAST_BLOB, volumeDescriptor,
                         detectorDescriptor, [radius, alpha, order, footprint])


class PhaseContrastBSplineVoxelProjectorCUDA(LinearOperator):
    def __init__(self, volumeDescriptor, detectorDescriptor, order=2,
                 footprint=_capi.FOOTPRINT_REFERENCE):
        super().__init__(_capi.PROJECTOR_PHASE_CONTRAST_BSPLINE, volumeDescriptor,
                         detectorDescriptor, [order, footprint])


# pyelsa aliases: the names without the CUDA suffix (CPU projectors in elsa) and the f-suffixed
# float instantiations resolve to the same device operators
JosephsMethodCUDAf = JosephsMethodCUDA
JosephsMethodf = JosephsMethod
SiddonsMethod = SiddonsMethodCUDAf = SiddonsMethodCUDA
BinaryMethodf = BinaryMethod
BlobProjectorf, BSplineProjectorf = BlobProjector, BSplineProjector
BlobVoxelProjector = BlobVoxelProjectorCUDAf = BlobVoxelProjectorCUDA
BSplineVoxelProjector = BSplineVoxelProjectorCUDAf = BSplineVoxelProjectorCUDA
PhaseContrastBlobVoxelProjector = PhaseContrastBlobVoxelProjectorCUDA
PhaseContrastBSplineVoxelProjector = PhaseContrastBSplineVoxelProjectorCUDA


# ---- proximal operators (proximal_operators/*) ------------------------------------------------------

class ProximalIdentity:
    params = (0.0, float("nan"), float("nan"), 1.0)


class ProximalBoxConstraint:
    def __init__(self, lower=None, upper=None):
        self.params = (1.0, float("nan") if lower is None else float(lower),
                       float("nan") if upper is None else float(upper), 1.0)


class ProximalL1:
    def __init__(self, sigma=1.0):
        self.params = (2.0, float("nan"), float("nan"), float(sigma))


# ---- solvers (solvers/*, bindings in pyelsa/pyelsa/bind_solvers.cpp) --------------------------------

class _Solver:
    _kind = None

    def __init__(self, A, b):
        self.A = A
        self.b = _as_dc(b, A.getRangeDescriptor())
        self.last = None  # the native session of the last solve (residual, timing)

    def _params(self):
        return ()

    def solve(self, iterations, x0=None):
        x = DataContainer.zeros(self.A.getDomainDescriptor()) if x0 is None else \
            DataContainer(_as_dc(x0, self.A.getDomainDescriptor()))
        s = self.A._stream()
        self.last = _capi.Solver(self._kind, self.A.native, self.b._ptr(), x._ptr(),
                                 use_x0=x0 is not None, stream=s, params=self._params())
        self.last.iterate(int(iterations), s)
        return x


class CGNE(_Solver):
    _kind = _capi.SOLVER_CGNE


class CGLS(_Solver):
    _kind = _capi.SOLVER_CGLS

    def __init__(self, A, b, eps=0.0, tol=1e-4):
        super().__init__(A, b)
        self.eps, self.tol = float(eps), float(tol)

    def _params(self):
        return (self.eps, self.tol)


class Landweber(_Solver):
    _kind = _capi.SOLVER_LANDWEBER

    def __init__(self, A, b, stepSize=None):
        super().__init__(A, b)
        self.stepSize = stepSize

    def _params(self):
        return (float(self.stepSize),) if self.stepSize is not None else ()


class APGD(_Solver):
    """APGD(A, b, prox, mu=None, eps=1e-6) (pyelsa's defaults, bind_solvers.cpp:222-228)."""
    _kind = _capi.SOLVER_APGD

    def __init__(self, A, b, prox=None, mu=None, eps=1e-6):
        super().__init__(A, b)
        self.prox = prox if prox is not None else ProximalIdentity()
        self.mu, self.eps = mu, float(eps)

    def _params(self):
        kind, lo, hi, sigma = self.prox.params
        return (float(self.mu) if self.mu is not None else 0.0, self.eps, kind, lo, hi, sigma)


FISTA = APGD


class SIRT(Landweber):
    """SIRT(A, b, stepSize=None) (solvers/SIRT.cpp)."""
    _kind = _capi.SOLVER_SIRT


class LeastSquares:
    """The functional 0.5 |A x - b|^2 (functionals/LeastSquares.h), the problem FGM / OGM solve."""

    def __init__(self, A, b):
        self.A = A
        self.b = b


class _MomentumSolver(_Solver):
    def __init__(self, problem, epsilon=1.1920928955078125e-07):
        super().__init__(problem.A, problem.b)
        self.epsilon = float(epsilon)

    def _params(self):
        return (self.epsilon,)


class FGM(_MomentumSolver):
    """FGM(LeastSquares(A, b), epsilon) (solvers/FGM.cpp)."""
    _kind = _capi.SOLVER_FGM


class OGM(_MomentumSolver):
    """OGM(LeastSquares(A, b), epsilon) (solvers/OGM.cpp); solve(n) applies OGM's final-step
    factor on iteration n."""
    _kind = _capi.SOLVER_OGM


class Scaling:
    """Diagonal operator (core/LinearOperators/Scaling.h), here as an SQS preconditioner:
    Scaling(descriptor, factors) with a DataContainer or an array of factors."""

    def __init__(self, descriptor, factors):
        self.descriptor = descriptor
        self.factors = _as_dc(factors, descriptor)

    def getScaleFactors(self):
        return self.factors


class SQS:
    """SQS on LeastSquares(A, b) (solvers/SQS.h:29-69) with elsa's constructor forms:
    SQS(problem[, subsets][, preconditioner], momentumAcceleration=True, epsilon=FLT_EPSILON).
    subsets: a list of LeastSquares problems, one per ordered subset (e.g. from a
    SubsetSampler); preconditioner: a Scaling (or a DataContainer / array of its diagonal)."""

    def __init__(self, problem, *args, momentumAcceleration=True,
                 epsilon=1.1920928955078125e-07):
        args = list(args)
        self.subsets = args.pop(0) if args and isinstance(args[0], (list, tuple)) else []
        self.preconditioner = None
        if args and not isinstance(args[0], (bool, float, int)):
            self.preconditioner = args.pop(0)
        if args:
            momentumAcceleration = bool(args.pop(0))
        if args:
            epsilon = float(args.pop(0))
        if args:
            raise TypeError("SQS: too many arguments")
        self.problem = problem
        self.momentum = bool(momentumAcceleration)
        self.epsilon = float(epsilon)
        self.last = None

    def solve(self, iterations, x0=None):
        A = self.problem.A
        b = _as_dc(self.problem.b, A.getRangeDescriptor())
        x = DataContainer.zeros(A.getDomainDescriptor()) if x0 is None else \
            DataContainer(_as_dc(x0, A.getDomainDescriptor()))
        subs = []
        self._keep = [b]
        for sp in self.subsets:
            bm = _as_dc(sp.b, sp.A.getRangeDescriptor())
            self._keep.append(bm)
            subs.append((sp.A.native, bm._ptr()))
        p = self.preconditioner
        pdc = None
        if p is not None:
            pdc = p.getScaleFactors() if isinstance(p, Scaling) else \
                _as_dc(p, A.getDomainDescriptor())
            self._keep.append(pdc)
        s = A._stream()
        self.last = _capi.Solver.sqs(A.native, b._ptr(), x._ptr(), subsets=subs,
                                     use_x0=x0 is not None, momentum=self.momentum,
                                     epsilon=self.epsilon,
                                     preconditioner_ptr=pdc._ptr() if pdc is not None else None,
                                     stream=s)
        self.last.iterate(int(iterations), s)
        return x


class SubsetSampler:
    """SubsetSampler<PlanarDetectorDescriptor, float> (projectors/SubsetSampler.h:22-129):
    ordered subsets of the poses of a detector descriptor. getPartitionedData returns one
    DataContainer per subset (the blocks of the reference's PartitionDescriptor)."""

    ROUND_ROBIN = _capi.SUBSET_ROUND_ROBIN
    ROTATIONAL_CLUSTERING = _capi.SUBSET_ROTATIONAL_CLUSTERING

    def __init__(self, volumeDescriptor, detectorDescriptor, nSubsets,
                 samplingStrategy=ROUND_ROBIN):
        if int(nSubsets) <= 1:
            raise _capi.InvalidArgumentError(1, "SubsetSampler: nSubsets must be >= 2")
        self._volume = volumeDescriptor
        self._full = detectorDescriptor
        self._n = int(nSubsets)
        dim = detectorDescriptor.getNumberOfDimensions()
        self._mapping = _capi.subset_split(dim, detectorDescriptor.poses, self._n,
                                           samplingStrategy)
        size = list(detectorDescriptor.getNumberOfCoefficientsPerDimension())
        spacing = list(detectorDescriptor.getSpacingPerDimension())
        self._detectors = [PlanarDetectorDescriptor(size[:-1] + [len(idx)],
                                                    detectorDescriptor.poses[idx], spacing)
                           for idx in self._mapping]

    @staticmethod
    def splitRoundRobin(indices, nSubsets):
        """Subset i takes positions i, i + n, ... of indices (SubsetSampler.cpp:56-69)."""
        out = [[] for _ in range(int(nSubsets))]
        for i, v in enumerate(indices):
            out[i % int(nSubsets)].append(int(v))
        return out

    @staticmethod
    def splitRotationalClustering(detectorDescriptor, nSubsets):
        """SubsetSampler.cpp:71-103, through elsa_subset_split."""
        return _capi.subset_split(detectorDescriptor.getNumberOfDimensions(),
                                  detectorDescriptor.poses, int(nSubsets),
                                  _capi.SUBSET_ROTATIONAL_CLUSTERING)

    def getIndexMapping(self):
        return [list(m) for m in self._mapping]

    def getSubsetDetectorDescriptors(self):
        return list(self._detectors)

    def getPartitionedData(self, sinogram):
        sino = _as_dc(sinogram, self._full)
        view = int(np.prod(self._full.getNumberOfCoefficientsPerDimension()[:-1]))
        out = []
        for idx, d in zip(self._mapping, self._detectors):
            block = DataContainer.zeros(d)
            _capi.gather_views(sino._ptr(), view, idx, self._full.getNumberOfGeometryPoses(),
                               block._ptr(), sino._stream())
            out.append(block)
        return out

    def getProjector(self, projectorClass):
        return projectorClass(self._volume, self._full)

    def getSubsetProjectors(self, projectorClass):
        return [projectorClass(self._volume, d) for d in self._detectors]


# ---- image files (io/, bindings in pyelsa/pyelsa/bind_io.cpp + hints/io_hints.cpp) ---------------

def _host_flat(data):
    dc = data if isinstance(data, DataContainer) else None
    if dc is not None:
        return dc.tensor.detach().cpu().numpy(), dc.descriptor
    arr = np.asarray(data, np.float32)
    return arr.reshape(-1, order="F"), DataDescriptor(arr.shape)


def _to_container(flat, dims, spacing):
    torch = _torch()
    dc = DataContainer.__new__(DataContainer)
    dc.tensor = torch.from_numpy(np.ascontiguousarray(flat, np.float32)).cuda()
    dc.descriptor = VolumeDescriptor(dims, spacing)
    return dc


class EDF:
    """EDF.readf(filename) -> DataContainer, EDF.write(data, filename) (io/EDFHandler.h)."""

    @staticmethod
    def readf(filename):
        flat, dims, spacing, _ = _capi.edf_read(filename)
        return _to_container(flat, dims, spacing)

    @staticmethod
    def write(data, filename):
        flat, desc = _host_flat(data)
        _capi.edf_write(filename, flat, desc.getNumberOfCoefficientsPerDimension(),
                        desc.getSpacingPerDimension())


class MHD:
    """MHD.readf(filename) -> DataContainer, MHD.write(data, metaFilename, rawFilename)
    (io/MHDHandler.h)."""

    @staticmethod
    def readf(filename):
        flat, dims, spacing, _ = _capi.mhd_read(filename)
        return _to_container(flat, dims, spacing)

    @staticmethod
    def write(data, metaFilename, rawFilename):
        flat, desc = _host_flat(data)
        _capi.mhd_write(metaFilename, rawFilename, flat,
                        desc.getNumberOfCoefficientsPerDimension(),
                        desc.getSpacingPerDimension())


class PGM:
    """PGM.write(data, filename) (io/PGMHandler.h)."""

    @staticmethod
    def write(data, filename):
        flat, desc = _host_flat(data)
        _capi.pgm_write(filename, flat, desc.getNumberOfCoefficientsPerDimension())


CGNEf, CGLSf, Landweberf, APGDf = CGNE, CGLS, Landweber, APGD
SIRTf, FGMf, OGMf, SQSf = SIRT, FGM, OGM, SQS


def powerIterations(op, niters=5):
    """Largest eigenvalue of op^T op (solvers/PowerIterations.cpp:10-27, applied to
    adjoint(A) * A as elsa's solvers do)."""
    return _capi.power_iterations(op.native, niters, op._stream())
