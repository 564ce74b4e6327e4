"""elsa_b200._pyelsa, the pybind11 module with pyelsa's names over the C++ layer
(include/elsa_b200.hpp): names and descriptors on the CPU; on the GPU the projectors against the
oracle (Fortran-order arrays, first index x), the buffer protocol, and solver results equal to
the ctypes module's (elsa_b200.pyelsa) bit for bit."""
import numpy as np
import pytest

from conftest import rel_l2


def test_module_names_and_descriptors():
    from elsa_b200 import _pyelsa as m
    for name in ("VolumeDescriptor", "CircleTrajectoryGenerator", "DataContainer",
                 "JosephsMethodCUDA", "JosephsMethodCUDAf", "SiddonsMethodCUDA",
                 "BlobVoxelProjectorCUDA", "BSplineVoxelProjectorCUDA",
                 "PhaseContrastBlobVoxelProjectorCUDA", "PhaseContrastBSplineVoxelProjectorCUDA",
                 "BinaryMethod", "BlobProjector", "BSplineProjector", "CGNE", "CGLS", "Landweber",
                 "APGD", "FISTA", "SIRT", "LeastSquares", "FGM", "OGM", "SQS", "ProximalL1",
                 "ProximalBoxConstraint"):
        assert hasattr(m, name), name
    v = m.VolumeDescriptor([12, 10, 8], [1.0, 1.0, 2.0])
    assert v.getNumberOfCoefficientsPerDimension() == [12, 10, 8]
    assert v.getNumberOfCoefficients() == 960
    assert v.getSpacingPerDimension() == [1.0, 1.0, 2.0]
    with pytest.raises(m.ElsaError):
        m.VolumeDescriptor([4, 0])


@pytest.mark.gpu
def test_native_projectors_against_oracle(cuda, oracle):
    from elsa_b200 import _pyelsa as m
    n, views = 24, 16
    vol = m.VolumeDescriptor([n, n, n])
    sino = m.CircleTrajectoryGenerator.createTrajectory(views, vol, 360, 10.0 * n, 2.5 * n,
                                                        [36, 36])
    assert sino.getNumberOfCoefficientsPerDimension() == [36, 36, views]
    poses = np.asarray(sino.poses(), np.float32).reshape(views, 40)
    dd = np.array([36, 36, views])
    rng = np.random.default_rng(4)
    x = rng.uniform(0, 1, (n, n, n)).astype(np.float32)  # indexed [x, y, z]
    y = rng.uniform(0, 1, (36, 36, views)).astype(np.float32)
    xf = x.reshape(-1, order="F")  # x fastest
    yf = y.reshape(-1, order="F")
    lut, support, wk = oracle.voxel_lut("blob", 3)
    cases = [
        (m.JosephsMethodCUDA(vol, sino), oracle.joseph(xf, (n, n, n), dd, poses),
         oracle.joseph_adjoint(yf, (n, n, n), dd, poses)),
        (m.SiddonsMethodCUDA(vol, sino), oracle.siddon(xf, (n, n, n), dd, poses),
         oracle.siddon_adjoint(yf, (n, n, n), dd, poses)),
        (m.BlobVoxelProjectorCUDA(vol, sino),
         oracle.voxel_project(False, xf, (n, n, n), dd, poses, lut, support, wk, 0),
         oracle.voxel_project(True, yf, (n, n, n), dd, poses, lut, support, wk, 0)),
    ]
    xd = m.DataContainer(x, vol)
    yd = m.DataContainer(y, sino)
    assert np.array_equal(np.asarray(xd), x)  # buffer protocol: Fortran-order host copy
    for A, ref_f, ref_a in cases:
        Ax = np.asarray(A.apply(xd))
        Aty = np.asarray(A.applyAdjoint(yd))
        assert Ax.shape == (36, 36, views) and Aty.shape == (n, n, n)
        assert rel_l2(Ax.reshape(-1, order="F"), ref_f) <= 1e-5
        assert rel_l2(Aty.reshape(-1, order="F"), ref_a) <= 1e-5


@pytest.mark.gpu
def test_native_solvers_equal_ctypes_layer(cuda, oracle):
    from elsa_b200 import _pyelsa as m
    import elsa_b200.pyelsa as ct
    from elsa_b200 import phantoms
    n, views = 24, 20
    xt = phantoms.modified_shepp_logan((n, n, n))  # x fastest (C order of (z, y, x))
    arr = xt.reshape(n, n, n).transpose(2, 1, 0)   # indexed [x, y, z]
    vol = m.VolumeDescriptor([n, n, n])
    sino = m.CircleTrajectoryGenerator.createTrajectory(views, vol, 360, 10.0 * n, 2.5 * n,
                                                        [36, 36])
    A = m.JosephsMethodCUDA(vol, sino)
    b = A.apply(m.DataContainer(arr, vol))
    cvol = ct.VolumeDescriptor([n, n, n])
    csino = ct.CircleTrajectoryGenerator.createTrajectory(views, cvol, 360, 10.0 * n, 2.5 * n,
                                                          detectorSize=[36, 36])
    cA = ct.JosephsMethodCUDA(cvol, csino)
    cb = cA.apply(ct.DataContainer(arr, cvol))
    assert np.array_equal(np.asarray(b), np.asarray(cb))
    for make, cmake in ((lambda: m.CGNE(A, b), lambda: ct.CGNE(cA, cb)),
                        (lambda: m.CGLS(A, b), lambda: ct.CGLS(cA, cb)),
                        (lambda: m.FGM(m.LeastSquares(A, b)),
                         lambda: ct.FGM(ct.LeastSquares(cA, cb))),
                        (lambda: m.SQS(m.LeastSquares(A, b)),
                         lambda: ct.SQS(ct.LeastSquares(cA, cb)))):
        sol = np.asarray(make().solve(8))
        csol = np.asarray(cmake().solve(8))
        assert np.array_equal(sol, csol.reshape(sol.shape))
    r0 = b.squaredL2Norm()
    sol = m.CGNE(A, b).solve(10)
    assert (A.apply(sol) - b).squaredL2Norm() < 0.1 * r0
