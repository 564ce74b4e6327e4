"""pyelsa-style API (elsa_b200.pyelsa) and torch autograd integration (elsa_b200.torch_ops) on the
GPU: end-to-end against the oracle, exact gradients of a data-fidelity loss, and an unrolled
gradient descent with learnable step sizes and per-step checkpointing."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _setup(oracle, n=32, views=30, det=48):
    import elsa_b200.pyelsa as elsa
    vol = elsa.VolumeDescriptor([n, n, n])
    sino = elsa.CircleTrajectoryGenerator.createTrajectory(views, vol, 360, 10.0 * n, 2.5 * n,
                                                           detectorSize=[det, det])
    return elsa, vol, sino


def test_pyelsa_joseph_and_cgne(cuda, oracle):
    elsa, vol, sino = _setup(oracle)
    A = elsa.JosephsMethodCUDA(vol, sino)
    rng = np.random.default_rng(1)
    x = rng.uniform(0, 1, (32, 32, 32)).astype(np.float32)  # indexed [x, y, z]
    Ax = A.apply(x)
    flat = x.reshape(-1, order="F")  # x fastest
    ref = oracle.joseph(flat, (32, 32, 32), sino.shape, sino.poses)
    assert rel_l2(np.asarray(Ax).reshape(-1, order="F"), ref) <= 1e-5
    assert np.asarray(Ax).shape == sino.shape
    # the pyelsa solver drives the same device session as the C ABI
    sol = elsa.CGNE(A, Ax).solve(5)
    assert np.asarray(sol).shape == (32, 32, 32)
    assert elsa.CGNE(A, Ax).solve(5).dot(sol) > 0
    # DataContainer arithmetic goes through the vector-op ABI
    d = Ax - Ax * 0.5
    assert rel_l2(np.asarray(d), 0.5 * np.asarray(Ax)) <= 1e-6
    assert abs(Ax.squaredL2Norm() - float(np.sum(np.square(ref, dtype=np.float64)))) <= \
        1e-5 * Ax.squaredL2Norm()


@pytest.mark.parametrize("cls", ["SiddonsMethodCUDA", "BlobVoxelProjectorCUDA",
                                 "BSplineVoxelProjectorCUDA",
                                 "PhaseContrastBlobVoxelProjectorCUDA"])
def test_pyelsa_projectors_adjoint(cuda, oracle, cls):
    elsa, vol, sino = _setup(oracle, 24, 12, 36)
    A = getattr(elsa, cls)(vol, sino)
    rng = np.random.default_rng(2)
    x = rng.uniform(0, 1, vol.shape).astype(np.float32)
    y = rng.uniform(0, 1, sino.shape).astype(np.float32)
    lhs = A.apply(x).dot(elsa.DataContainer(y, sino))
    rhs = elsa.DataContainer(x, vol).dot(A.applyAdjoint(y))
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs) + 1e-3


def test_pyelsa_solvers(cuda, oracle):
    elsa, vol, sino = _setup(oracle, 24, 20, 36)
    A = elsa.JosephsMethodCUDA(vol, sino)
    from elsa_b200 import phantoms
    x = phantoms.modified_shepp_logan((24, 24, 24)).reshape(-1)  # x fastest
    b = A.apply(elsa.DataContainer(cuda.from_numpy(x), vol))
    r0 = b.squaredL2Norm()
    for solver in (elsa.CGNE(A, b), elsa.CGLS(A, b), elsa.Landweber(A, b),
                   elsa.APGD(A, b, elsa.ProximalBoxConstraint(0.0)),
                   elsa.FISTA(A, b, elsa.ProximalL1(1e-3)), elsa.SIRT(A, b),
                   elsa.FGM(elsa.LeastSquares(A, b)), elsa.OGM(elsa.LeastSquares(A, b)),
                   elsa.SQS(elsa.LeastSquares(A, b)),
                   elsa.SQS(elsa.LeastSquares(A, b), elsa.Scaling(vol, np.ones((24, 24, 24))),
                            False)):
        sol = solver.solve(15)
        res = (A.apply(sol) - b).squaredL2Norm()
        assert res < 0.2 * r0, type(solver).__name__


def test_autograd_gradient_exact(cuda, oracle):
    """Gradient of L(x) = 0.5 |A x - y|^2 through project(): equals A^T (A x - y) of the FP64
    oracle, and matches central differences (eps = 1e-3) of the FP64 oracle loss along 16
    seeded directions."""
    import torch
    from elsa_b200.torch_ops import project
    elsa, vol, sino = _setup(oracle)
    A = elsa.JosephsMethodCUDA(vol, sino)
    vd, dd, poses = (32, 32, 32), sino.shape, sino.poses
    rng = np.random.default_rng(3)
    x0 = rng.uniform(0, 1, 32 ** 3)
    y = rng.uniform(0, 1, int(np.prod(dd))) * 10
    x = torch.tensor(x0, dtype=torch.float32, device="cuda", requires_grad=True)
    yt = torch.tensor(y, dtype=torch.float32, device="cuda")
    loss = 0.5 * ((project(x, A) - yt) ** 2).sum()
    loss.backward()
    g = x.grad.double().cpu().numpy()
    x32 = np.float32(x0).astype(np.float64)

    def L(v):
        r = oracle.joseph(v, vd, dd, poses, dtype=np.float64) - y
        return 0.5 * float(r @ r)

    g64 = oracle.joseph_adjoint(oracle.joseph(x32, vd, dd, poses, dtype=np.float64) - y, vd, dd,
                                poses, dtype=np.float64)
    assert rel_l2(g, g64) <= 1e-5
    eps = 1e-3
    for k in range(16):
        d = np.random.default_rng(100 + k).standard_normal(x0.size)
        d /= np.linalg.norm(d)
        fd = (L(x32 + eps * d) - L(x32 - eps * d)) / (2 * eps)
        assert abs(fd - g @ d) <= 1e-4 * abs(fd) + 1e-3 * np.linalg.norm(g), (k, fd, g @ d)


def test_unrolled_gradient_descent(cuda, oracle):
    """10 unrolled gradient steps x_{k+1} = x_k - a_k A^T (A x_k - y) with learnable a_k and
    per-step activation checkpointing; d loss / d a_k against central differences."""
    import torch
    from torch.utils.checkpoint import checkpoint
    from elsa_b200.torch_ops import project, backproject
    elsa, vol, sino = _setup(oracle, 24, 20, 36)
    A = elsa.JosephsMethodCUDA(vol, sino)
    from elsa_b200 import phantoms
    xt = torch.from_numpy(phantoms.modified_shepp_logan((24, 24, 24)).reshape(-1)).cuda()
    y = project(xt, A).detach()
    lam = elsa.powerIterations(A, 20)

    def step(x, a):
        return x - a * backproject(project(x, A) - y, A)

    def run(alphas, ckpt):
        x = torch.zeros_like(xt)
        for k in range(alphas.shape[0]):
            x = checkpoint(step, x, alphas[k], use_reentrant=False) if ckpt else step(x, alphas[k])
        return ((x - xt).double() ** 2).sum()

    base = torch.full((10,), 1.0 / lam, dtype=torch.float32, device="cuda")
    alphas = base.clone().requires_grad_(True)
    loss = run(alphas, True)
    loss.backward()
    g = alphas.grad.double().cpu().numpy()
    # the checkpointed and the plain graph give the same gradient
    a2 = base.clone().requires_grad_(True)
    run(a2, False).backward()
    assert np.allclose(g, a2.grad.double().cpu().numpy(), rtol=1e-5, atol=0)
    # the final iterate is affine in each a_k, so the loss is quadratic in a_k and the central
    # difference is exact up to rounding
    gmax = float(np.abs(g).max())
    for k in (0, 4, 9):
        h = 0.05 / lam
        ap, am = base.clone(), base.clone()
        ap[k] += h
        am[k] -= h
        with torch.no_grad():
            fd = (run(ap, False) - run(am, False)).item() / (2 * h)
        assert abs(fd - g[k]) <= 5e-2 * max(abs(fd), abs(g[k])) + 1e-3 * gmax, (k, fd, g[k])


def test_pyelsa_ordered_subsets(cuda, oracle):
    """SubsetSampler + SQS in ordered-subset mode (the reference's usage: subset projectors and
    partitioned data as LeastSquares problems) against the C ABI run on the same subsets."""
    import elsa_b200
    elsa, vol, sino = _setup(oracle, 24, 30, 36)
    A = elsa.JosephsMethodCUDA(vol, sino)
    from elsa_b200 import phantoms
    x = phantoms.modified_shepp_logan((24, 24, 24)).reshape(-1)
    b = A.apply(elsa.DataContainer(cuda.from_numpy(x), vol))
    sampler = elsa.SubsetSampler(vol, sino, 3, elsa.SubsetSampler.ROTATIONAL_CLUSTERING)
    blocks = sampler.getPartitionedData(b)
    projs = sampler.getSubsetProjectors(elsa.JosephsMethodCUDA)
    subsets = [elsa.LeastSquares(p, d) for p, d in zip(projs, blocks)]
    sol = elsa.SQS(elsa.LeastSquares(A, b), subsets).solve(4)
    r0 = b.squaredL2Norm()
    assert (A.apply(sol) - b).squaredL2Norm() < 0.2 * r0
    # the same run through the C ABI
    s = cuda.cuda.current_stream().cuda_stream
    xd = cuda.zeros(A.native.domain_size, device="cuda")
    sv = elsa_b200.Solver.sqs(A.native, b._ptr(), xd.data_ptr(),
                              subsets=[(p.native, d._ptr()) for p, d in zip(projs, blocks)],
                              stream=s)
    sv.iterate(4, s)
    cuda.cuda.synchronize()
    assert np.array_equal(xd.cpu().numpy(), sol.tensor.cpu().numpy())
    sv.close()


def test_pyelsa_image_files(cuda, oracle, tmp_path):
    """EDF / MHD / PGM through pyelsa's names: a device DataContainer written and read back keeps
    its values, sizes and spacing (io/tests/test_EDFHandler.cpp, test_MHDHandler.cpp)."""
    import elsa_b200.pyelsa as elsa
    vol = elsa.VolumeDescriptor([11, 17], [0.5, 2.0])
    rng = np.random.default_rng(1)
    arr = rng.standard_normal((11, 17)).astype(np.float32)
    dc = elsa.DataContainer(arr, vol)
    elsa.EDF.write(dc, str(tmp_path / "a.edf"))
    back = elsa.EDF.readf(str(tmp_path / "a.edf"))
    assert back.getDataDescriptor() == vol
    assert np.array_equal(np.asarray(back), arr)
    elsa.MHD.write(dc, str(tmp_path / "a.mhd"), str(tmp_path / "a.raw"))
    back = elsa.MHD.readf(str(tmp_path / "a.mhd"))
    assert back.getDataDescriptor() == vol and np.array_equal(np.asarray(back), arr)
    elsa.PGM.write(dc, str(tmp_path / "a.pgm"))
    assert open(tmp_path / "a.pgm").read().startswith("P2\n11 17\n255\n")


def test_pyelsa_fast_flag(cuda, oracle):
    """JosephsMethodCUDA(..., fast=True) is elsa's unmatched fast adjoint (the C ABI's Joseph
    parameter 1); JosephsMethod and the default JosephsMethodCUDA are the matched operator."""
    import elsa_b200
    elsa, vol, sino = _setup(oracle)
    rng = np.random.default_rng(4)
    y = rng.uniform(0, 1, tuple(sino.shape)).astype(np.float32)
    fast = elsa.JosephsMethodCUDA(vol, sino, fast=True)
    matched = elsa.JosephsMethodCUDA(vol, sino)
    cpu_name = elsa.JosephsMethod(vol, sino)
    a_fast = np.asarray(fast.applyAdjoint(y)).ravel()
    a_matched = np.asarray(matched.applyAdjoint(y)).ravel()
    assert np.array_equal(a_matched, np.asarray(cpu_name.applyAdjoint(y)).ravel())
    p = elsa_b200.Projector(elsa_b200.PROJECTOR_JOSEPH, list(vol.shape), list(sino.shape),
                            sino.poses, [1.0])
    yd = cuda.from_numpy(np.ascontiguousarray(y).reshape(-1, order="F")).cuda()
    out = cuda.empty(p.domain_size, device="cuda")
    p.apply_adjoint_ptr(yd.data_ptr(), out.data_ptr(), cuda.cuda.current_stream().cuda_stream)
    cuda.cuda.synchronize()
    a_fast_x_fastest = np.asarray(fast.applyAdjoint(y)).ravel(order="F")
    assert np.array_equal(a_fast_x_fastest, out.cpu().numpy())
    assert not np.array_equal(a_fast, a_matched)


def test_autograd_warns_for_the_fast_adjoint(cuda, oracle):
    """Gradients through JosephsMethodCUDA(..., fast=True) use its unmatched backprojection: the
    torch op says so (once per operator); the matched operator stays silent."""
    import warnings

    from elsa_b200.torch_ops import project
    elsa, vol, sino = _setup(oracle, n=16, views=8, det=24)
    fast = elsa.JosephsMethodCUDA(vol, sino, fast=True)
    matched = elsa.JosephsMethodCUDA(vol, sino)
    assert not fast.native.matched and matched.native.matched
    x = cuda.rand(16 ** 3, device="cuda", requires_grad=True)
    def ours(caught):
        return [w for w in caught if "fast backprojection" in str(w.message)]

    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter("always")
        project(x, matched).sum().backward()
        assert not ours(caught)
        project(x, fast).sum().backward()
        project(x, fast).sum().backward()
    assert len(ours(caught)) == 1
