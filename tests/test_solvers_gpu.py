"""Fused vector operations and device-resident solvers (through the C ABI) against numpy float64
and the oracle's restatement of elsa's solvers (oracle/solvers.py)."""
import ctypes

import numpy as np
import pytest

from conftest import record_parity, rel_l2

pytestmark = pytest.mark.gpu

# Solver tolerance: relative L2 of the iterate after the stated number of iterations against the
# FP32 oracle. Both sides run float32 vectors with float64 inner products over projectors that
# agree to ~3e-7, and both are deterministic (the oracle's adjoints add in a fixed order), so each
# distance is one fixed number; it is written to the parity record (conftest.record_parity)
# beside the distance of the FP32 oracle from the FP64 oracle. Landweber/APGD/SIRT are
# contractions and stay within 1e-5. CG-type recurrences (CGNE, CGLS, FGM, OGM) amplify the
# last-bit differences of the projectors on these noise-free, ill-conditioned problems; their
# bounds are fixed per solver and problem, a few times the measured distance.
CG_BOUNDS = {  # measured on a B200 (device vs FP32 oracle; FP32 vs FP64 oracle in brackets)
    ("cgne", "fan2d_64"): 5e-4,         # 1.9e-4 (4.0e-2)
    ("cgne", "cone3d_24"): 1e-5,        # 2.7e-6 (3.2e-6)
    ("cgls", "fan2d_64"): 1e-4,         # 2.3e-5 (4.0e-2)
    ("cgls", "cone3d_24"): 1e-5,        # 3.6e-7 (3.2e-7)
    ("cgls_damped", "fan2d_64"): 1.5e-3,  # 5.8e-4 (1.2e-4)
    ("cgls_damped", "cone3d_24"): 1e-5,   # 1.3e-6 (1.1e-6)
    ("fgm", "fan2d_64"): 1e-5, ("fgm", "cone3d_24"): 1e-5,  # 2.5e-7, 2.3e-7
    ("ogm", "fan2d_64"): 1e-5, ("ogm", "cone3d_24"): 1e-5,  # 6.1e-7, 3.3e-7
}
GD_TOL = 1e-5


def _vecop(torch, name, *args):
    from elsa_b200 import _capi
    _capi.call(name, *args)
    torch.cuda.synchronize()


@pytest.mark.parametrize("n", [0, 1, 3, 1000, 4097, (1 << 20) + 3])
@pytest.mark.parametrize("offset", [0, 1])
def test_dot_and_norm(cuda, n, offset):
    torch = cuda
    rng = np.random.default_rng(n + 17 * offset)
    xs = rng.standard_normal(n + offset).astype(np.float32)
    ys = rng.standard_normal(n + offset).astype(np.float32)
    x = torch.from_numpy(xs).cuda()
    y = torch.from_numpy(ys).cuda()
    res = torch.full((2,), np.nan, dtype=torch.float64, device="cuda")
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    xp = ctypes.c_void_p(x.data_ptr() + 4 * offset)
    yp = ctypes.c_void_p(y.data_ptr() + 4 * offset)
    _vecop(torch, "elsa_dot", xp, yp, n, ctypes.c_void_p(res.data_ptr()), s)
    _vecop(torch, "elsa_squared_l2_norm", xp, n, ctypes.c_void_p(res.data_ptr() + 8), s)
    got = res.cpu().numpy()
    x64 = xs[offset:].astype(np.float64)
    y64 = ys[offset:].astype(np.float64)
    ref_dot = float(np.dot(x64, y64))
    ref_sq = float(np.dot(x64, x64))
    scale = max(1.0, float(np.dot(np.abs(x64), np.abs(y64))))
    assert abs(got[0] - ref_dot) <= 1e-13 * scale
    assert abs(got[1] - ref_sq) <= 1e-13 * max(1.0, ref_sq)
    # deterministic: the same call gives the same bits
    res2 = torch.full((1,), np.nan, dtype=torch.float64, device="cuda")
    _vecop(torch, "elsa_dot", xp, yp, n, ctypes.c_void_p(res2.data_ptr()), s)
    assert res2.cpu().numpy()[0] == got[0]


@pytest.mark.parametrize("n", [1, 1000, 4097, (1 << 20) + 3])
def test_lincomb(cuda, n):
    torch = cuda
    rng = np.random.default_rng(n)
    xs = rng.standard_normal(n).astype(np.float32)
    ys = rng.standard_normal(n).astype(np.float32)
    x = torch.from_numpy(xs).cuda()
    y = torch.from_numpy(ys).cuda()
    out = torch.full((n,), np.nan, dtype=torch.float32, device="cuda")
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    a, b = 0.75, -1.3
    _vecop(torch, "elsa_lincomb", ctypes.c_float(a), ctypes.c_void_p(x.data_ptr()),
           ctypes.c_float(b), ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(out.data_ptr()), n, s)
    ref = np.float32(a) * xs + np.float32(b) * ys
    # one rounding of difference at most (the device may fuse one multiply into the add)
    tol = 4 * np.finfo(np.float32).eps * (np.abs(a * xs) + np.abs(b * ys)).max()
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=0, atol=tol)
    # in place: out aliases x
    _vecop(torch, "elsa_lincomb", ctypes.c_float(a), ctypes.c_void_p(x.data_ptr()),
           ctypes.c_float(b), ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(x.data_ptr()), n, s)
    assert torch.equal(x, out)


# Small problems the oracle projects in well under a second per application.
PROBLEMS = {
    "fan2d_64": dict(vol=(64, 64), views=90, s2c=500, c2d=125, det=[92]),
    "cone3d_24": dict(vol=(24, 24, 24), views=30, s2c=240, c2d=60, det=[36, 36]),
}


def _problem(torch, oracle, name, kind=None):
    import elsa_b200
    from elsa_b200 import phantoms
    c = PROBLEMS[name]
    poses, det = oracle.circle_trajectory(c["vol"], c["views"], 360, c["s2c"], c["c2d"], c["det"])
    proj = elsa_b200.Projector(elsa_b200.PROJECTOR_JOSEPH if kind is None else kind, c["vol"],
                               det, poses)
    vol = c["vol"]
    phantom = np.asarray(phantoms.modified_shepp_logan(tuple(reversed(vol))), np.float32)
    A = lambda v: oracle.joseph(v, vol, det, poses).ravel()  # noqa: E731
    At = lambda v: oracle.joseph_adjoint(v, vol, det, poses).ravel()  # noqa: E731
    b = A(phantom.ravel())
    return proj, A, At, b, phantom.size


def _f64_ops(oracle, name):
    c = PROBLEMS[name]
    vol = c["vol"]
    poses, det = oracle.circle_trajectory(vol, c["views"], 360, c["s2c"], c["c2d"], c["det"])
    A = lambda v: oracle.joseph(np.asarray(v, np.float64), vol, det, poses,  # noqa: E731
                                dtype=np.float64).ravel()
    At = lambda v: oracle.joseph_adjoint(np.asarray(v, np.float64), vol, det,  # noqa: E731
                                         poses, dtype=np.float64).ravel()
    return A, At


def _check_cg(solver, name, x, xr, x64, res, hist, hist64):
    """Fixed iterate bound of CG_BOUNDS and a residual bound; both distances are recorded."""
    bound = CG_BOUNDS[(solver, name)]
    e32, e3264 = rel_l2(x, xr), rel_l2(xr, x64)
    record_parity("%s_%s" % (solver, name), gpu_f32=e32, gpu_f64=rel_l2(x, x64), f32_f64=e3264,
                  bound=bound)
    print("%s %s: gpu-f32 %.3g, f32-f64 %.3g" % (solver, name, e32, e3264))
    assert e32 <= bound
    if res is not None:
        assert abs(res - hist[-1]) <= max(1e-3 * hist[-1], 4.0 * abs(hist[-1] - hist64[-1]))


def _run_solver(torch, proj, kind, b_np, iterations, params=(), x0=None, chunks=1):
    import elsa_b200
    b = torch.from_numpy(np.ascontiguousarray(b_np, np.float32)).cuda()
    x = torch.full((proj.domain_size,), np.nan, dtype=torch.float32, device="cuda")
    if x0 is not None:
        x.copy_(torch.from_numpy(np.ascontiguousarray(x0, np.float32)))
    s = torch.cuda.current_stream().cuda_stream
    solver = elsa_b200.Solver(kind, proj, b.data_ptr(), x.data_ptr(), use_x0=x0 is not None,
                              stream=s, params=params)
    per = iterations // chunks
    for _ in range(chunks):
        solver.iterate(per, s)
    res = solver.squared_residual(s)
    step = solver.step_size()
    torch.cuda.synchronize()
    out = x.cpu().numpy()
    solver.close()
    return out, res, step


@pytest.mark.parametrize("name", sorted(PROBLEMS))
def test_power_iterations(cuda, oracle, name):
    import elsa_b200
    from oracle import solvers as S
    proj, A, At, b, n = _problem(cuda, oracle, name)
    lam = elsa_b200.power_iterations(proj, 5, cuda.cuda.current_stream().cuda_stream)
    ref = S.power_iterations(A, At, n, 5)
    assert abs(lam - ref) <= 1e-5 * abs(ref), (lam, ref)


@pytest.mark.parametrize("name", sorted(PROBLEMS))
def test_cgne_parity(cuda, oracle, name):
    import elsa_b200
    from oracle import solvers as S
    proj, A, At, b, n = _problem(cuda, oracle, name)
    x, res, _ = _run_solver(cuda, proj, elsa_b200.SOLVER_CGNE, b, 10, chunks=2)
    xr, hist = S.cgne(A, At, b, n, 10)
    A64, At64 = _f64_ops(oracle, name)
    x64, hist64 = S.cgne(A64, At64, b, n, 10, dtype=np.float64)
    _check_cg("cgne", name, x, xr, x64, res, hist, hist64)


@pytest.mark.parametrize("name", sorted(PROBLEMS))
def test_cgls_parity(cuda, oracle, name):
    import elsa_b200
    from oracle import solvers as S
    proj, A, At, b, n = _problem(cuda, oracle, name)
    x, res, _ = _run_solver(cuda, proj, elsa_b200.SOLVER_CGLS, b, 10)
    xr, hist = S.cgls(A, At, b, n, 10)
    A64, At64 = _f64_ops(oracle, name)
    x64, hist64 = S.cgls(A64, At64, b, n, 10, dtype=np.float64)
    _check_cg("cgls", name, x, xr, x64, res, hist, hist64)
    # damped, warm start from a seeded random x0
    x0 = np.random.default_rng(3).random(n).astype(np.float32)
    x, _, _ = _run_solver(cuda, proj, elsa_b200.SOLVER_CGLS, b, 8, params=(2.0, 1e-4), x0=x0)
    xr, hist = S.cgls(A, At, b, n, 8, x0=x0, eps=2.0)
    x64, hist64 = S.cgls(A64, At64, b, n, 8, x0=x0, eps=2.0, dtype=np.float64)
    _check_cg("cgls_damped", name, x, xr, x64, None, hist, hist64)


def test_cgls_tolerance_stops(cuda, oracle):
    import elsa_b200
    from oracle import solvers as S
    proj, A, At, b, n = _problem(cuda, oracle, "fan2d_64")
    # tol above |A^T b|^2: the reference returns before the first iteration (x = 0)
    big = 10.0 * float(np.sum(np.square(At(b), dtype=np.float64)))
    x, _, _ = _run_solver(cuda, proj, elsa_b200.SOLVER_CGLS, b, 5, params=(0.0, big))
    xr, hist = S.cgls(A, At, b, n, 5, tol=big)
    assert not hist and not np.any(xr) and not np.any(x)


@pytest.mark.parametrize("name", sorted(PROBLEMS))
def test_landweber_parity(cuda, oracle, name):
    import elsa_b200
    from oracle import solvers as S
    proj, A, At, b, n = _problem(cuda, oracle, name)
    x, _, step = _run_solver(cuda, proj, elsa_b200.SOLVER_LANDWEBER, b, 12)
    xr, step_r = S.landweber(A, At, b, n, 12)
    assert abs(step - step_r) <= 1e-5 * step_r
    assert rel_l2(x, xr) <= GD_TOL
    x, _, step = _run_solver(cuda, proj, elsa_b200.SOLVER_LANDWEBER, b, 6, params=(step_r / 2,))
    xr, _ = S.landweber(A, At, b, n, 6, step=step_r / 2)
    assert step == step_r / 2
    assert rel_l2(x, xr) <= GD_TOL


@pytest.mark.parametrize("prox", ["identity", "box", "l1"])
def test_apgd_parity(cuda, oracle, prox):
    import elsa_b200
    from oracle import solvers as S
    proj, A, At, b, n = _problem(cuda, oracle, "cone3d_24")
    if prox == "identity":
        params, kw = (0.0,), {}
    elif prox == "box":
        params, kw = (0.0, S.F32_EPS, 1, 0.0, 0.5), dict(kind=1, lower=0.0, upper=0.5)
    else:
        params, kw = (0.0, S.F32_EPS, 2, np.nan, np.nan, 0.05), dict(kind=2, sigma=0.05)
    x, g2, step = _run_solver(cuda, proj, elsa_b200.SOLVER_APGD, b, 10, params=params)
    xr, mu_r, hist = S.apgd(A, At, b, n, 10, **kw)
    assert abs(step - mu_r) <= 1e-5 * mu_r
    assert rel_l2(x, xr) <= GD_TOL
    assert abs(g2 - hist[-1]) <= 1e-3 * hist[-1]


def test_apgd_epsilon_stops(cuda, oracle):
    import elsa_b200
    from oracle import solvers as S
    proj, A, At, b, n = _problem(cuda, oracle, "fan2d_64")
    # epsilon above the first |grad|^2: one update, then the iterate stays put
    g0 = float(np.sum(np.square(At(b), dtype=np.float64)))
    x, _, _ = _run_solver(cuda, proj, elsa_b200.SOLVER_APGD, b, 6, params=(0.0, 2 * g0))
    xr, _, hist = S.apgd(A, At, b, n, 6, epsilon=2 * g0)
    assert len(hist) == 1
    assert rel_l2(x, xr) <= GD_TOL


def test_solver_argument_errors(cuda, oracle):
    import elsa_b200
    proj, A, At, b, n = _problem(cuda, oracle, "fan2d_64")
    bt = cuda.from_numpy(b).cuda()
    x = cuda.zeros(n, dtype=cuda.float32, device="cuda")
    with pytest.raises(elsa_b200.InvalidArgumentError):
        elsa_b200.Solver(elsa_b200.SOLVER_SQS + 1, proj, bt.data_ptr(), x.data_ptr())
    with pytest.raises(elsa_b200.InvalidArgumentError):  # SQS momentum flag must be 0 or 1
        elsa_b200.Solver(elsa_b200.SOLVER_SQS, proj, bt.data_ptr(), x.data_ptr(), params=(0.5,))
    with pytest.raises(elsa_b200.InvalidArgumentError):
        elsa_b200.Solver(elsa_b200.SOLVER_LANDWEBER, proj, bt.data_ptr(), x.data_ptr(),
                         params=(1.0, 2.0))
    with pytest.raises(elsa_b200.InvalidArgumentError):
        elsa_b200.Solver(elsa_b200.SOLVER_APGD, proj, bt.data_ptr(), x.data_ptr(),
                         params=(0.0, 1e-7, 5))
    with pytest.raises(elsa_b200.InvalidArgumentError):
        elsa_b200.Solver(elsa_b200.SOLVER_APGD, proj, bt.data_ptr(), x.data_ptr(),
                         params=(0.0, 1e-7, 1, 1.0, 0.0))


@pytest.mark.parametrize("name", sorted(PROBLEMS))
def test_sirt_parity(cuda, oracle, name):
    import elsa_b200
    from oracle import solvers as S
    proj, A, At, b, n = _problem(cuda, oracle, name)
    x, _, step = _run_solver(cuda, proj, elsa_b200.SOLVER_SIRT, b, 12)
    xr, step_r = S.sirt(A, At, b, n, 12)
    assert abs(step - step_r) <= 1e-5 * step_r
    assert rel_l2(x, xr) <= GD_TOL


@pytest.mark.parametrize("kind", ["fgm", "ogm"])
@pytest.mark.parametrize("name", sorted(PROBLEMS))
def test_fgm_ogm_parity(cuda, oracle, name, kind):
    import elsa_b200
    from oracle import solvers as S
    proj, A, At, b, n = _problem(cuda, oracle, name)
    sk = elsa_b200.SOLVER_FGM if kind == "fgm" else elsa_b200.SOLVER_OGM
    x, g2, step = _run_solver(cuda, proj, sk, b, 10)
    xr, lip, hist = getattr(S, kind)(A, At, b, n, 10)
    assert abs(step - 1.0 / lip) <= 1e-5 / lip
    # accelerated gradient methods amplify rounding like CG: same bound as the CG solvers
    A64, At64 = _f64_ops(oracle, name)
    x64, _, h64 = getattr(S, kind)(A64, At64, b, n, 10, dtype=np.float64)
    _check_cg(kind, name, x, xr, x64, g2, hist, h64)
