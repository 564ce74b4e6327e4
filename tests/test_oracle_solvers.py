"""The oracle's solver restatements on a small dense operator (CPU only): the reference solvers'
own test strategy (solvers/tests/test_CGNE.cpp, test_CGLS.cpp, test_Landweber.cpp, test_APGD.cpp,
test_PowerIterations.cpp use Identity/Scaling fixtures and check convergence to the solution)."""
import numpy as np

from oracle import solvers as S


def _dense(seed=0, m=40, n=24):
    rng = np.random.default_rng(seed)
    M = rng.standard_normal((m, n)).astype(np.float32)
    x = rng.standard_normal(n).astype(np.float32)
    A = lambda v: M @ np.asarray(v, np.float32)  # noqa: E731
    At = lambda v: M.T @ np.asarray(v, np.float32)  # noqa: E731
    return M, A, At, (M @ x).astype(np.float32), x


def test_power_iterations_scaling():
    # powerIterations of a scaling operator returns the scale (test_PowerIterations.cpp)
    A = lambda v: 3.0 * np.asarray(v, np.float32)  # noqa: E731
    lam = S.power_iterations(A, A, 16, 5)
    assert abs(lam - 9.0) < 1e-5


def test_power_iterations_dense():
    M, A, At, _, _ = _dense()
    ref = float(np.linalg.eigvalsh((M.T.astype(np.float64) @ M))[-1])
    assert abs(S.power_iterations(A, At, M.shape[1], 50) - ref) <= 1e-4 * ref


def test_cg_solvers_converge():
    M, A, At, b, x = _dense()
    n = M.shape[1]
    for solve in (lambda: S.cgne(A, At, b, n, 60)[0], lambda: S.cgls(A, At, b, n, 60)[0]):
        assert np.linalg.norm(solve() - x) <= 1e-3 * np.linalg.norm(x)


def test_cgls_damping_matches_tikhonov():
    M, A, At, b, _ = _dense(1)
    n, eps = M.shape[1], 0.7
    x, _ = S.cgls(A, At, b, n, 80, eps=eps, tol=0.0)
    M64 = M.astype(np.float64)
    ref = np.linalg.solve(M64.T @ M64 + eps * eps * np.eye(n), M64.T @ b)
    assert np.linalg.norm(x - ref) <= 1e-3 * np.linalg.norm(ref)


def test_landweber_and_apgd_converge():
    M, A, At, b, x = _dense(2, 60, 16)
    n = M.shape[1]
    xl, _ = S.landweber(A, At, b, n, 3000, power_iters=200)
    xa, _, _ = S.apgd(A, At, b, n, 600, epsilon=0.0, power_iters=200)
    for sol in (xl, xa):
        assert np.linalg.norm(sol - x) <= 1e-2 * np.linalg.norm(x)


def test_prox_operators():
    z = np.array([-2.0, -0.1, 0.0, 0.3, 1.5], np.float32)
    np.testing.assert_allclose(S.prox(z, 0.5, 1, lower=0.0, upper=1.0), [0, 0, 0, 0.3, 1.0],
                               atol=1e-7)
    np.testing.assert_allclose(S.prox(z, 0.5, 2, sigma=0.4), [-1.8, 0, 0, 0.1, 1.3], atol=1e-6)
    np.testing.assert_array_equal(S.prox(z, 0.5, 0), z)


def test_sirt_fgm_ogm_converge():
    M, A, At, b, x = _dense(4, 60, 16)
    M = np.abs(M)  # SIRT's row / column sums need a non-negative system
    A = lambda v: M @ np.asarray(v, np.float32)  # noqa: E731
    At = lambda v: M.T @ np.asarray(v, np.float32)  # noqa: E731
    b = (M @ x).astype(np.float32)
    n = M.shape[1]
    xs, _ = S.sirt(A, At, b, n, 4000, power_iters=200)
    xf, _, _ = S.fgm(A, At, b, n, 3000, epsilon=0.0)
    xo, _, _ = S.ogm(A, At, b, n, 3000, epsilon=0.0)
    for sol in (xs, xf, xo):
        assert np.linalg.norm(sol - x) <= 2e-2 * np.linalg.norm(x)
