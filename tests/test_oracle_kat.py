"""Pins the oracle (CPU restatement of elsa) against elsa's own known-answer tests."""
import numpy as np
import pytest

from conftest import rel_l2
from kat_cases import binary_cases, joseph_cases, lut_cases, siddon_cases


def _run(O, fn, case, dtype):
    vol, det = case["vol"], case["det"]
    y = fn(case["x"], vol, det, case["poses"], dtype=dtype)
    bp = fn.adjoint(case["y"], vol, det, case["poses"], dtype=dtype)
    return y, bp


class _Joseph:
    def __init__(self, O):
        self.O = O

    def __call__(self, x, vol, det, poses, dtype):
        return self.O.joseph(x, vol, det, poses, dtype=dtype)

    def adjoint(self, y, vol, det, poses, dtype):
        return self.O.joseph_adjoint(y, vol, det, poses, dtype=dtype)


class _Siddon(_Joseph):
    def __call__(self, x, vol, det, poses, dtype):
        return self.O.siddon(x, vol, det, poses, dtype=dtype)

    def adjoint(self, y, vol, det, poses, dtype):
        return self.O.siddon_adjoint(y, vol, det, poses, dtype=dtype)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_joseph_kat(oracle, dtype):
    for case in joseph_cases(oracle):
        y, bp = _run(oracle, _Joseph(oracle), case, dtype)
        tol = case.get("tol", 1e-5)
        np.testing.assert_allclose(y, case["y_expect"], rtol=tol, err_msg=case["name"])
        assert rel_l2(bp, case["bp_expect"]) <= tol, case["name"]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_siddon_kat(oracle, dtype):
    for case in siddon_cases(oracle):
        y, bp = _run(oracle, _Siddon(oracle), case, dtype)
        np.testing.assert_allclose(y, case["y_expect"], rtol=1e-5, err_msg=case["name"])
        assert rel_l2(bp, case["bp_expect"]) <= 1e-5, case["name"]


class _Binary(_Joseph):
    def __call__(self, x, vol, det, poses, dtype):
        return self.O.binary(x, vol, det, poses, dtype=dtype)

    def adjoint(self, y, vol, det, poses, dtype):
        return self.O.binary_adjoint(y, vol, det, poses, dtype=dtype)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_binary_kat(oracle, dtype):
    for case in binary_cases(oracle):
        y, bp = _run(oracle, _Binary(oracle), case, dtype)
        np.testing.assert_array_equal(y, case["y_expect"], err_msg=case["name"])
        np.testing.assert_array_equal(bp.reshape(case["bp_expect"].shape), case["bp_expect"],
                                      err_msg=case["name"])


def _approx_ok(got, want, tol):
    # doctest Approx: |a - b| < eps * (1 + max(|a|, |b|))
    return abs(got - want) < tol * (1.0 + max(abs(got), abs(want)))


def test_lut_projector_kat(oracle):
    lut = oracle.blob_lut()
    bad = []
    for case in lut_cases(oracle):
        y = oracle.lut_project(False, case["x"], case["vol"], case["det"], case["poses"], lut,
                               2.0, 2)
        for got, want in zip(y, case["y_expect"]):
            if not _approx_ok(float(got), float(want), case["tol"]):
                bad.append((case["name"], float(got), float(want)))
    assert not bad, bad[:10]


def test_joseph_outputs_overwritten(oracle):
    """test_JosephsMethod.cpp:322-436: outputs are zeroed by the projector."""
    poses, det = oracle.circle_trajectory([8, 8], 4, 360, 40, 10)
    y = oracle.joseph(np.zeros(64, np.float32), [8, 8], det, poses)
    assert not y.any()
    x = oracle.joseph_adjoint(np.zeros(int(np.prod(det)), np.float32), [8, 8], det, poses)
    assert not x.any()


def test_missing_rays_are_zero(oracle):
    """test_JosephsMethod.cpp:438-640: rays that miss the volume project to 0."""
    poses = np.stack([oracle.geometry2d(100.0, 5.0, 0.0, [1, 1], [2.5, 2.5], [1, 1], [0.5, 0.5],
                                        0.0, [10.0, 0.0])])
    y = oracle.joseph(np.ones(25, np.float32), [5, 5], [1, 1], poses)
    assert y[0] == 0.0


def test_adjoint_dot_oracle(oracle):
    """<A x, y> = <x, A^T y> for the oracle itself (float64 data, exact up to rounding)."""
    rng = np.random.default_rng(1)
    for vol, nang, s2c, c2d, det in (((16, 16), 12, 80, 20, [23]),
                                     ((12, 12, 12), 10, 60, 15, [17, 17])):
        poses, dd = oracle.circle_trajectory(vol, nang, 360, s2c, c2d, det)
        x = rng.uniform(0, 1, int(np.prod(vol)))
        y = rng.uniform(0, 1, int(np.prod(dd)))
        for mode in (0, 1):
            Ax = oracle.joseph(x, vol, dd, poses, dtype=np.float64, mode=mode)
            Aty = oracle.joseph_adjoint(y, vol, dd, poses, dtype=np.float64, mode=mode)
            assert abs(Ax @ y - x @ Aty) <= 1e-12 * abs(Ax @ y)
        Ax = oracle.siddon(x, vol, dd, poses, dtype=np.float64)
        Aty = oracle.siddon_adjoint(y, vol, dd, poses, dtype=np.float64)
        assert abs(Ax @ y - x @ Aty) <= 1e-12 * abs(Ax @ y)


def test_accumulated_positions_matter(oracle):
    """The reference accumulates pos += step (DrivingDirectionTraversal.cpp:265); evaluating
    pos0 + j*step instead already moves a 48^3 cone-beam projection by more than 1e-6, which is
    why the CUDA kernels reproduce the accumulation exactly."""
    from elsa_b200 import phantoms
    vol = (48, 48, 48)
    poses, dd = oracle.circle_trajectory(vol, 24, 360, 480, 120, [72, 72])
    x = phantoms.modified_shepp_logan(vol)
    y0 = oracle.joseph(x, vol, dd, poses, mode=0)
    y1 = oracle.joseph(x, vol, dd, poses, mode=1)
    assert rel_l2(y1, y0) > 1e-6


def test_oracle_adjoints_deterministic(oracle):
    """The oracle's adjoints add their contributions in a fixed order (ray ranges scattered into
    partial volumes, summed in range order): the same bits for every thread count and run."""
    vol = (20, 24, 28)
    poses, det = oracle.circle_trajectory(vol, 12, 360, 200, 50, [32, 30])
    y = np.random.default_rng(4).uniform(0, 1, int(np.prod(det))).astype(np.float32)
    fns = [lambda: oracle.joseph_adjoint(y, vol, det, poses),
           lambda: oracle.siddon_adjoint(y, vol, det, poses),
           lambda: oracle.binary_adjoint(y, vol, det, poses),
           lambda: oracle.joseph_adjoint(y.astype(np.float64), vol, det, poses,
                                         dtype=np.float64)]
    threads = oracle.num_threads()
    try:
        oracle.set_num_threads(1)
        single = [f() for f in fns]
        oracle.set_num_threads(max(2, threads))
        multi = [f() for f in fns]
        again = [f() for f in fns]
    finally:
        oracle.set_num_threads(threads)
    for a, b, c in zip(single, multi, again):
        assert np.array_equal(a, b) and np.array_equal(b, c)
