"""The oracle's blob / B-spline restatement against elsa's golden arrays and known answers (CPU)."""
import json
import os

import numpy as np
import pytest

from kat_cases import voxel_cases

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "voxel_luts.json")


def _approx(a, b, eps):
    """doctest Approx: |a - b| < eps * (1 + max(|a|, |b|)) (test_routines use this semantic)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.all(np.abs(a - b) < eps * (1.0 + np.maximum(np.abs(a), np.abs(b))))


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def test_bessel_against_scipy(oracle):
    """core/tests/test_Bessel.cpp compares bessi0..4 against std::cyl_bessel_i on [0, 4]; here
    also on [4, 20] (alpha = 10.83 is the default blob parameter) and for m = 5, 6."""
    sp = pytest.importorskip("scipy.special")
    for m in range(7):
        for x in np.concatenate([np.linspace(0, 4, 101), np.linspace(4, 20, 81)]):
            ref = float(sp.iv(m, x))
            got = oracle.bessel(m, x)
            assert _approx(got, ref, 1.2e-5), (m, x, got, ref)


def test_projected_blob_lut_golden(oracle, golden):
    """test_Luts.cpp:125-246: ProjectedBlob<data_t, 101>(2, 10.83, 2) LUT at i/50."""
    exp = np.array(golden["luts"]["projected_blob_lut_a2_alpha10.83_m2"])
    lut = oracle.blob_lut(2.0, 10.83, 2, 0, 101)
    for i in range(99):
        got = oracle.lut_lerp(lut, 2.0, i / 50.0)
        assert _approx(got, exp[i], 1e-6), (i, got, exp[i])


def test_projected_bspline_lut_golden(oracle, golden):
    """test_Luts.cpp:249-305: ProjectedBSpline<data_t, 101>(dim 2, order 3) LUT at i/50."""
    exp = np.array(golden["luts"]["projected_bspline_lut_order3_dim2"])
    lut = oracle.bspline_lut(2, 3, 0, 101)
    support = oracle.bspline_support(3)
    for i in range(101):
        got = oracle.lut_lerp(lut, support, i / 50.0)
        assert _approx(got, exp[i], 1e-6), (i, got, exp[i])


@pytest.mark.parametrize("a", [1.0, 2.0])
def test_projected_blob_derivative_golden(oracle, golden, a):
    """test_BlobDerivative.cpp:17-46 (derivative) and test_BlobGradientHelper.cpp:17-46
    (normalized gradient = derivative / s), s = i * a / 100."""
    scale = 100.0 if a == 1.0 else 50.0
    for key, exp in golden["blob_derivative_projected"].items():
        alpha = float(key.split("_alpha")[1].split("_m")[0])
        m = int(key.split("_m")[1])
        a32, al32 = float(np.float32(a)), float(np.float32(alpha))
        for i in range(101):
            x = float(np.float32(i / scale))
            got = oracle.blob_projected(x, a32, al32, m, 1)
            assert _approx(got, exp[i], 1.2e-5), (key, i, got, exp[i])
            if i >= 1:
                g = oracle.blob_projected(x, a32, al32, m, 2)
                assert _approx(g, exp[i] / x, 1.2e-5), (key, i, g, exp[i] / x)


def test_voxel_kats(oracle):
    for c in voxel_cases(oracle):
        lut, support, wk = oracle.voxel_lut("blob", c["dim"])
        y = oracle.voxel_project(False, c["x"], c["vol"], c["det"], c["poses"], lut, support, wk)
        tol = c["rtol"] * np.abs(c["y_expect"]) + 1e-7
        assert np.all(np.abs(y - c["y_expect"]) <= tol), (c["name"], y, c["y_expect"])


@pytest.mark.parametrize("kind", ["blob", "bspline", "phase_blob", "phase_bspline"])
@pytest.mark.parametrize("dim", [2, 3])
def test_voxel_adjointness(oracle, kind, dim):
    vol = (20, 20) if dim == 2 else (12, 12, 12)
    det = [30] if dim == 2 else [18, 18]
    poses, dd = oracle.circle_trajectory(vol, 9, 360, 10 * vol[0], 2.5 * vol[0], det)
    lut, support, wk = oracle.voxel_lut(kind, dim)
    rng = np.random.default_rng(4)
    x = rng.uniform(0, 1, int(np.prod(vol)))
    y = rng.uniform(0, 1, int(np.prod(dd)))
    Ax = oracle.voxel_project(False, x, vol, dd, poses, lut, support, wk, dtype=np.float64)
    Aty = oracle.voxel_project(True, y, vol, dd, poses, lut, support, wk, dtype=np.float64)
    assert abs(Ax @ y - x @ Aty) <= 1e-12 * abs(Ax @ y)


def test_loop_modes(oracle):
    """The reference CPU loop (mode 0) visits a rows x cols block with the u and v extents of the
    clamped footprint swapped (VoxelComputation.h:88-113); the footprint rectangle (mode 1) agrees
    with it exactly when both extents are equal, e.g. for the centre voxel of an odd volume, whose
    centre projects to the same fraction in u and v. Over a whole volume the extents often
    differ (floor(c + r) - ceil(c - r) depends on the fraction of c), so the two modes differ."""
    vol = (15, 15, 15)
    poses, det = oracle.circle_trajectory(vol, 8, 360, 150, 40, [41, 41])
    lut, support, wk = oracle.voxel_lut("blob", 3)
    x = np.zeros(vol, np.float32)
    x[7, 7, 7] = 1
    y0 = oracle.voxel_project(False, x, vol, det, poses, lut, support, wk, loop_mode=0)
    y1 = oracle.voxel_project(False, x, vol, det, poses, lut, support, wk, loop_mode=1)
    np.testing.assert_array_equal(y0, y1)
    x = np.random.default_rng(0).uniform(0, 1, vol).astype(np.float32)
    y0 = oracle.voxel_project(False, x, vol, det, poses, lut, support, wk, loop_mode=0)
    y1 = oracle.voxel_project(False, x, vol, det, poses, lut, support, wk, loop_mode=1)
    assert np.any(y0 != y1)
