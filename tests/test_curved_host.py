"""Curved-detector planar coordinates (CurvedDetectorDescriptor) from the C ABI and the oracle
against the reference's tests/test_CurvedDetectorDescriptor.cpp:254-409 (angle 2, s2d 14)."""
import numpy as np
import pytest

import elsa_b200


def _both(oracle, dim, nu, nv):
    a = elsa_b200.curved_detector_coords(dim, nu, nv, 2.0, 14.0)
    b = oracle.curved_coords(dim, nu, nv, 2.0, 14.0)
    assert np.array_equal(a, b)  # the same float operations on both sides
    return a


def test_planar_coords_2d_golden(oracle):
    c5 = _both(oracle, 2, 5, 1)[0, :, 0]
    assert c5[2] == 2.5
    np.testing.assert_allclose(c5[[0, 1, 3, 4]], [0.60392, 1.51253, 3.48747, 4.39608], rtol=1e-5)
    assert 2.5 - c5[0] == pytest.approx(abs(2.5 - c5[4]))
    c6 = _both(oracle, 2, 6, 1)[0, :, 0]
    np.testing.assert_allclose(c6, [0.61183, 1.52298, 2.50083, 3.49917, 4.47702, 5.38817],
                               rtol=1e-5)


def test_planar_coords_3d_golden(oracle):
    c = _both(oracle, 3, 5, 5).reshape(-1, 2)  # pixel index u + 5 v
    for k, idx in enumerate((2, 7, 12, 17, 22)):  # the centre column: x stays, y counts up
        assert c[idx, 0] == pytest.approx(2.5) and c[idx, 1] == pytest.approx(0.5 + k)
    assert 2.5 - c[20, 0] == pytest.approx(abs(2.5 - c[24, 0]))
    assert 2.5 - c[9, 1] == pytest.approx(abs(2.5 - c[19, 1]))
    assert c[1, 0] - c[0, 0] < c[2, 0] - c[1, 0]
    assert c[0, 1] < c[1, 1] and c[20, 1] > c[21, 1]
    c68 = _both(oracle, 3, 6, 8).reshape(-1, 2)
    assert 3 - c68[42, 0] == pytest.approx(abs(3 - c68[47, 0]))
    assert 4 - c68[5, 1] == pytest.approx(abs(4 - c68[47, 1]))
    assert c68[1, 0] - c68[0, 0] < c68[3, 0] - c68[2, 0]


def test_curved_argument_errors():
    with pytest.raises(elsa_b200.InvalidArgumentError):
        elsa_b200.curved_detector_coords(2, 5, 1, 0.0, 14.0)
    with pytest.raises(elsa_b200.InvalidArgumentError):
        elsa_b200.curved_detector_coords(2, 5, 1, 1.0, -3.0)


def test_pyelsa_curved_trajectory(oracle):
    import elsa_b200.pyelsa as elsa
    vol = elsa.VolumeDescriptor([16, 16, 16])
    d = elsa.CurvedCircleTrajectoryGenerator.createTrajectory(8, vol, 360, 160, 40, 0.5,
                                                              detectorSize=[24, 20])
    flat, _ = oracle.circle_trajectory((16, 16, 16), 8, 360, 160, 40, [24, 20])
    np.testing.assert_array_equal(d.poses, flat)  # same poses as the flat trajectory
    assert d.s2d == 200.0 and d.getRadius() == pytest.approx(48.0)
    coords = d.getPlanarCoords()
    assert len(coords) == 24 * 20
    np.testing.assert_allclose(coords[0], oracle.curved_coords(3, 24, 20, 0.5, 200.0)[0, 0],
                               rtol=0)
