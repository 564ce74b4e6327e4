"""Host-side parts of the pyelsa-style API (no GPU): descriptors and trajectories."""
import numpy as np
import pytest


def test_descriptors_and_trajectory(oracle):
    import elsa_b200.pyelsa as elsa
    vol = elsa.VolumeDescriptor([64, 48, 32], [1.0, 1.0, 2.0])
    assert vol.getNumberOfDimensions() == 3
    assert vol.getNumberOfCoefficients() == 64 * 48 * 32
    np.testing.assert_allclose(vol.getLocationOfOrigin(), [32, 24, 32])
    sino = elsa.CircleTrajectoryGenerator.createTrajectory(20, vol, 200, 640, 160,
                                                           detectorSize=[96, 80])
    assert sino.shape == (96, 80, 20)
    assert sino.getNumberOfGeometryPoses() == 20
    poses, det = oracle.circle_trajectory((64, 48, 32), 20, 200, 640, 160, [96, 80],
                                          vol_spacing=[1.0, 1.0, 2.0])
    np.testing.assert_array_equal(sino.poses, poses)
    with pytest.raises(NotImplementedError):
        elsa.CircleTrajectoryGenerator.createTrajectory(4, vol, 360, 100, 10,
                                                        principalPointOffset=[1.0, 0.0])
    with pytest.raises(ValueError):
        elsa.VolumeDescriptor([0, 4])
