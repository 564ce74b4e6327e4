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


def test_subset_sampler_descriptors(oracle):
    """SubsetSampler (projectors/SubsetSampler.cpp:10-49): one detector descriptor per subset
    with that subset's poses, in the mapping's order (test_SubsetSampler.cpp's 20-view 2D
    case with 4 subsets)."""
    import elsa_b200.pyelsa as elsa
    vol = elsa.VolumeDescriptor([16, 16])
    sino = elsa.CircleTrajectoryGenerator.createTrajectory(20, vol, 360, 1600, 16)
    sampler = elsa.SubsetSampler(vol, sino, 4)
    mapping = sampler.getIndexMapping()
    assert mapping == elsa.SubsetSampler.splitRoundRobin(range(20), 4)
    for idx, d in zip(mapping, sampler.getSubsetDetectorDescriptors()):
        assert d.shape == (sino.shape[0], len(idx))
        np.testing.assert_array_equal(d.poses, sino.poses[idx])
    rot = elsa.SubsetSampler(vol, sino, 4, elsa.SubsetSampler.ROTATIONAL_CLUSTERING)
    assert sorted(v for m in rot.getIndexMapping() for v in m) == list(range(20))
    with pytest.raises(ValueError):
        elsa.SubsetSampler(vol, sino, 1)
