"""Ordered-subset splits (projectors/SubsetSampler.cpp) through the C ABI (host only) and in the
oracle, against the golden mappings of the reference's tests/test_SubsetSampler.cpp, and the
oracle's SQS restatement on the reference's SQS test problem type (tests/test_SQS.cpp)."""
import numpy as np
import pytest

import elsa_b200


def _circle32(oracle):
    # CircleTrajectoryGenerator::createTrajectory(32, 32 x 32 volume, 360, 32 * 100, 32)
    return oracle.circle_trajectory((32, 32), 32, 360, 3200.0, 32.0)


@pytest.mark.parametrize("n_subsets", [4, 5])
def test_round_robin_golden(oracle, n_subsets):
    from oracle import solvers as S
    poses, _ = _circle32(oracle)
    for mapping in (elsa_b200.subset_split(2, poses, n_subsets, elsa_b200.SUBSET_ROUND_ROBIN),
                    S.subset_split_round_robin(range(32), n_subsets)):
        assert len(mapping) == n_subsets
        for i, part in enumerate(mapping):
            # test_SubsetSampler.cpp:47-82: 8 per subset for 4; 7, 7, 6, 6, 6 for 5
            want = 8 if n_subsets == 4 else (7 if i <= 1 else 6)
            assert len(part) == want
            assert part == [j * n_subsets + i for j in range(want)]


def test_rotational_clustering_golden(oracle):
    from oracle import solvers as S
    poses, _ = _circle32(oracle)
    golden = [[15, 11, 7, 3, 0, 27, 23, 19], [14, 10, 6, 2, 30, 26, 22, 18],
              [13, 9, 5, 1, 29, 25, 21, 17], [12, 8, 4, 31, 28, 24, 20, 16]]
    # test_SubsetSampler.cpp:84-97
    assert elsa_b200.subset_split(2, poses, 4, elsa_b200.SUBSET_ROTATIONAL_CLUSTERING) == golden
    assert S.subset_split_rotational(2, poses, 4) == golden


def test_rotational_clustering_3d_matches_oracle(oracle):
    """3D circle (distinct acos distances only for the first half-turn; the split still covers
    every pose once)."""
    from oracle import solvers as S
    poses, _ = oracle.circle_trajectory((16, 16, 16), 25, 180, 160.0, 40.0, [24, 24])
    got = elsa_b200.subset_split(3, poses, 3, elsa_b200.SUBSET_ROTATIONAL_CLUSTERING)
    assert sorted(v for part in got for v in part) == list(range(25))
    assert got == S.subset_split_rotational(3, poses, 3)


def test_split_argument_errors(oracle):
    poses, _ = _circle32(oracle)
    with pytest.raises(elsa_b200.InvalidArgumentError):
        elsa_b200.subset_split(2, poses, 1)  # nSubsets must be >= 2
    with pytest.raises(elsa_b200.InvalidArgumentError):
        elsa_b200.subset_split(2, poses, 4, strategy=7)
    with pytest.raises(elsa_b200.InvalidArgumentError):
        elsa_b200.subset_split(4, poses, 4)


@pytest.mark.parametrize("momentum", [True, False])
@pytest.mark.parametrize("precond", [False, True])
def test_oracle_sqs_solves_scaling_problem(momentum, precond):
    """test_SQS.cpp:19-90: LeastSquares(Scaling(|r|), b) on an 8 x 9 volume, 50 iterations
    (200 with JacobiPreconditioner(scaling, false), i.e. the diagonal |r| itself), converges:
    |A x - b|^2 == Approx(0), doctest's default epsilon of 100 FLT_EPSILON."""
    from oracle import solvers as S
    rng = np.random.default_rng(666)
    n = 72
    b = rng.uniform(-1, 1, n).astype(np.float32)
    # |U(-1, 1)| as the reference's setRandom().cwiseAbs(), kept in [0.25, 1] so that every
    # coordinate contracts within the iteration counts of the reference test
    a = (0.25 + 0.75 * np.abs(rng.uniform(-1, 1, n))).astype(np.float32)
    A = lambda v: (a * v).astype(np.float32)  # noqa: E731
    p = a if precond else None
    x, hist, stopped = S.sqs(A, A, b, n, 200 if precond else 50, momentum=momentum, precond=p)
    diff = A(x) - b
    assert float(np.dot(diff.astype(np.float64), diff)) <= 100 * np.finfo(np.float32).eps
    assert all(np.isfinite(hist))
