"""The header-only C++ layer (include/elsa_b200.hpp): compiles and links here; runs on the GPU
and agrees with the oracle."""
import os
import subprocess

import numpy as np
import pytest

from conftest import rel_l2


def test_cxx_layer_builds(tmp_path):
    from elsa_b200 import build as b
    b.build()
    import cxx_layer
    exe = cxx_layer.build(str(tmp_path))
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_cxx_layer_runs(cuda, oracle, tmp_path):
    import cxx_layer
    from oracle import solvers as S
    exe = cxx_layer.build(str(tmp_path))
    out = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.startswith("ok")
    vol = (24, 24, 24)
    poses = np.fromfile(tmp_path / "poses.f32", np.float32).reshape(-1, 40)
    det = (36, 36, 30)
    ref_poses, ref_det = oracle.circle_trajectory(vol, 30, 360, 240, 60, [36, 36])
    np.testing.assert_array_equal(poses, ref_poses)
    x = np.zeros((24, 24, 24), np.float32)
    x[6:18, 6:18, 6:18] = 1
    b = oracle.joseph(x, vol, det, poses)
    assert rel_l2(np.fromfile(tmp_path / "sino.f32", np.float32), b) <= 1e-5
    A = lambda v: oracle.joseph(v, vol, det, poses)  # noqa: E731
    At = lambda v: oracle.joseph_adjoint(v, vol, det, poses)  # noqa: E731
    n = x.size
    assert rel_l2(np.fromfile(tmp_path / "cgne.f32", np.float32), S.cgne(A, At, b, n, 8)[0]) <= 1e-4
    assert rel_l2(np.fromfile(tmp_path / "cgls.f32", np.float32), S.cgls(A, At, b, n, 8)[0]) <= 1e-4
    ref = S.apgd(A, At, b, n, 8, kind=1, lower=0.0)[0]
    assert rel_l2(np.fromfile(tmp_path / "apgd.f32", np.float32), ref) <= 1e-5
