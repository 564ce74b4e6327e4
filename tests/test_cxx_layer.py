"""The header-only C++ layer (include/elsa_b200.hpp): compiles and links here; runs on the GPU
and agrees with the oracle."""
import os
import subprocess

import numpy as np
import pytest

import elsa_b200

from conftest import rel_l2


def test_cxx_layer_builds(tmp_path):
    from elsa_b200 import build as b
    b.build()
    import cxx_layer
    exe = cxx_layer.build(str(tmp_path))
    assert os.path.exists(exe)


def _load(tmp_path, name):
    return np.fromfile(tmp_path / name, np.float32)


@pytest.mark.gpu
def test_cxx_layer_runs(cuda, oracle, tmp_path):
    import cxx_layer
    from oracle import solvers as S
    exe = cxx_layer.build(str(tmp_path))
    out = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    fields = out.stdout.split()
    assert fields[0] == "ok" and fields[-1] == "1"  # the second autotune call hit the cache
    vol = (24, 24, 24)
    poses = _load(tmp_path, "poses.f32").reshape(-1, 40)
    det = (36, 36, 30)
    ref_poses, ref_det = oracle.circle_trajectory(vol, 30, 360, 240, 60, [36, 36])
    np.testing.assert_array_equal(poses, ref_poses)
    x = np.zeros((24, 24, 24), np.float32)
    x[6:18, 6:18, 6:18] = 1
    b_ref = oracle.joseph(x, vol, det, poses)
    b = _load(tmp_path, "sino.f32")
    assert rel_l2(b, b_ref) <= 1e-5
    # the solvers against the oracle on the same measurements
    A = lambda v: oracle.joseph(v, vol, det, poses)  # noqa: E731
    At = lambda v: oracle.joseph_adjoint(v, vol, det, poses)  # noqa: E731
    A64 = lambda v: oracle.joseph(v, vol, det, poses, dtype=np.float64)  # noqa: E731
    At64 = lambda v: oracle.joseph_adjoint(v, vol, det, poses, dtype=np.float64)  # noqa: E731
    n = x.size
    assert rel_l2(_load(tmp_path, "cgne.f32"), S.cgne(A, At, b, n, 8)[0]) <= 1e-4
    assert rel_l2(_load(tmp_path, "cgls.f32"), S.cgls(A, At, b, n, 8)[0]) <= 1e-4
    ref = S.apgd(A, At, b, n, 8, kind=1, lower=0.0)[0]
    assert rel_l2(_load(tmp_path, "apgd.f32"), ref) <= 1e-5
    assert rel_l2(_load(tmp_path, "sirt.f32"), S.sirt(A, At, b, n, 6)[0]) <= 1e-5
    for kind in ("fgm", "ogm"):
        xr = getattr(S, kind)(A, At, b, n, 6)[0]
        x64 = getattr(S, kind)(A64, At64, b, n, 6, dtype=np.float64)[0]
        assert rel_l2(_load(tmp_path, kind + ".f32"), xr) <= max(1e-4, 4 * rel_l2(xr, x64)), kind
    xr = S.sqs(A, At, b, n, 4)[0]
    x64 = S.sqs(A64, At64, b, n, 4, dtype=np.float64)[0]
    assert rel_l2(_load(tmp_path, "sqs.f32"), xr) <= max(1e-4, 4 * rel_l2(xr, x64))
    # ordered subsets (round robin, 3 subsets) with the Scaling preconditioner
    split = S.subset_split_round_robin(range(30), 3)
    views = b.reshape(30, -1)
    subsets, subsets64 = [], []
    for i, idx in enumerate(split):
        block = _load(tmp_path, "block%d.f32" % i)
        np.testing.assert_array_equal(block, views[idx].ravel())
        pm, dm = poses[idx], (36, 36, len(idx))
        subsets.append((lambda v, pm=pm, dm=dm: oracle.joseph(v, vol, dm, pm),
                        lambda v, pm=pm, dm=dm: oracle.joseph_adjoint(v, vol, dm, pm), block))
        subsets64.append((lambda v, pm=pm, dm=dm: oracle.joseph(v, vol, dm, pm, dtype=np.float64),
                          lambda v, pm=pm, dm=dm: oracle.joseph_adjoint(v, vol, dm, pm,
                                                                        dtype=np.float64),
                          block))
    diag = np.float32(0.5) + np.float32(0.5) * (np.arange(n) % 7).astype(np.float32) / \
        np.float32(6.0)
    xr = S.sqs(A, At, b, n, 3, subsets=subsets, precond=diag)[0]
    x64 = S.sqs(A64, At64, b, n, 3, subsets=subsets64, precond=diag, dtype=np.float64)[0]
    assert rel_l2(_load(tmp_path, "sqs_os.f32"), xr) <= max(1e-4, 4 * rel_l2(xr, x64))
    # BinaryMethod and the ray-driven LUT projectors
    xf = x.ravel()
    assert rel_l2(_load(tmp_path, "binary.f32"), oracle.binary(xf, vol, det, poses)) <= 1e-5
    ref = oracle.lut_project(False, xf, vol, det, poses, oracle.blob_lut(), 2.0, 2)
    assert rel_l2(_load(tmp_path, "rayblob.f32"), ref) <= 1e-5
    ref = oracle.lut_project(False, xf, vol, det, poses, oracle.bspline_lut(3, 2),
                             oracle.bspline_support(2), 2)
    assert rel_l2(_load(tmp_path, "raybspline.f32"), ref) <= 1e-5
    # Siddon's two adjoints: the same sums in another order
    ref = oracle.siddon_adjoint(b, vol, det, poses)
    for name in ("siddon_adj_scatter.f32", "siddon_adj_owner.f32"):
        assert rel_l2(_load(tmp_path, name), ref) <= 1e-5, name
    # the curved detector
    coords = oracle.curved_coords(3, 36, 36, 0.6, 300.0)
    np.testing.assert_array_equal(_load(tmp_path, "curved_coords.f32"),
                                  np.asarray(coords, np.float32).ravel())
    ref = oracle.joseph(xf, vol, det, poses, coords=coords)
    assert rel_l2(_load(tmp_path, "curved.f32"), ref) <= 1e-5
    # the fast flag: elsa's unmatched adjoint, close to but not the matched one
    fast, matched = _load(tmp_path, "fast_adjoint.f32"), _load(tmp_path, "matched_adjoint.f32")
    assert rel_l2(matched, oracle.joseph_adjoint(b, vol, det, poses)) <= 1e-5
    assert not np.array_equal(fast, matched)
    assert np.corrcoef(fast.astype(np.float64), matched.astype(np.float64))[0, 1] > 0.7
    # image files written by the C++ layer read back here
    data, dims, spacing, _ = elsa_b200.edf_read(str(tmp_path / "sino.edf"))
    assert dims == [36, 36, 30] and np.array_equal(data, b)
    data, dims, _, _ = elsa_b200.mhd_read(str(tmp_path / "sino.mhd"))
    assert dims == [36, 36, 30] and np.array_equal(data, b)
    assert open(tmp_path / "slice.pgm").read().startswith("P2\n24 24\n255\n")
