"""Joseph projector on the GPU (through the C ABI) against the oracle and elsa's KATs."""
import numpy as np
import pytest

from conftest import rel_l2
from kat_cases import joseph_cases

pytestmark = pytest.mark.gpu

PARITY = 1e-5  # relative L2 vs the FP32 CPU path (the parity bound)


def _gpu_pair(torch, proj, x_np, y_np):
    """A x and A^T y computed on the device via elsa_projector_apply/_adjoint."""
    x = torch.from_numpy(np.ascontiguousarray(x_np, np.float32).ravel()).cuda()
    y = torch.from_numpy(np.ascontiguousarray(y_np, np.float32).ravel()).cuda()
    Ax = torch.empty(proj.range_size, dtype=torch.float32, device="cuda").fill_(np.nan)
    Aty = torch.empty(proj.domain_size, dtype=torch.float32, device="cuda").fill_(np.nan)
    s = torch.cuda.current_stream().cuda_stream
    proj.apply_ptr(x.data_ptr(), Ax.data_ptr(), s)
    proj.apply_adjoint_ptr(y.data_ptr(), Aty.data_ptr(), s)
    torch.cuda.synchronize()
    return Ax.cpu().numpy(), Aty.cpu().numpy()


def _projector(vol, det, poses):
    import elsa_b200
    return elsa_b200.Projector(elsa_b200.PROJECTOR_JOSEPH, vol, det, poses)


def test_joseph_kats_gpu(cuda, oracle):
    for case in joseph_cases(oracle):
        proj = _projector(case["vol"], case["det"], case["poses"])
        y, bp = _gpu_pair(cuda, proj, case["x"], case["y"])
        tol = case.get("tol", 1e-5)
        np.testing.assert_allclose(y, case["y_expect"], rtol=tol, err_msg=case["name"])
        assert rel_l2(bp, case["bp_expect"]) <= tol, case["name"]


CONFIGS = {
    # 2D fan beam, the 128^2 / 180 views / 182 pixels problem
    "fan2d_128": dict(vol=(128, 128), views=180, s2c=1000, c2d=250, det=[182]),
    # 3D cone beam, a reduced cone-beam case with the same source/detector ratios
    "cone3d_64": dict(vol=(64, 64, 64), views=60, s2c=640, c2d=160, det=[96, 96]),
    # non-cubic volume, anisotropic detector, short arc
    "cone3d_noncubic": dict(vol=(48, 40, 56), views=17, s2c=500, c2d=120, det=[80, 64],
                            arc=200),
}


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_joseph_parity(cuda, oracle, name):
    from elsa_b200 import phantoms
    c = CONFIGS[name]
    poses, det = oracle.circle_trajectory(c["vol"], c["views"], c.get("arc", 360), c["s2c"],
                                          c["c2d"], c["det"])
    proj = _projector(c["vol"], det, poses)
    rng = np.random.default_rng(7)
    shape = tuple(reversed(c["vol"]))
    if len(shape) == 3 and len(set(shape)) == 1:
        x = phantoms.modified_shepp_logan(shape)
    else:
        x = rng.uniform(0, 1, shape).astype(np.float32)
    y = rng.uniform(0, 1, int(np.prod(det))).astype(np.float32)
    Ax, Aty = _gpu_pair(cuda, proj, x, y)
    ref_Ax = oracle.joseph(x, c["vol"], det, poses)
    ref_Aty = oracle.joseph_adjoint(y, c["vol"], det, poses)
    e_fwd, e_adj = rel_l2(Ax, ref_Ax), rel_l2(Aty, ref_Aty)
    # the float64 instantiation of the oracle, for the record
    d_Ax = oracle.joseph(x.astype(np.float64), c["vol"], det, poses, dtype=np.float64)
    print("%s: fwd %.3g adj %.3g (vs f64 fwd %.3g), fallback tiles %d ppm"
          % (name, e_fwd, e_adj, rel_l2(Ax, d_Ax), proj.info(4)))
    assert proj.info(3) == 0  # no timed-out pipeline wait
    assert proj.info(8) == 0  # every tap lies in a brick whose ray window holds its ray
    assert e_fwd <= PARITY
    assert e_adj <= PARITY


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_joseph_adjointness_and_determinism(cuda, oracle, name):
    c = CONFIGS[name]
    poses, det = oracle.circle_trajectory(c["vol"], c["views"], c.get("arc", 360), c["s2c"],
                                          c["c2d"], c["det"])
    proj = _projector(c["vol"], det, poses)
    rng = np.random.default_rng(11)
    x = rng.uniform(0, 1, int(np.prod(c["vol"]))).astype(np.float32)
    y = rng.uniform(0, 1, int(np.prod(det))).astype(np.float32)
    Ax, Aty = _gpu_pair(cuda, proj, x, y)
    lhs = float(Ax.astype(np.float64) @ y)
    rhs = float(x.astype(np.float64) @ Aty)
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)
    # atomic-free adjoint and forward: bitwise reproducible
    Ax2, Aty2 = _gpu_pair(cuda, proj, x, y)
    assert np.array_equal(Aty.view(np.uint32), Aty2.view(np.uint32))
    assert np.array_equal(Ax.view(np.uint32), Ax2.view(np.uint32))


@pytest.mark.parametrize("views", [3, 20, 30])
def test_joseph_host_entry_points(cuda, oracle, views):
    """Host-buffer entry points: with enough views the 3D operator pipelines the copies of view
    groups with the kernels; the results equal the device entry points bit for bit (also with a
    one-chunk adjoint, which takes the plain path)."""
    import elsa_b200
    poses, det = oracle.circle_trajectory((32, 32, 32), views, 360, 320, 80, [48, 48])
    proj = _projector((32, 32, 32), det, poses)
    rng = np.random.default_rng(3)
    x = rng.uniform(0, 1, 32 ** 3).astype(np.float32)
    y = rng.uniform(0, 1, int(np.prod(det))).astype(np.float32)
    Ax, Aty = _gpu_pair(cuda, proj, x, y)
    assert np.array_equal(proj.apply_host(x), Ax)
    assert np.array_equal(proj.apply_adjoint_host(y), Aty)
    xp = cuda.from_numpy(x).pin_memory().numpy()  # page-locked buffers take the async copies
    yp = cuda.from_numpy(y).pin_memory().numpy()
    assert np.array_equal(proj.apply_host(xp), Ax)
    assert np.array_equal(proj.apply_adjoint_host(yp), Aty)
    proj.set_knob(elsa_b200.KNOB_ADJOINT_CHUNKS, 1)
    _, Aty1 = _gpu_pair(cuda, proj, x, y)
    assert np.array_equal(proj.apply_adjoint_host(y), Aty1)


@pytest.mark.slow
def test_joseph_full_size_subset(cuda, oracle):
    """256^3 volume, 384^2 detector, 8 of the 360 poses of the full cone-beam trajectory."""
    from elsa_b200 import phantoms
    vol = (256, 256, 256)
    poses, det = oracle.circle_trajectory(vol, 360, 360, 2560, 640, [384, 384])
    sel = np.array([0, 45, 90, 135, 180, 225, 300, 359])
    poses = np.ascontiguousarray(poses[sel])
    det = np.array([384, 384, len(sel)])
    proj = _projector(vol, det, poses)
    x = phantoms.modified_shepp_logan(vol)
    rng = np.random.default_rng(5)
    y = rng.uniform(0, 1, int(np.prod(det))).astype(np.float32)
    Ax, Aty = _gpu_pair(cuda, proj, x, y)
    assert rel_l2(Ax, oracle.joseph(x, vol, det, poses)) <= PARITY
    assert rel_l2(Aty, oracle.joseph_adjoint(y, vol, det, poses)) <= PARITY


def test_2d_adjoint_after_smaller_projector(cuda, oracle):
    """The 2D adjoint's shared-memory limit is a per-kernel device attribute: a projector with
    fewer views created later must not lower it below what an earlier one needs."""
    vol = (64, 64)
    poses, det = oracle.circle_trajectory(vol, 120, 360, 500, 125, [92])
    big = _projector(vol, det, poses)
    small_poses, small_det = oracle.circle_trajectory(vol, 10, 360, 500, 125, [92])
    small = _projector(vol, small_det, small_poses)
    rng = np.random.default_rng(5)
    y = rng.uniform(0, 1, big.range_size).astype(np.float32)
    x = rng.uniform(0, 1, big.domain_size).astype(np.float32)
    _, bp = _gpu_pair(cuda, big, x, y)
    assert rel_l2(bp, oracle.joseph_adjoint(y, vol, det, poses)) <= PARITY
    ys = rng.uniform(0, 1, small.range_size).astype(np.float32)
    _, bps = _gpu_pair(cuda, small, x, ys)
    assert rel_l2(bps, oracle.joseph_adjoint(ys, vol, small_det, small_poses)) <= PARITY


@pytest.mark.parametrize("vol,det,views", [((48, 40, 36), [64, 56], 30), ((100, 72), [150], 90)])
def test_fast_adjoint_mode(cuda, oracle, vol, det, views):
    """JosephsMethodCUDA(..., fast = true): the forward is unchanged, the adjoint is elsa's
    voxel-driven texture backprojection (not the transpose: compared loosely with the matched
    one here; tests/test_reference_cuda.py pins it on the reference's own kernel)."""
    import elsa_b200
    poses, dd = oracle.circle_trajectory(vol, views, 360, 10.0 * vol[0], 2.5 * vol[0], det)
    matched = _projector(vol, dd, poses)
    fast = elsa_b200.Projector(elsa_b200.PROJECTOR_JOSEPH, vol, dd, poses, [1.0])
    rng = np.random.default_rng(21)
    x = rng.uniform(0, 1, int(np.prod(vol))).astype(np.float32)
    y = rng.uniform(0, 1, int(np.prod(dd))).astype(np.float32)
    f0, a0 = _gpu_pair(cuda, matched, x, y)
    f1, a1 = _gpu_pair(cuda, fast, x, y)
    assert np.array_equal(f0.view(np.uint32), f1.view(np.uint32))
    assert np.all(np.isfinite(a1))
    assert np.corrcoef(a0.astype(np.float64), a1.astype(np.float64))[0, 1] > 0.7
    _, a2 = _gpu_pair(cuda, fast, x, y)  # no atomics: bit-reproducible
    assert np.array_equal(a1.view(np.uint32), a2.view(np.uint32))
    assert fast.knob_candidates(elsa_b200.KNOB_ADJOINT_CHUNKS) == []
    assert fast.knob_candidates(elsa_b200.KNOB_ADJOINT_SCATTER) == []
    assert fast.info(7) == 1


def test_fast_adjoint_arguments(cuda, oracle):
    import elsa_b200
    poses, dd = oracle.circle_trajectory((16, 16, 16), 8, 360, 160, 40, [24, 24])
    with pytest.raises(elsa_b200.InvalidArgumentError):
        elsa_b200.Projector(elsa_b200.PROJECTOR_JOSEPH, (16, 16, 16), dd, poses, [1.0, 0.0])
    with pytest.raises(elsa_b200.ElsaError):
        elsa_b200.Projector(elsa_b200.PROJECTOR_JOSEPH, (16, 16, 16), dd, poses, [1.0],
                            curved=(0.5, 200.0))


def test_bounded_wait_runs_out(cuda, oracle):
    """The TMA forward's barrier waits are bounded: with the copies withheld and a short limit
    every wait runs out, the kernel records bit 0 of the error word and returns, and the context
    stays usable: the next forward (copies restored) is correct and leaves the word at 0."""
    import elsa_b200
    vol = (32, 32, 32)
    poses, det = oracle.circle_trajectory(vol, 24, 360, 320, 80, [48, 48])
    proj = _projector(vol, det, poses)
    rng = np.random.default_rng(8)
    x = rng.uniform(0, 1, 32 ** 3).astype(np.float32)
    y = rng.uniform(0, 1, int(np.prod(det))).astype(np.float32)
    assert proj.info(3) == 0
    proj.wait_test(20000, True)  # ~10 microseconds per wait, no copies issued
    _gpu_pair(cuda, proj, x, y)
    assert proj.info(3) & 1
    proj.wait_test(0, False)  # default limit, copies issued; clears the error word
    assert proj.info(3) == 0
    Ax, _ = _gpu_pair(cuda, proj, x, y)
    assert proj.info(3) == 0
    assert rel_l2(Ax, oracle.joseph(x, vol, det, poses)) <= PARITY
    # projectors without bounded waits refuse the hook
    siddon = elsa_b200.Projector(elsa_b200.PROJECTOR_SIDDON, vol, det, poses)
    with pytest.raises(elsa_b200.ElsaError):
        siddon.wait_test(20000, True)


@pytest.mark.parametrize("vol,det,views", [((48, 48, 48), [72, 72], 36),
                                           ((40, 56, 72), [88, 64], 25)])
def test_checkpoint_depth_same_adjoint(cuda, oracle, vol, det, views):
    """Deeper checkpoint slabs (knob CHECKPOINT_DEPTH: less memory) give the same 3D matched
    adjoint bit for bit, in single and batched launches: a brick inside a slab catches up from the
    slab's checkpoint with the same float additions the ray would have made."""
    import elsa_b200
    torch = cuda
    n = max(vol)
    poses, dd = oracle.circle_trajectory(vol, views, 360, 10.0 * n, 2.5 * n, det)
    proj = _projector(vol, dd, poses)
    assert proj.knob(elsa_b200.KNOB_CHECKPOINT_DEPTH) == 16  # small problem: the default
    assert proj.knob_candidates(elsa_b200.KNOB_CHECKPOINT_DEPTH) == [16, 32, 64, 128]
    rng = np.random.default_rng(17)
    x = rng.uniform(0, 1, int(np.prod(vol))).astype(np.float32)
    y = rng.uniform(0, 1, proj.range_size).astype(np.float32)
    _, a16 = _gpu_pair(torch, proj, x, y)
    assert rel_l2(a16, oracle.joseph_adjoint(y, vol, dd, poses)) <= PARITY
    s = torch.cuda.current_stream().cuda_stream
    yb = torch.from_numpy(np.stack([y, y[::-1].copy()])).cuda()
    for cpd in (32, 64, 128):
        proj.set_knob(elsa_b200.KNOB_CHECKPOINT_DEPTH, cpd)
        assert proj.knob(elsa_b200.KNOB_CHECKPOINT_DEPTH) == cpd
        assert proj.info(8) == 0
        _, a = _gpu_pair(torch, proj, x, y)
        assert np.array_equal(a.view(np.uint32), a16.view(np.uint32)), cpd
        out = torch.full((2, proj.domain_size), np.nan, device="cuda")
        proj.apply_adjoint_batch_ptr(yb.data_ptr(), proj.range_size, out.data_ptr(),
                                     proj.domain_size, 2, s)
        torch.cuda.synchronize()
        assert np.array_equal(out[0].cpu().numpy().view(np.uint32), a16.view(np.uint32)), cpd
    with pytest.raises(elsa_b200.InvalidArgumentError):
        proj.set_knob(elsa_b200.KNOB_CHECKPOINT_DEPTH, 24)
