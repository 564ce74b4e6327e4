"""Siddon projector on the GPU (through the C ABI) against the oracle and elsa's KATs."""
import numpy as np
import pytest

from conftest import rel_l2
from kat_cases import siddon_cases

pytestmark = pytest.mark.gpu

PARITY = 1e-5  # relative L2 vs the FP32 CPU path


def _gpu_pair(torch, proj, x_np, y_np):
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
    return elsa_b200.Projector(elsa_b200.PROJECTOR_SIDDON, vol, det, poses)


def test_siddon_kats_gpu(cuda, oracle):
    for case in siddon_cases(oracle):
        proj = _projector(case["vol"], case["det"], case["poses"])
        y, bp = _gpu_pair(cuda, proj, case["x"], case["y"])
        np.testing.assert_allclose(y, case["y_expect"], rtol=1e-5, err_msg=case["name"])
        assert rel_l2(bp, case["bp_expect"]) <= 1e-5, case["name"]


CONFIGS = {
    "fan2d_128": dict(vol=(128, 128), views=180, s2c=1000, c2d=250, det=[182]),
    "cone3d_64": dict(vol=(64, 64, 64), views=60, s2c=640, c2d=160, det=[96, 96]),
    "cone3d_noncubic": dict(vol=(48, 40, 56), views=17, s2c=500, c2d=120, det=[80, 64],
                            arc=200),
}


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_siddon_parity(cuda, oracle, name):
    from elsa_b200 import phantoms
    c = CONFIGS[name]
    poses, det = oracle.circle_trajectory(c["vol"], c["views"], c.get("arc", 360), c["s2c"],
                                          c["c2d"], c["det"])
    proj = _projector(c["vol"], det, poses)
    rng = np.random.default_rng(9)
    shape = tuple(reversed(c["vol"]))
    if len(shape) == 3 and len(set(shape)) == 1:
        x = phantoms.modified_shepp_logan(shape)
    else:
        x = rng.uniform(0, 1, shape).astype(np.float32)
    y = rng.uniform(0, 1, int(np.prod(det))).astype(np.float32)
    Ax, Aty = _gpu_pair(cuda, proj, x, y)
    ref_Ax = oracle.siddon(x, c["vol"], det, poses)
    ref_Aty = oracle.siddon_adjoint(y, c["vol"], det, poses)
    d_Ax = oracle.siddon(x.astype(np.float64), c["vol"], det, poses, dtype=np.float64)
    e_fwd, e_adj = rel_l2(Ax, ref_Ax), rel_l2(Aty, ref_Aty)
    print("%s: fwd %.3g adj %.3g (vs f64 fwd %.3g), class spacing %d, visits %d"
          % (name, e_fwd, e_adj, rel_l2(Ax, d_Ax), proj.info(0), proj.info(2)))
    assert e_fwd <= PARITY
    assert e_adj <= PARITY
    # the forward replays the reference's float operations: bit-identical sums
    mism = int(np.count_nonzero(Ax.view(np.uint32) !=
                                np.asarray(ref_Ax, np.float32).ravel().view(np.uint32)))
    print("%s: forward values differing from the oracle in any bit: %d of %d"
          % (name, mism, Ax.size))
    assert mism == 0


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_siddon_adjointness_and_determinism(cuda, oracle, name):
    c = CONFIGS[name]
    poses, det = oracle.circle_trajectory(c["vol"], c["views"], c.get("arc", 360), c["s2c"],
                                          c["c2d"], c["det"])
    proj = _projector(c["vol"], det, poses)
    rng = np.random.default_rng(12)
    x = rng.uniform(0, 1, int(np.prod(c["vol"]))).astype(np.float32)
    y = rng.uniform(0, 1, int(np.prod(det))).astype(np.float32)
    import elsa_b200
    assert proj.knob(elsa_b200.KNOB_ADJOINT_SCATTER) == 0  # default: the brick owner
    proj.set_knob(elsa_b200.KNOB_ADJOINT_SCATTER, 1)
    Ax, Aty = _gpu_pair(cuda, proj, x, y)  # the scatter adjoint
    lhs = float(Ax.astype(np.float64) @ y)
    rhs = float(x.astype(np.float64) @ Aty)
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)
    # the brick-owner adjoint is bit-reproducible; the forward always is
    proj.set_knob(elsa_b200.KNOB_ADJOINT_SCATTER, 0)
    assert proj.info(8) == 0  # every visit lies in a brick whose ray window holds its ray
    Ax1, Aty1 = _gpu_pair(cuda, proj, x, y)
    Ax2, Aty2 = _gpu_pair(cuda, proj, x, y)
    assert np.array_equal(Aty1.view(np.uint32), Aty2.view(np.uint32))
    assert np.array_equal(Ax.view(np.uint32), Ax2.view(np.uint32))
    assert rel_l2(Aty, Aty1) <= 1e-6
    # visit count agrees with the oracle's crossing count
    assert proj.info(2) == oracle.siddon_visit_count(c["vol"], det, poses)


@pytest.mark.parametrize("binary", [False, True])
@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_scatter_adjoint_parity(cuda, oracle, name, binary):
    """The atomic-scatter adjoint (knob ADJOINT_SCATTER = 1) against the oracle and the
    deterministic brick-owner adjoint: the same sums in another order."""
    import elsa_b200
    c = CONFIGS[name]
    poses, det = oracle.circle_trajectory(c["vol"], c["views"], c.get("arc", 360), c["s2c"],
                                          c["c2d"], c["det"])
    kind = elsa_b200.PROJECTOR_BINARY if binary else elsa_b200.PROJECTOR_SIDDON
    proj = elsa_b200.Projector(kind, c["vol"], det, poses)
    rng = np.random.default_rng(13)
    x = rng.uniform(0, 1, int(np.prod(c["vol"]))).astype(np.float32)
    y = rng.uniform(0, 1, int(np.prod(det))).astype(np.float32)
    y[::7] = 0.0  # rays with nothing to add are skipped
    assert proj.knob(elsa_b200.KNOB_ADJOINT_SCATTER) == 0  # default: the brick owner
    proj.set_knob(elsa_b200.KNOB_ADJOINT_SCATTER, 1)  # releases the owner's tables
    assert proj.info(7) == 1
    assert proj.knob_candidates(elsa_b200.KNOB_ADJOINT_CHUNKS) == []
    _, a_scatter = _gpu_pair(cuda, proj, x, y)
    proj.set_knob(elsa_b200.KNOB_ADJOINT_SCATTER, 0)  # builds the brick-owner adjoint
    assert proj.knob_candidates(elsa_b200.KNOB_ADJOINT_CHUNKS)
    _, a_owner = _gpu_pair(cuda, proj, x, y)
    adj = oracle.binary_adjoint if binary else oracle.siddon_adjoint
    ref = adj(y, c["vol"], det, poses)
    assert rel_l2(a_scatter, ref) <= PARITY, name
    assert rel_l2(a_scatter, a_owner) <= 1e-6, name
    assert rel_l2(a_owner, ref) <= PARITY, name
    # back to scatter (the owner's buffers are released) and once more to the owner
    proj.set_knob(elsa_b200.KNOB_ADJOINT_SCATTER, 1)
    _, a_again = _gpu_pair(cuda, proj, x, y)
    assert rel_l2(a_again, a_scatter) <= 1e-6, name
    proj.set_knob(elsa_b200.KNOB_ADJOINT_SCATTER, 0)
    _, a_back = _gpu_pair(cuda, proj, x, y)
    assert np.array_equal(a_back.view(np.uint32), a_owner.view(np.uint32))


def test_siddon_cgls(cuda, oracle):
    """CGLS through the Siddon operator against the oracle restatement."""
    import elsa_b200
    from elsa_b200 import phantoms
    from oracle import solvers as S
    vol = (24, 24, 24)
    poses, det = oracle.circle_trajectory(vol, 30, 360, 240, 60, [36, 36])
    proj = _projector(vol, det, poses)
    x_true = np.asarray(phantoms.modified_shepp_logan(vol), np.float32).ravel()
    A = lambda v: oracle.siddon(v, vol, det, poses).ravel()  # noqa: E731
    At = lambda v: oracle.siddon_adjoint(v, vol, det, poses).ravel()  # noqa: E731
    b_np = A(x_true)
    torch = cuda
    b = torch.from_numpy(b_np).cuda()
    x = torch.zeros(proj.domain_size, dtype=torch.float32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    solver = elsa_b200.Solver(elsa_b200.SOLVER_CGLS, proj, b.data_ptr(), x.data_ptr(), stream=s)
    solver.iterate(8, s)
    torch.cuda.synchronize()
    xr, _ = S.cgls(A, At, b_np, x_true.size, 8)
    assert rel_l2(x.cpu().numpy(), xr) <= 1e-4


def test_binary_kats_gpu(cuda, oracle):
    """BinaryMethod (the Siddon kernels with weight 1) against test_BinaryMethod.cpp's cases:
    exact, both directions."""
    import elsa_b200
    from kat_cases import binary_cases
    for case in binary_cases(oracle):
        proj = elsa_b200.Projector(elsa_b200.PROJECTOR_BINARY, case["vol"], case["det"],
                                   case["poses"])
        y, bp = _gpu_pair(cuda, proj, case["x"], case["y"])
        np.testing.assert_array_equal(y, case["y_expect"], err_msg=case["name"])
        np.testing.assert_array_equal(bp.reshape(case["bp_expect"].shape), case["bp_expect"],
                                      err_msg=case["name"])


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_binary_parity(cuda, oracle, name):
    """Forward bit-identical to the oracle (same visits and float sums), adjoint within 1e-5
    (the oracle adds with atomics in varying order)."""
    import elsa_b200
    c = CONFIGS[name]
    poses, det = oracle.circle_trajectory(c["vol"], c["views"], c.get("arc", 360), c["s2c"],
                                          c["c2d"], c["det"])
    proj = elsa_b200.Projector(elsa_b200.PROJECTOR_BINARY, c["vol"], det, poses)
    rng = np.random.default_rng(21)
    x = rng.uniform(0, 1, int(np.prod(c["vol"]))).astype(np.float32)
    y = rng.uniform(0, 1, int(np.prod(det))).astype(np.float32)
    Ax, Aty = _gpu_pair(cuda, proj, x, y)
    ref_Ax = np.asarray(oracle.binary(x, c["vol"], det, poses), np.float32).ravel()
    ref_Aty = oracle.binary_adjoint(y, c["vol"], det, poses)
    assert np.array_equal(Ax.view(np.uint32), ref_Ax.view(np.uint32))
    assert rel_l2(Aty, ref_Aty) <= PARITY
    # adjointness <A x, y> = <x, A^T y>
    lhs = float(np.dot(Ax.astype(np.float64), y))
    rhs = float(np.dot(x.astype(np.float64), Aty))
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)
