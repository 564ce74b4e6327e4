"""Ray-driven projectors on a curved detector (CurvedDetectorDescriptor) on the GPU against the
oracle's rays through the same planar pixel coordinates."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

PARITY = 1e-5

CONFIGS = {
    "fan2d_64": dict(vol=(64, 64), views=60, s2c=500, c2d=125, det=[92], angle=1.2),
    "cone3d_32": dict(vol=(32, 32, 32), views=24, s2c=320, c2d=80, det=[48, 40], angle=0.8),
}


def _pair(torch, proj, x, y):
    xd = torch.from_numpy(np.ascontiguousarray(x, np.float32).ravel()).cuda()
    yd = torch.from_numpy(np.ascontiguousarray(y, np.float32).ravel()).cuda()
    Ax = torch.full((proj.range_size,), float("nan"), device="cuda")
    Aty = torch.full((proj.domain_size,), float("nan"), device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    proj.apply_ptr(xd.data_ptr(), Ax.data_ptr(), s)
    proj.apply_adjoint_ptr(yd.data_ptr(), Aty.data_ptr(), s)
    torch.cuda.synchronize()
    return Ax.cpu().numpy(), Aty.cpu().numpy()


@pytest.mark.parametrize("kind", ["joseph", "siddon", "binary"])
@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_curved_parity(cuda, oracle, name, kind):
    import elsa_b200
    c = CONFIGS[name]
    vol = c["vol"]
    poses, det = oracle.circle_trajectory(vol, c["views"], 360, c["s2c"], c["c2d"], c["det"])
    s2d = float(np.float32(c["s2c"]) + np.float32(c["c2d"]))
    dim = len(vol)
    coords = oracle.curved_coords(dim, det[0], det[1] if dim == 3 else 1, c["angle"], s2d)
    code = {"joseph": elsa_b200.PROJECTOR_JOSEPH, "siddon": elsa_b200.PROJECTOR_SIDDON,
            "binary": elsa_b200.PROJECTOR_BINARY}[kind]
    proj = elsa_b200.Projector(code, vol, det, poses, curved=(c["angle"], s2d))
    rng = np.random.default_rng(4)
    x = rng.uniform(0, 1, int(np.prod(vol))).astype(np.float32)
    y = rng.uniform(0, 1, int(np.prod(det))).astype(np.float32)
    Ax, Aty = _pair(cuda, proj, x, y)
    fwd = getattr(oracle, kind)
    adj = getattr(oracle, kind + "_adjoint")
    ref_Ax = np.asarray(fwd(x, vol, det, poses, coords=coords), np.float32).ravel()
    ref_Aty = adj(y, vol, det, poses, coords=coords)
    assert rel_l2(Ax, ref_Ax) <= PARITY, (name, kind)
    assert rel_l2(Aty, ref_Aty) <= PARITY, (name, kind)
    if kind != "joseph":
        # thread-per-ray replay of the reference's float operations: bit-identical
        assert np.array_equal(Ax.view(np.uint32), ref_Ax.view(np.uint32))
    # the curvature changes the projection: the flat detector's result differs
    flat = np.asarray(fwd(x, vol, det, poses), np.float32).ravel()
    assert rel_l2(flat, ref_Ax) > 1e-4


def test_curved_voxel_projector_refused(cuda, oracle):
    import elsa_b200
    poses, det = oracle.circle_trajectory((16, 16, 16), 8, 360, 160, 40, [24, 24])
    with pytest.raises(elsa_b200.ElsaError):
        elsa_b200.Projector(elsa_b200.PROJECTOR_BLOB, (16, 16, 16), det, poses,
                            curved=(0.5, 200.0))


def test_pyelsa_curved_operator(cuda, oracle):
    import elsa_b200.pyelsa as elsa
    vol = elsa.VolumeDescriptor([24, 24, 24])
    sino = elsa.CurvedCircleTrajectoryGenerator.createTrajectory(20, vol, 360, 240, 60, 0.6,
                                                                 detectorSize=[36, 36])
    A = elsa.JosephsMethodCUDA(vol, sino)
    from elsa_b200 import phantoms
    x = phantoms.modified_shepp_logan((24, 24, 24)).reshape(-1)
    b = A.apply(elsa.DataContainer(cuda.from_numpy(x), vol))
    coords = oracle.curved_coords(3, 36, 36, 0.6, 300.0)
    ref = oracle.joseph(x, (24, 24, 24), list(sino.shape), sino.poses, coords=coords)
    assert rel_l2(b.tensor.cpu().numpy(), ref) <= PARITY
    sol = elsa.CGNE(A, b).solve(10)
    assert (A.apply(sol) - b).squaredL2Norm() < 0.1 * b.squaredL2Norm()
