"""Ray-driven blob / B-spline projector (elsa's LutProjector: BlobProjector, BSplineProjector) on
the GPU against the reference's test_LutProjector.cpp cases and the oracle's restatement."""
import numpy as np
import pytest

from conftest import rel_l2
from kat_cases import lut_cases

pytestmark = pytest.mark.gpu

PARITY = 1e-5


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


def test_lut_projector_kats_gpu(cuda, oracle):
    import elsa_b200
    bad = []
    for case in lut_cases(oracle):
        proj = elsa_b200.Projector(elsa_b200.PROJECTOR_RAY_BLOB, case["vol"], case["det"],
                                   case["poses"])
        y, _ = _pair(cuda, proj, case["x"], np.zeros(int(np.prod(case["det"])), np.float32))
        for got, want in zip(y, case["y_expect"]):
            got, want = float(got), float(want)
            if not abs(got - want) < case["tol"] * (1.0 + max(abs(got), abs(want))):
                bad.append((case["name"], got, want))
    assert not bad, bad[:10]


CONFIGS = {
    "fan2d_48": dict(vol=(48, 48), views=40, s2c=400, c2d=100, det=[68]),
    "cone3d_20": dict(vol=(20, 20, 20), views=12, s2c=200, c2d=50, det=[28, 28]),
}


@pytest.mark.parametrize("kind", ["blob", "bspline"])
@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_lut_projector_parity(cuda, oracle, name, kind):
    import elsa_b200
    c = CONFIGS[name]
    vol = c["vol"]
    dim = len(vol)
    poses, det = oracle.circle_trajectory(vol, c["views"], 360, c["s2c"], c["c2d"], c["det"])
    if kind == "blob":
        code, lut, radius, support = elsa_b200.PROJECTOR_RAY_BLOB, oracle.blob_lut(), 2.0, 2
    else:
        code, lut = elsa_b200.PROJECTOR_RAY_BSPLINE, oracle.bspline_lut(dim, 2)
        radius, support = oracle.bspline_support(2), 2
    proj = elsa_b200.Projector(code, vol, det, poses)
    rng = np.random.default_rng(8)
    x = rng.uniform(0, 1, int(np.prod(vol))).astype(np.float32)
    y = rng.uniform(0, 1, int(np.prod(det))).astype(np.float32)
    Ax, Aty = _pair(cuda, proj, x, y)
    ref_Ax = oracle.lut_project(False, x, vol, det, poses, lut, radius, support)
    ref_Aty = oracle.lut_project(True, y, vol, det, poses, lut, radius, support)
    # the forward sums every ray in the reference's order: bit-identical
    assert np.array_equal(Ax.view(np.uint32), np.asarray(ref_Ax, np.float32).view(np.uint32))
    assert rel_l2(Aty, ref_Aty) <= PARITY
    # fixed-point sums: the adjoint is deterministic
    _, Aty2 = _pair(cuda, proj, x, y)
    assert np.array_equal(Aty.view(np.uint32), Aty2.view(np.uint32))
    # the FP64 restatement bounds the float error of both
    ref64 = oracle.lut_project(True, y.astype(np.float64), vol, det, poses, lut, radius, support,
                               dtype=np.float64)
    assert rel_l2(Aty, ref64) <= PARITY


def test_lut_projector_arguments(cuda, oracle):
    import elsa_b200
    poses, det = oracle.circle_trajectory((16, 16), 8, 360, 160, 40, [24])
    with pytest.raises(elsa_b200.InvalidArgumentError):
        elsa_b200.Projector(elsa_b200.PROJECTOR_RAY_BLOB, (16, 16), det, poses,
                            [2.0, 10.83, 2.0, 0.0])
    with pytest.raises(elsa_b200.ElsaError):
        elsa_b200.Projector(elsa_b200.PROJECTOR_RAY_BSPLINE, (16, 16), det, poses,
                            curved=(0.5, 200.0))
