"""Blob / B-spline voxel projectors (absorption and phase contrast) on the GPU through the C ABI,
against the oracle (oracle/voxel_oracle.cpp) and elsa's known answers."""
import numpy as np
import pytest

from conftest import rel_l2
from kat_cases import voxel_cases

pytestmark = pytest.mark.gpu

PARITY = 1e-5  # relative L2 vs the FP32 CPU path

KINDS = {"blob": 2, "bspline": 3, "phase_blob": 4, "phase_bspline": 5}


def _pair(torch, proj, x_np, y_np):
    x = torch.from_numpy(np.ascontiguousarray(x_np, np.float32).ravel()).cuda()
    y = torch.from_numpy(np.ascontiguousarray(y_np, np.float32).ravel()).cuda()
    Ax = torch.full((proj.range_size,), np.nan, dtype=torch.float32, device="cuda")
    Aty = torch.full((proj.domain_size,), np.nan, dtype=torch.float32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    proj.apply_ptr(x.data_ptr(), Ax.data_ptr(), s)
    proj.apply_adjoint_ptr(y.data_ptr(), Aty.data_ptr(), s)
    torch.cuda.synchronize()
    return Ax.cpu().numpy(), Aty.cpu().numpy()


def _projector(name, vol, det, poses, mode=0):
    import elsa_b200
    params = (2.0, 10.83, 2.0, float(mode)) if name.endswith("blob") else (2.0, float(mode))
    return elsa_b200.Projector(KINDS[name], vol, det, poses, params)


def test_voxel_kats_gpu(cuda, oracle):
    """test_BlobVoxelProjector.cpp:25-244 (702 geometries, default blob)."""
    for c in voxel_cases(oracle):
        proj = _projector("blob", c["vol"], c["det"], c["poses"])
        y, _ = _pair(cuda, proj, c["x"], np.zeros(int(np.prod(c["det"])), np.float32))
        tol = c["rtol"] * np.abs(c["y_expect"]) + 1e-7
        assert np.all(np.abs(y - c["y_expect"]) <= tol), (c["name"], y, c["y_expect"])


CONFIGS = {
    "fan2d_96": dict(vol=(96, 96), views=90, det=[136]),
    "cone3d_40": dict(vol=(40, 40, 40), views=36, det=[60, 60]),
    "cone3d_noncubic": dict(vol=(36, 28, 44), views=15, det=[64, 48], arc=200),
}


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("name", sorted(KINDS))
@pytest.mark.parametrize("cfg", sorted(CONFIGS))
def test_voxel_parity(cuda, oracle, cfg, name, mode):
    c = CONFIGS[cfg]
    vol = c["vol"]
    n = vol[0]
    poses, det = oracle.circle_trajectory(vol, c["views"], c.get("arc", 360), 10.0 * n,
                                          2.5 * n, c["det"])
    proj = _projector(name, vol, det, poses, mode)
    rng = np.random.default_rng(21)
    x = rng.uniform(0, 1, int(np.prod(vol))).astype(np.float32)
    y = rng.uniform(0, 1, int(np.prod(det))).astype(np.float32)
    import elsa_b200
    Ax, Aty = _pair(cuda, proj, x, y)
    lut, support, wk = oracle.voxel_lut(name, len(vol))
    ref_Ax = oracle.voxel_project(False, x, vol, det, poses, lut, support, wk, mode)
    ref_Aty = oracle.voxel_project(True, y, vol, det, poses, lut, support, wk, mode)
    d_Ax = oracle.voxel_project(False, x, vol, det, poses, lut, support, wk, mode, np.float64)
    e_fwd, e_adj = rel_l2(Ax, ref_Ax), rel_l2(Aty, ref_Aty)
    # with exact weights the adjoint gathers in the reference's order with the reference's float
    # operations: bit-identical to the CPU loop
    assert proj.knob(elsa_b200.KNOB_EXACT_WEIGHTS) == 0  # default: the forward's weights
    proj.set_knob(elsa_b200.KNOB_EXACT_WEIGHTS, 1)
    _, Aty_exact = _pair(cuda, proj, x, y)
    mism = int(np.count_nonzero(Aty_exact.view(np.uint32) != ref_Aty.view(np.uint32)))
    print("%s %s mode %d: fwd %.3g adj %.3g (fwd vs f64 %.3g), exact-weight adjoint bit "
          "mismatches %d" % (cfg, name, mode, e_fwd, e_adj, rel_l2(Ax, d_Ax), mism))
    assert e_fwd <= PARITY
    assert e_adj <= PARITY
    assert mism == 0


@pytest.mark.parametrize("name", sorted(KINDS))
def test_voxel_adjointness(cuda, oracle, name):
    vol = (32, 32, 32)
    poses, det = oracle.circle_trajectory(vol, 24, 360, 320.0, 80.0, [48, 48])
    proj = _projector(name, vol, det, poses, 1)
    rng = np.random.default_rng(5)
    x = rng.uniform(0, 1, int(np.prod(vol))).astype(np.float32)
    y = rng.uniform(0, 1, int(np.prod(det))).astype(np.float32)
    Ax, Aty = _pair(cuda, proj, x, y)
    lhs = float(Ax.astype(np.float64) @ y)
    rhs = float(x.astype(np.float64) @ Aty)
    assert abs(lhs - rhs) <= 1e-5 * max(abs(lhs), np.abs(Ax).astype(np.float64) @ y)
    # the adjoint is deterministic
    _, Aty2 = _pair(cuda, proj, x, y)
    assert np.array_equal(Aty.view(np.uint32), Aty2.view(np.uint32))
