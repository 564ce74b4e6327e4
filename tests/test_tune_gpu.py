"""The autotuner and the launch knobs on the GPU: every knob value computes the same operator
(checked against the oracle at the 1e-5 relative L2 bound, and against each other), the tuner
keeps a candidate, and a second projector of the same shape takes the cached choice."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

PARITY = 1e-5  # relative L2 vs the FP32 CPU path


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


def _case(oracle, kind, vol, views, det):
    import elsa_b200
    n = vol[0]
    poses, dd = oracle.circle_trajectory(vol, views, 360, 10.0 * n, 2.5 * n, det)
    proj = elsa_b200.Projector(kind, vol, dd, poses)
    rng = np.random.default_rng(11)
    x = rng.uniform(0, 1, int(np.prod(vol))).astype(np.float32)
    y = rng.uniform(0, 1, proj.range_size).astype(np.float32)
    if kind == elsa_b200.PROJECTOR_JOSEPH:
        ref = oracle.joseph(x, vol, dd, poses), oracle.joseph_adjoint(y, vol, dd, poses)
    elif kind == elsa_b200.PROJECTOR_SIDDON:
        ref = oracle.siddon(x, vol, dd, poses), oracle.siddon_adjoint(y, vol, dd, poses)
    else:
        lut, sup, wk = oracle.voxel_lut("blob", len(vol))
        ref = (oracle.voxel_project(False, x, vol, dd, poses, lut, sup, wk, 0),
               oracle.voxel_project(True, y, vol, dd, poses, lut, sup, wk, 0))
    return proj, x, y, ref


CASES = {
    "joseph3d": (0, (32, 32, 32), 24, [48, 48]),
    "joseph2d": (0, (64, 64), 90, [92]),
    "siddon3d": (1, (32, 32, 32), 24, [48, 48]),
    "siddon2d": (1, (64, 64), 90, [92]),
    "blob3d": (2, (16, 16, 16), 8, [24, 24]),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_every_knob_value_is_the_same_operator(cuda, oracle, name):
    import elsa_b200
    kind, vol, views, det = CASES[name]
    proj, x, y, (rf, ra) = _case(oracle, kind, vol, views, det)
    f0, a0 = _pair(cuda, proj, x, y)
    assert rel_l2(f0, rf) <= PARITY and rel_l2(a0, ra) <= PARITY
    tunable = 0
    for knob in (elsa_b200.KNOB_FORWARD_THREADS, elsa_b200.KNOB_ADJOINT_CHUNKS,
                 elsa_b200.KNOB_ADJOINT_THREADS, elsa_b200.KNOB_ADJOINT_SCATTER,
                 elsa_b200.KNOB_EXACT_WEIGHTS, elsa_b200.KNOB_CHECKPOINT_DEPTH):
        cands = proj.knob_candidates(knob)
        if not cands:
            continue
        tunable += 1
        default = proj.knob(knob)
        for v in cands:
            proj.set_knob(knob, v)
            assert proj.knob(knob) == v
            f, a = _pair(cuda, proj, x, y)
            assert rel_l2(f, rf) <= PARITY, (name, knob, v)
            assert rel_l2(a, ra) <= PARITY, (name, knob, v)
            if knob == elsa_b200.KNOB_FORWARD_THREADS:
                # the block size changes nothing in a thread-per-ray forward
                assert np.array_equal(f, f0), (name, v)
            if knob in (elsa_b200.KNOB_ADJOINT_THREADS, elsa_b200.KNOB_CHECKPOINT_DEPTH):
                assert np.array_equal(a, a0), (name, v)
            if knob in (elsa_b200.KNOB_ADJOINT_CHUNKS, elsa_b200.KNOB_ADJOINT_SCATTER):
                # only the order of the additions changes
                assert rel_l2(a, a0) <= 1e-6, (name, v)
            if knob == elsa_b200.KNOB_EXACT_WEIGHTS:
                # adjoint weights a few ulp apart (the forward adds with atomics: order varies)
                assert rel_l2(f, f0) <= 1e-6 and rel_l2(a, a0) <= 1e-6, (name, v)
        proj.set_knob(knob, default)
        with pytest.raises(elsa_b200.InvalidArgumentError):
            proj.set_knob(knob, max(cands) * 2 + 3)
    assert tunable >= 1, name


@pytest.mark.parametrize("name", sorted(CASES))
def test_autotune_and_cache(cuda, oracle, name):
    import elsa_b200
    kind, vol, views, det = CASES[name]
    elsa_b200.tune_cache_clear()
    proj, x, y, (rf, ra) = _case(oracle, kind, vol, views, det)
    s = cuda.cuda.current_stream().cuda_stream
    values, hit = proj.autotune(s)
    assert not hit
    for k, key in enumerate(elsa_b200._capi.KNOB_NAMES):
        cands = proj.knob_candidates(k)
        if cands:
            assert values[key] in cands
        assert proj.knob(k) == values[key]
    f, a = _pair(cuda, proj, x, y)
    assert rel_l2(f, rf) <= PARITY and rel_l2(a, ra) <= PARITY
    assert elsa_b200.tune_cache_size() == 1
    # a second projector of the same shape takes the cached values without timing
    proj2, _, _, _ = _case(oracle, kind, vol, views, det)
    values2, hit2 = proj2.autotune(s)
    assert hit2 and values2 == values
    values3, hit3 = proj2.autotune(s, force=True)
    assert not hit3
    proj.close()
    proj2.close()
    elsa_b200.tune_cache_clear()
