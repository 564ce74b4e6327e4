"""SQS (solvers/SQS.cpp) on the device through the C ABI against the oracle's restatement
(oracle/solvers.py): the full problem and ordered subsets (SubsetSampler round robin and
rotational clustering), with and without momentum, with a diagonal preconditioner, and the
early stop."""
import numpy as np
import pytest

from conftest import record_parity, rel_l2

pytestmark = pytest.mark.gpu

# Device and FP32 oracle are both deterministic, so every distance is one fixed number, recorded
# with the FP32-FP64 distance (conftest.record_parity); every case meets the 1e-5 bound.
SQS_BOUNDS = {  # measured on a B200: 1.1e-7 to 2.8e-7 for every case
    ("full_momentum", "fan2d_64"): 1e-5, ("full_momentum", "cone3d_24"): 1e-5,
    ("full_plain", "fan2d_64"): 1e-5, ("full_plain", "cone3d_24"): 1e-5,
    ("os_round_robin", "fan2d_64"): 1e-5, ("os_round_robin", "cone3d_24"): 1e-5,
    ("os_rotational", "fan2d_64"): 1e-5, ("os_rotational", "cone3d_24"): 1e-5,
    ("preconditioned", "fan2d_64"): 1e-5, ("early_stop", "fan2d_64"): 1e-5,
}


def _check(case, name, x, xr, x64=None):
    bound = SQS_BOUNDS[(case, name)]
    e32 = rel_l2(x, xr)
    fields = dict(gpu_f32=e32, bound=bound)
    if x64 is not None:
        fields.update(gpu_f64=rel_l2(x, x64), f32_f64=rel_l2(xr, x64))
    record_parity("sqs_%s_%s" % (case, name), **fields)
    assert e32 <= bound, (case, name, e32, bound)


PROBLEMS = {
    "fan2d_64": dict(vol=(64, 64), views=90, s2c=500, c2d=125, det=[92]),
    "cone3d_24": dict(vol=(24, 24, 24), views=30, s2c=240, c2d=60, det=[36, 36]),
}


def _setup(torch, oracle, name, n_subsets=0, strategy=0):
    import elsa_b200
    from elsa_b200 import phantoms
    c = PROBLEMS[name]
    vol = c["vol"]
    poses, det = oracle.circle_trajectory(vol, c["views"], 360, c["s2c"], c["c2d"], c["det"])
    proj = elsa_b200.Projector(elsa_b200.PROJECTOR_JOSEPH, vol, det, poses)
    phantom = np.asarray(phantoms.modified_shepp_logan(tuple(reversed(vol))), np.float32).ravel()

    def ops(p, dtype=np.float32):
        d = list(det[:-1]) + [len(p)]
        A = lambda v: oracle.joseph(np.asarray(v, dtype), vol, d, p, dtype=dtype).ravel()  # noqa
        At = lambda v: oracle.joseph_adjoint(np.asarray(v, dtype), vol, d, p,  # noqa: E731
                                             dtype=dtype).ravel()
        return A, At

    A, At = ops(poses)
    b = A(phantom)
    view = int(np.prod(det[:-1]))
    parts = []
    if n_subsets:
        split = elsa_b200.subset_split(len(vol), poses, n_subsets, strategy)
        for idx in split:
            sp = np.ascontiguousarray(poses[idx])
            bm = np.concatenate([b[v * view:(v + 1) * view] for v in idx])
            parts.append((idx, sp, bm))
    return elsa_b200, proj, poses, det, b, phantom.size, A, At, ops, parts


def _device_sqs(torch, elsa_b200, proj, det, b, n, parts, iterations, momentum=True,
                epsilon=1.1920928955078125e-07, precond=None):
    s = torch.cuda.current_stream().cuda_stream
    bd = torch.from_numpy(np.ascontiguousarray(b, np.float32)).cuda()
    x = torch.full((n,), float("nan"), device="cuda")
    subsets, keep = [], []
    view = int(np.prod(det[:-1]))
    for idx, sp, _ in parts:
        pm = elsa_b200.Projector(elsa_b200.PROJECTOR_JOSEPH, proj.vol_dims,
                                 list(det[:-1]) + [len(idx)], sp)
        bm = torch.empty(len(idx) * view, device="cuda")
        elsa_b200.gather_views(bd.data_ptr(), view, idx, det[-1], bm.data_ptr(), s)
        subsets.append((pm, bm.data_ptr()))
        keep.append(bm)
    pd = None
    if precond is not None:
        pd = torch.from_numpy(np.ascontiguousarray(precond, np.float32)).cuda()
    sol = elsa_b200.Solver.sqs(proj, bd.data_ptr(), x.data_ptr(), subsets=subsets,
                               momentum=momentum, epsilon=epsilon,
                               preconditioner_ptr=pd.data_ptr() if pd is not None else None,
                               stream=s)
    sol.iterate(iterations, s)
    g2 = sol.squared_residual(s)
    torch.cuda.synchronize()
    out = x.cpu().numpy()
    sol.close()
    return out, g2, keep


@pytest.mark.parametrize("momentum", [True, False])
@pytest.mark.parametrize("name", sorted(PROBLEMS))
def test_sqs_full_problem(cuda, oracle, name, momentum):
    from oracle import solvers as S
    elsa_b200, proj, poses, det, b, n, A, At, ops, _ = _setup(cuda, oracle, name)
    x, g2, _ = _device_sqs(cuda, elsa_b200, proj, det, b, n, [], 8, momentum=momentum)
    xr, hist, _ = S.sqs(A, At, b, n, 8, momentum=momentum)
    A64, At64 = ops(poses, np.float64)
    x64, h64, _ = S.sqs(A64, At64, b, n, 8, momentum=momentum, dtype=np.float64)
    _check("full_momentum" if momentum else "full_plain", name, x, xr, x64)
    assert abs(g2 - hist[-1]) <= max(1e-3 * hist[-1], 4.0 * abs(hist[-1] - h64[-1]))


@pytest.mark.parametrize("strategy", [0, 1])
@pytest.mark.parametrize("name", sorted(PROBLEMS))
def test_sqs_ordered_subsets(cuda, oracle, name, strategy):
    from oracle import solvers as S
    elsa_b200, proj, poses, det, b, n, A, At, ops, parts = _setup(cuda, oracle, name, 3, strategy)
    x, g2, _ = _device_sqs(cuda, elsa_b200, proj, det, b, n, parts, 4)
    subs = [ops(sp) + (bm,) for _, sp, bm in parts]
    xr, hist, _ = S.sqs(A, At, b, n, 4, subsets=subs)
    subs64 = [ops(sp, np.float64) + (bm,) for _, sp, bm in parts]
    A64, At64 = ops(poses, np.float64)
    x64, _, _ = S.sqs(A64, At64, b, n, 4, subsets=subs64, dtype=np.float64)
    _check("os_rotational" if strategy else "os_round_robin", name, x, xr, x64)
    assert len(hist) == 12  # 4 iterations x 3 subsets
    assert abs(g2 - hist[-1]) <= 1e-3 * hist[-1] + 1e-30


def test_sqs_preconditioner(cuda, oracle):
    from oracle import solvers as S
    elsa_b200, proj, poses, det, b, n, A, At, ops, _ = _setup(cuda, oracle, "fan2d_64")
    rng = np.random.default_rng(3)
    p = rng.uniform(0.5, 1.5, n).astype(np.float32)
    x, _, _ = _device_sqs(cuda, elsa_b200, proj, det, b, n, [], 6, precond=p)
    xr, _, _ = S.sqs(A, At, b, n, 6, precond=p)
    A64, At64 = ops(poses, np.float64)
    x64, _, _ = S.sqs(A64, At64, b, n, 6, precond=p, dtype=np.float64)
    _check("preconditioned", "fan2d_64", x, xr, x64)


def test_sqs_early_stop(cuda, oracle):
    """A large epsilon stops both after the same number of steps (full problem: the device flag;
    subsets: the host's full-gradient confirmation); later iterations leave x unchanged."""
    from oracle import solvers as S
    elsa_b200, proj, poses, det, b, n, A, At, ops, parts = _setup(cuda, oracle, "fan2d_64", 3, 0)
    for use_parts in ([], parts):
        subs = [ops(sp) + (bm,) for _, sp, bm in use_parts] or None
        xr, hist, stopped = S.sqs(A, At, b, n, 30, subsets=subs, epsilon=0.3)
        assert stopped and len(hist) < 30 * max(1, len(use_parts))
        x, _, _ = _device_sqs(cuda, elsa_b200, proj, det, b, n, use_parts, 30, epsilon=0.3)
        _check("early_stop", "fan2d_64", x, xr)


def test_sqs_graph_and_batch(cuda, oracle):
    """Full-problem SQS runs as a CUDA graph and in solve_batch with the same result as the
    plain iterations; the subset form refuses graphs (it synchronizes on the host)."""
    elsa_b200, proj, poses, det, b, n, A, At, ops, parts = _setup(cuda, oracle, "cone3d_24", 2, 0)
    torch = cuda
    bd = torch.from_numpy(np.ascontiguousarray(b, np.float32)).cuda()
    s = torch.cuda.current_stream().cuda_stream
    xa = torch.zeros(n, device="cuda")
    xb = torch.zeros(n, device="cuda")
    sa = elsa_b200.Solver(elsa_b200.SOLVER_SQS, proj, bd.data_ptr(), xa.data_ptr(), stream=s)
    sa.iterate(5, s)
    sb = elsa_b200.Solver(elsa_b200.SOLVER_SQS, proj, bd.data_ptr(), xb.data_ptr(), stream=s)
    torch.cuda.synchronize()
    elsa_b200.solve_batch([sb], 5, 2)
    torch.cuda.synchronize()
    assert np.array_equal(xa.cpu().numpy(), xb.cpu().numpy())
    _, _, keep = _device_sqs(torch, elsa_b200, proj, det, b, n, parts, 1)
    view = int(np.prod(det[:-1]))
    subsets = []
    for idx, sp, _ in parts:
        pm = elsa_b200.Projector(elsa_b200.PROJECTOR_JOSEPH, proj.vol_dims,
                                 list(det[:-1]) + [len(idx)], sp)
        bm = torch.empty(len(idx) * view, device="cuda")
        elsa_b200.gather_views(bd.data_ptr(), view, idx, det[-1], bm.data_ptr(), s)
        subsets.append((pm, bm.data_ptr()))
        keep.append(bm)
    xc = torch.zeros(n, device="cuda")
    sc = elsa_b200.Solver.sqs(proj, bd.data_ptr(), xc.data_ptr(), subsets=subsets, stream=s)
    st = torch.cuda.Stream()
    with pytest.raises(elsa_b200.ElsaError):
        sc.iterate_graph(2, st.cuda_stream)
    for sol in (sa, sb, sc):
        sol.close()


def test_gather_views_and_errors(cuda, oracle):
    import elsa_b200
    torch = cuda
    sino = torch.arange(5 * 7, dtype=torch.float32, device="cuda")
    out = torch.empty(3 * 7, device="cuda")
    elsa_b200.gather_views(sino.data_ptr(), 7, [4, 0, 2], 5, out.data_ptr())
    torch.cuda.synchronize()
    ref = sino.cpu().numpy().reshape(5, 7)[[4, 0, 2]].ravel()
    assert np.array_equal(out.cpu().numpy(), ref)
    with pytest.raises(elsa_b200.InvalidArgumentError):
        elsa_b200.gather_views(sino.data_ptr(), 7, [5], 5, out.data_ptr())
    elsa_b200_, proj, poses, det, b, n, A, At, ops, _ = _setup(cuda, oracle, "fan2d_64")
    bd = torch.from_numpy(np.ascontiguousarray(b, np.float32)).cuda()
    x = torch.zeros(n, device="cuda")
    with pytest.raises(elsa_b200.InvalidArgumentError):  # one subset is not a split
        elsa_b200.Solver.sqs(proj, bd.data_ptr(), x.data_ptr(), subsets=[(proj, bd.data_ptr())])
    other = elsa_b200.Projector(elsa_b200.PROJECTOR_JOSEPH, (32, 32), [46, 10],
                                oracle.circle_trajectory((32, 32), 10, 360, 300, 80, [46])[0])
    with pytest.raises(elsa_b200.InvalidArgumentError):  # subset over another volume
        elsa_b200.Solver.sqs(proj, bd.data_ptr(), x.data_ptr(),
                             subsets=[(other, bd.data_ptr()), (other, bd.data_ptr())])
