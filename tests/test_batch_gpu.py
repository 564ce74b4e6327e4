"""Graph-captured solver iterations and batched concurrent solves: bit-identical to plain
iterations for the deterministic projectors (the graph replays the same launches; streams only
change the overlap). The voxel projectors' forward adds with float atomics, so there the batched
iterate agrees to rounding only."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _instances(oracle, torch, kinds):
    import elsa_b200
    from elsa_b200 import phantoms
    out = []
    rng = np.random.default_rng(7)
    for i, (kind, n) in enumerate(kinds):
        views = int(rng.integers(20, 60))
        poses, det = oracle.circle_trajectory((n, n, n), views, 360, 10.0 * n, 2.5 * n,
                                              [int(1.5 * n), int(1.5 * n)])
        proj = elsa_b200.Projector(kind, (n, n, n), det, poses)
        x = torch.from_numpy(phantoms.modified_shepp_logan((n, n, n)).reshape(-1)).cuda()
        b = torch.empty(proj.range_size, dtype=torch.float32, device="cuda")
        proj.apply_ptr(x.data_ptr(), b.data_ptr(), torch.cuda.current_stream().cuda_stream)
        out.append((proj, b))
    torch.cuda.synchronize()
    return out


def _solvers(torch, insts, kind):
    import elsa_b200
    s = torch.cuda.current_stream().cuda_stream
    xs, solvers = [], []
    for proj, b in insts:
        x = torch.zeros(proj.domain_size, dtype=torch.float32, device="cuda")
        solvers.append(elsa_b200.Solver(kind, proj, b.data_ptr(), x.data_ptr(), stream=s))
        xs.append(x)
    torch.cuda.synchronize()
    return xs, solvers


@pytest.mark.parametrize("solver_kind", [0, 1])  # CGNE, CGLS
def test_batch_matches_plain(cuda, oracle, solver_kind):
    import elsa_b200
    torch = cuda
    kinds = [(elsa_b200.PROJECTOR_JOSEPH, 24), (elsa_b200.PROJECTOR_JOSEPH, 32),
             (elsa_b200.PROJECTOR_SIDDON, 24), (elsa_b200.PROJECTOR_JOSEPH, 40),
             (elsa_b200.PROJECTOR_BLOB, 16)]
    insts = _instances(oracle, torch, kinds)
    xs_plain, plain = _solvers(torch, insts, solver_kind)
    s = torch.cuda.current_stream().cuda_stream
    for sol in plain:
        sol.iterate(6, s)
    torch.cuda.synchronize()
    xs_batch, batch = _solvers(torch, insts, solver_kind)
    elsa_b200.solve_batch(batch, 6, streams=3)
    _compare(kinds, xs_plain, xs_batch)
    # more graph launches continue the iteration exactly like plain iterations
    elsa_b200.solve_batch(batch, 4, streams=2)
    for sol in plain:
        sol.iterate(4, s)
    torch.cuda.synchronize()
    _compare(kinds, xs_plain, xs_batch)


def _compare(kinds, xs_plain, xs_batch):
    import elsa_b200
    for (kind, _), a, b in zip(kinds, xs_plain, xs_batch):
        if kind == elsa_b200.PROJECTOR_JOSEPH:
            assert bool((a == b).all()), kind
        else:
            # Siddon's default adjoint scatters with atomics: the order of its additions varies
            assert float((a - b).norm() / a.norm()) <= 1e-4, kind


def test_graph_needs_created_stream(cuda, oracle):
    import elsa_b200
    torch = cuda
    insts = _instances(oracle, torch, [(elsa_b200.PROJECTOR_JOSEPH, 16)])
    _, (sol,) = _solvers(torch, insts, 0)
    with pytest.raises(elsa_b200.InvalidArgumentError):
        sol.iterate_graph(2, 0)
    st = torch.cuda.Stream()
    sol.iterate_graph(2, st.cuda_stream)
    st.synchronize()


@pytest.mark.parametrize("graph", [False, True])
def test_batched_cgne_matches_plain_sessions(cuda, oracle, graph):
    """elsa_batch_cgne (forwards side by side, every adjoint in one launch per axis grid over an
    instance table, vector updates batched): each instance's iterate equals that of its own
    CGNE session bit for bit, also across further iterations and as one CUDA graph."""
    import elsa_b200
    torch = cuda
    J = elsa_b200.PROJECTOR_JOSEPH
    kinds = [(J, 24), (J, 40), (J, 16), (J, 32), (J, 24), (J, 48)]
    insts = _instances(oracle, torch, kinds)
    xs_plain, plain = _solvers(torch, insts, 0)
    s = torch.cuda.current_stream().cuda_stream
    for sol in plain:
        sol.iterate(5, s)
    torch.cuda.synchronize()
    xs = [torch.full((p.domain_size,), np.nan, device="cuda") for p, _ in insts]
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        batch = elsa_b200.BatchCGNE([p for p, _ in insts], [b.data_ptr() for _, b in insts],
                                    [x.data_ptr() for x in xs], st.cuda_stream)
        (batch.iterate_graph if graph else batch.iterate)(5, st.cuda_stream)
    st.synchronize()
    for a, b in zip(xs_plain, xs):
        assert bool((a == b).all())
    res = batch.squared_residuals(st.cuda_stream)
    for r, sol in zip(res, plain):
        assert r == sol.squared_residual(s)
    with torch.cuda.stream(st):
        (batch.iterate_graph if graph else batch.iterate)(3, st.cuda_stream)
    st.synchronize()
    for sol in plain:
        sol.iterate(3, s)
    torch.cuda.synchronize()
    for a, b in zip(xs_plain, xs):
        assert bool((a == b).all())
    batch.close()


def test_batched_cgne_refuses_other_operators(cuda, oracle):
    import elsa_b200
    torch = cuda
    insts = _instances(oracle, torch, [(elsa_b200.PROJECTOR_JOSEPH, 16),
                                       (elsa_b200.PROJECTOR_SIDDON, 16)])
    xs = [torch.zeros(p.domain_size, device="cuda") for p, _ in insts]
    with pytest.raises(elsa_b200.ElsaError):
        elsa_b200.BatchCGNE([p for p, _ in insts], [b.data_ptr() for _, b in insts],
                            [x.data_ptr() for x in xs])


def test_batched_cgne_deep_checkpoints_and_knob_guard(cuda, oracle):
    """Instances with deeper checkpoint slabs (less memory) batch like the others: the same
    iterates as their plain sessions. While a batch holds an operator its adjoint knobs are
    fixed (the batch points into its tables); closing the batch releases them."""
    import elsa_b200
    torch = cuda
    J = elsa_b200.PROJECTOR_JOSEPH
    insts = _instances(oracle, torch, [(J, 24), (J, 40), (J, 32)])
    insts[1][0].set_knob(elsa_b200.KNOB_CHECKPOINT_DEPTH, 64)
    insts[2][0].set_knob(elsa_b200.KNOB_CHECKPOINT_DEPTH, 32)
    xs_plain, plain = _solvers(torch, insts, 0)
    s = torch.cuda.current_stream().cuda_stream
    for sol in plain:
        sol.iterate(4, s)
    torch.cuda.synchronize()
    xs = [torch.zeros(p.domain_size, device="cuda") for p, _ in insts]
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        batch = elsa_b200.BatchCGNE([p for p, _ in insts], [b.data_ptr() for _, b in insts],
                                    [x.data_ptr() for x in xs], st.cuda_stream)
        batch.iterate(4, st.cuda_stream)
    st.synchronize()
    for a, b in zip(xs_plain, xs):
        assert bool((a == b).all())
    for p, _ in insts:
        with pytest.raises(elsa_b200.InvalidArgumentError):
            p.set_knob(elsa_b200.KNOB_CHECKPOINT_DEPTH, 128)
    batch.close()
    for sol in plain:
        sol.close()
    insts[0][0].set_knob(elsa_b200.KNOB_CHECKPOINT_DEPTH, 128)  # released
    assert insts[0][0].knob(elsa_b200.KNOB_CHECKPOINT_DEPTH) == 128
