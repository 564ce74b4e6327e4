"""The native path of the view-sharded CGNE (the C ABI's split CGNE, NCCL all-reduces on the
solver stream) on one GPU as a one-rank group: bit-identical to the single-GPU CGNE session, and
against the oracle's single-process CGNE. Several ranks need several GPUs; the exchange logic is
covered with two gloo ranks in test_sharded_cpu.py."""
import os
import socket

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def test_sharded_cgne_native_one_rank(cuda, oracle):
    import torch
    import torch.distributed as dist
    import elsa_b200
    from elsa_b200 import phantoms
    from elsa_b200.sharded import ShardedCGNE, native_split
    from oracle import solvers as S
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        vol = (24, 24, 24)
        poses, det = oracle.circle_trajectory(vol, 30, 360, 240, 60, [36, 36])
        x = phantoms.modified_shepp_logan(vol).ravel()
        b = oracle.joseph(x, vol, det, poses)
        split, proj, (lo, hi) = native_split(elsa_b200.PROJECTOR_JOSEPH, vol, poses, det, 0, 1)
        assert (lo, hi) == (0, 30)
        bd = torch.from_numpy(b).cuda()
        solver = ShardedCGNE(split, bd)
        xs, hist = solver.solve(6)
        xs = xs.cpu().numpy()
        # one rank: the same kernels in the same order as the single-GPU session
        xd = torch.zeros(proj.domain_size, device="cuda")
        st = torch.cuda.current_stream().cuda_stream
        sess = elsa_b200.Solver(elsa_b200.SOLVER_CGNE, proj, bd.data_ptr(), xd.data_ptr(),
                                stream=st)
        sess.iterate(6, st)
        torch.cuda.synchronize()
        assert np.array_equal(xs, xd.cpu().numpy())
        assert hist[-1] == sess.squared_residual(st)
        sess.close()
        A = lambda v: oracle.joseph(v, vol, det, poses)  # noqa: E731
        At = lambda v: oracle.joseph_adjoint(v, vol, det, poses)  # noqa: E731
        xr, hr = S.cgne(A, At, b, int(np.prod(vol)), 6)
        assert rel_l2(xs, xr) <= 1e-5
        np.testing.assert_allclose(hist, hr, rtol=1e-3)
        split.close()
    finally:
        dist.destroy_process_group()
