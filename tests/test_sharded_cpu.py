"""View-sharded CGNE (elsa_b200.sharded) with two gloo ranks on CPU, the projections done by the
oracle on each rank's block of views, against a single-process CGNE over all views."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _problem():
    from oracle import oracle as O
    from elsa_b200 import phantoms
    vol = (20, 20, 20)
    poses, det = O.circle_trajectory(vol, 18, 360, 200, 50, [30, 30])
    x = phantoms.modified_shepp_logan(vol).ravel()
    b = O.joseph(x, vol, det, poses)
    return O, vol, poses, det, b


def _rank_main(rank, world, port, out_path):
    import torch
    import torch.distributed as dist
    from elsa_b200.sharded import ShardedCGNE, TorchSplitCGNE, view_block
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        O, vol, poses, det, b = _problem()
        lo, hi = view_block(len(poses), rank, world)
        dloc = [int(det[0]), int(det[1]), hi - lo]
        ploc = np.ascontiguousarray(poses[lo:hi])
        npix = int(det[0] * det[1])
        b_loc = torch.from_numpy(np.ascontiguousarray(b[lo * npix:hi * npix]))

        def fwd(v):
            return torch.from_numpy(O.joseph(v.numpy(), vol, dloc, ploc))

        def adj(y):
            return torch.from_numpy(O.joseph_adjoint(y.numpy(), vol, dloc, ploc))

        solver = ShardedCGNE(TorchSplitCGNE(fwd, adj, int(np.prod(vol))), b_loc)
        x, hist = solver.solve(6)
        if rank == 0:
            np.savez(out_path, x=x.numpy(), hist=np.array(hist))
        else:
            np.savez(out_path + ".r1", x=x.numpy())
    finally:
        dist.destroy_process_group()


def test_view_block_partition():
    from elsa_b200.sharded import view_block
    for n, w in ((360, 8), (17, 4), (5, 5), (3, 3)):
        blocks = [view_block(n, r, w) for r in range(w)]
        assert blocks[0][0] == 0 and blocks[-1][1] == n
        assert all(blocks[i][1] == blocks[i + 1][0] for i in range(w - 1))
        sizes = [hi - lo for lo, hi in blocks]
        assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1
    with pytest.raises(ValueError, match="at least one view per rank"):
        view_block(3, 0, 4)


def test_sharded_cgne_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    from oracle import solvers as S
    from conftest import rel_l2
    out = str(tmp_path / "rank0.npz")
    mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True,
                       start_method="spawn")
    res = np.load(out)
    res1 = np.load(out + ".r1.npz")
    # replicated iterates stay identical on every rank
    assert np.array_equal(res["x"], res1["x"])
    O, vol, poses, det, b = _problem()
    A = lambda v: O.joseph(v, vol, det, poses)  # noqa: E731
    At = lambda v: O.joseph_adjoint(v, vol, det, poses)  # noqa: E731
    xr, hist = S.cgne(A, At, b, int(np.prod(vol)), 6)
    assert rel_l2(res["x"], xr) <= 1e-4
    np.testing.assert_allclose(res["hist"], hist, rtol=1e-3)
