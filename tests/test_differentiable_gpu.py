"""Batched applies and the differentiable projector at the size of the batched configuration:
8 volumes of 128^3 seeded random ellipsoids, 180 views, 192^2 detector (source-centre 1280,
centre-detector 320), loss 0.5 |A x - y|^2 through torch autograd.

* elsa_projector_apply_batch / _adjoint_batch equal the single applies bit for bit;
* the batch gradient equals the FP64 oracle's A^T (A x - y) (relative L2 <= 1e-5 per volume);
* 16 seeded central differences (eps = 1e-3) of the FP64 oracle loss agree with <grad, d>;
* a 10-step unrolled gradient descent with learnable step sizes back-propagates the same
  gradients with and without per-step checkpointing, matches central differences in the step
  sizes, and the peak memory of both forms is recorded.
"""
import numpy as np
import pytest

from conftest import record_parity, rel_l2

pytestmark = pytest.mark.gpu


def _batch_pair(torch, proj, xb, yb):
    s = torch.cuda.current_stream().cuda_stream
    B = xb.shape[0]
    Ax = torch.full((B, proj.range_size), np.nan, device="cuda")
    Aty = torch.full((B, proj.domain_size), np.nan, device="cuda")
    proj.apply_batch_ptr(xb.data_ptr(), proj.domain_size, Ax.data_ptr(), proj.range_size, B, s)
    proj.apply_adjoint_batch_ptr(yb.data_ptr(), proj.range_size, Aty.data_ptr(),
                                 proj.domain_size, B, s)
    torch.cuda.synchronize()
    return Ax, Aty


def _single_pair(torch, proj, x, y):
    s = torch.cuda.current_stream().cuda_stream
    Ax = torch.full((proj.range_size,), np.nan, device="cuda")
    Aty = torch.full((proj.domain_size,), np.nan, device="cuda")
    proj.apply_ptr(x.data_ptr(), Ax.data_ptr(), s)
    proj.apply_adjoint_ptr(y.data_ptr(), Aty.data_ptr(), s)
    torch.cuda.synchronize()
    return Ax, Aty


@pytest.mark.parametrize("kind, vol, det, views", [
    ("JOSEPH", (32, 32, 32), [48, 48], 24),
    ("JOSEPH", (36, 28, 44), [64, 48], 17),
    ("JOSEPH", (64, 64), [92], 60),
    ("SIDDON", (24, 24, 24), [36, 36], 12),
])
def test_batch_equals_single_applies(cuda, oracle, kind, vol, det, views):
    import elsa_b200
    torch = cuda
    n = vol[0]
    poses, dd = oracle.circle_trajectory(vol, views, 360, 10.0 * n, 2.5 * n, det)
    proj = elsa_b200.Projector(getattr(elsa_b200, "PROJECTOR_" + kind), vol, dd, poses)
    if proj.knob(elsa_b200.KNOB_ADJOINT_SCATTER) == 1:
        proj.set_knob(elsa_b200.KNOB_ADJOINT_SCATTER, 0)  # bit-reproducible adjoint to compare
    g = torch.Generator(device="cuda").manual_seed(5)
    for B in (1, 3, 5):  # the batch copies grow between calls
        xb = torch.rand(B, proj.domain_size, device="cuda", generator=g)
        yb = torch.rand(B, proj.range_size, device="cuda", generator=g)
        Ax, Aty = _batch_pair(torch, proj, xb, yb)
        for b in range(B):
            a1, t1 = _single_pair(torch, proj, xb[b], yb[b])
            assert torch.equal(Ax[b], a1), (B, b)
            assert torch.equal(Aty[b], t1), (B, b)
    # an empty batch is a no-op
    proj.apply_batch_ptr(xb.data_ptr(), proj.domain_size, Ax.data_ptr(), proj.range_size, 0,
                         torch.cuda.current_stream().cuda_stream)
    with pytest.raises(elsa_b200.InvalidArgumentError):  # overlapping elements are refused
        proj.apply_batch_ptr(xb.data_ptr(), 1, Ax.data_ptr(), proj.range_size, 2,
                             torch.cuda.current_stream().cuda_stream)


CFG = dict(n=128, batch=8, views=180, det=[192, 192], s2c=1280.0, c2d=320.0)


@pytest.fixture(scope="module")
def cfg_batch(oracle):
    import elsa_b200
    from elsa_b200 import phantoms
    n = CFG["n"]
    vol = (n, n, n)
    poses, det = oracle.circle_trajectory(vol, CFG["views"], 360, CFG["s2c"], CFG["c2d"],
                                          CFG["det"])
    proj = elsa_b200.Projector(elsa_b200.PROJECTOR_JOSEPH, vol, det, poses)
    xt = np.stack([phantoms.random_ellipsoids(n, 20, seed=b).ravel()
                   for b in range(CFG["batch"])])
    return vol, poses, det, proj, xt


@pytest.mark.slow
def test_batch_gradient_fp64_and_central_differences(cuda, oracle, cfg_batch):
    import torch
    from elsa_b200.torch_ops import project
    vol, poses, det, proj, xt = cfg_batch
    B = xt.shape[0]
    rng = np.random.default_rng(11)
    # data from the true volumes, gradient at a perturbed estimate
    y = project(torch.from_numpy(xt).cuda(), proj).detach()
    x0 = (0.9 * xt + 0.05 * rng.uniform(0, 1, xt.shape)).astype(np.float32)
    x = torch.tensor(x0, device="cuda", requires_grad=True)
    loss = 0.5 * ((project(x, proj) - y) ** 2).sum()
    loss.backward()
    g = x.grad.double().cpu().numpy()
    yh = y.double().cpu().numpy()
    errs = []
    for b in range(B):
        xb = x0[b].astype(np.float64)
        r = oracle.joseph(xb, vol, det, poses, dtype=np.float64) - yh[b]
        g64 = oracle.joseph_adjoint(r, vol, det, poses, dtype=np.float64)
        errs.append(rel_l2(g[b], g64))
    # central differences of the FP64 loss, direction k on volume k mod B
    eps, worst = 1e-3, 0.0
    for k in range(16):
        b = k % B
        d = np.random.default_rng(100 + k).standard_normal(xt.shape[1])
        d /= np.linalg.norm(d)

        def L(v):
            r = oracle.joseph(v, vol, det, poses, dtype=np.float64) - yh[b]
            return 0.5 * float(r @ r)

        xb = x0[b].astype(np.float64)
        fd = (L(xb + eps * d) - L(xb - eps * d)) / (2 * eps)
        an = float(g[b] @ d)
        worst = max(worst, abs(fd - an) / (abs(fd) + 1e-12))
        assert abs(fd - an) <= 1e-4 * abs(fd) + 1e-3 * np.linalg.norm(g[b]), (k, fd, an)
    record_parity("cfg_batch8_128_gradient", gpu_vs_f64_worst=max(errs),
                  central_difference_worst_relative=worst, directions=16, eps=eps, bound=1e-5)
    assert max(errs) <= 1e-5, errs


@pytest.mark.slow
def test_batch_unrolled_descent_checkpointed(cuda, oracle, cfg_batch):
    import torch
    from torch.utils.checkpoint import checkpoint
    from elsa_b200.torch_ops import backproject, project
    vol, poses, det, proj, xt_np = cfg_batch
    xt = torch.from_numpy(xt_np).cuda()
    y = project(xt, proj).detach()
    import elsa_b200
    lam = elsa_b200.power_iterations(proj, 20, torch.cuda.current_stream().cuda_stream)

    def step(x, a):
        return x - a * backproject(project(x, proj) - y, proj)

    def run(alphas, ckpt):
        x = torch.zeros_like(xt)
        for k in range(alphas.shape[0]):
            x = checkpoint(step, x, alphas[k], use_reentrant=False) if ckpt else step(x, alphas[k])
        return ((x - xt).double() ** 2).sum()

    base = torch.full((10,), 1.0 / lam, dtype=torch.float32, device="cuda")
    peaks, grads = {}, {}
    for ckpt in (True, False):
        torch.cuda.synchronize()
        torch.cuda.reset_peak_memory_stats()
        start = torch.cuda.memory_allocated()
        alphas = base.clone().requires_grad_(True)
        run(alphas, ckpt).backward()
        torch.cuda.synchronize()
        peaks[ckpt] = torch.cuda.max_memory_allocated() - start
        grads[ckpt] = alphas.grad.double().cpu().numpy()
    g = grads[True]
    assert np.allclose(g, grads[False], rtol=1e-5, atol=0)
    gmax = float(np.abs(g).max())
    for k in (0, 4, 9):  # the loss is quadratic in each a_k: central differences are exact
        h = 0.05 / lam
        ap, am = base.clone(), base.clone()
        ap[k] += h
        am[k] -= h
        with torch.no_grad():
            fd = (run(ap, False) - run(am, False)).item() / (2 * h)
        assert abs(fd - g[k]) <= 5e-2 * max(abs(fd), abs(g[k])) + 1e-3 * gmax, (k, fd, g[k])
    record_parity("cfg_batch8_128_unrolled_10", peak_bytes_checkpointed=int(peaks[True]),
                  peak_bytes_plain=int(peaks[False]))
    print("peak memory: checkpointed %.1f MB, plain %.1f MB" % (peaks[True] / 1e6,
                                                                peaks[False] / 1e6))
    # The projector functions save nothing for backward (their backward is the other operator),
    # so a step keeps only A^T(A x - y) for the gradient of its step size: a volume batch, as
    # large as the step input that checkpointing keeps instead. Both forms hold about ten
    # volume batches; checkpointing must not cost more than one step's transient memory.
    batch_bytes = 4 * xt.numel()
    sino_bytes = 4 * y.numel()
    assert peaks[False] <= 14 * batch_bytes + 4 * sino_bytes
    assert peaks[True] <= peaks[False] + 2 * sino_bytes + 2 * batch_bytes
