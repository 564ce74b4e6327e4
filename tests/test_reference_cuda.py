"""elsa's own CUDA projector kernels (projectors_cuda/projector_kernels/*.cu, built by
oracle/ref_cuda/build.py into oracle/_ref/librefcuda.so) beside this library's kernels on the same
GPU: the harness loads and exports its entry points (CPU), the reference kernels agree with this
library's operators where they compute the same operator (GPU), and both are timed on the
benchmark workloads (GPU; prints one JSON line, run with -s to see it).

The reference's CUDA Joseph forward interpolates through the texture unit (9-bit fixed-point
weights) with its own boundary rule, and its default adjoint (`fast`, JosephsMethodCUDA.h:60-67)
is a voxel-driven backprojection, not the transpose: those are compared loosely. Its Siddon and
voxel kernels compute the same operator as the CPU path up to float rounding and atomic order."""
import json
import os

import numpy as np
import pytest

from conftest import rel_l2


def _ref():
    from oracle import ref_cuda
    if not ref_cuda.built():
        pytest.skip("oracle/_ref/librefcuda.so not built (needs the reference source tree)")
    return ref_cuda


def test_reference_cuda_exports():
    ref_cuda = _ref()
    L = ref_cuda.lib()
    assert all(hasattr(L, s) for s in ref_cuda.SYMBOLS)


def _cuda_voxel_emulation(vol, det, poses, lut, radius, differential, x=None, y=None,
                          row_shift=True):
    """float64 restatement of the reference's CUDA voxel kernel (ProjectVoxelsCUDA.cu:97-176):
    weights over the footprint rectangle [ceil(c - r s), floor(c + r s)] of both detector axes.
    With row_shift, footprint row k is read / written k pixels to the right of the pixel whose
    weight it carries, as the kernel's detector pointer does (jStride = nu + 1 - iStride,
    ProjectVoxelsCUDA.cu:147); without it, this is the CPU path's operator
    (VoxelComputation.h:88, jStride = nu - iStride), which this library and the oracle compute.
    Forward of x, or adjoint of y; the sinogram carries one pose of zero padding for the shift."""
    nx, ny, nz = vol
    nu, nv, npose = det
    poses = np.asarray(poses, np.float64).reshape(npose, -1)
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    v = np.stack([xx.ravel() + 0.5, yy.ravel() + 0.5, zz.ravel() + 0.5, np.ones(xx.size)])
    n = len(lut)
    lut = np.asarray(lut, np.float64)
    out = np.zeros(nu * nv * (npose + 1)) if x is not None else np.zeros(xx.size)
    if y is not None:
        y = np.concatenate([y, np.zeros(nu * nv)])
    sdd = float(np.float32(poses[0, 39]))
    for p in range(npose):
        d = poses[p, 0:12].reshape(3, 4) @ v
        c0, c1 = d[0] / d[2] - 0.5, d[1] / d[2] - 0.5
        scale = np.abs(sdd / np.linalg.norm(poses[p, 27:39].reshape(3, 4) @ v, axis=0))
        r = radius * scale
        lo0, hi0 = np.maximum(0, np.ceil(c0 - r)), np.minimum(nu - 1, np.floor(c0 + r))
        lo1, hi1 = np.maximum(0, np.ceil(c1 - r)), np.minimum(nv - 1, np.floor(c1 + r))
        width = int(np.ceil(2 * r.max())) + 2
        for oj in range(width):
            for oi in range(width):
                i, j = lo0 + oi, lo1 + oj
                m = (i <= hi0) & (j <= hi1)
                prim = c0 - i
                t = np.hypot(prim, c1 - j) / scale
                idx = np.abs(t) / radius * (n - 1)
                ok = m & (idx <= n - 1)
                a = np.floor(np.where(ok, idx, 0)).astype(np.int64)
                b = np.ceil(np.where(ok, idx, 0)).astype(np.int64)
                frac = np.where(ok, idx, 0) - a
                w = np.where(ok, frac * lut[b] + (1 - frac) * lut[a], 0.0)
                if differential:
                    w = prim / scale * w
                pix = (p * nv + j[ok]).astype(np.int64) * nu + i[ok].astype(np.int64)
                if row_shift:
                    pix = pix + (j[ok] - lo1[ok]).astype(np.int64)
                if x is not None:
                    np.add.at(out, pix, w[ok] * x[ok])
                else:
                    out[ok] += w[ok] * y[pix]
    return out[:nu * nv * npose] if x is not None else out


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32).ravel()).cuda()


def _ours(torch, kind, vol, det, poses, x, y):
    import elsa_b200
    proj = elsa_b200.Projector(kind, vol, det, poses)
    Ax = torch.empty(proj.range_size, device="cuda")
    Aty = torch.empty(proj.domain_size, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    proj.apply_ptr(x.data_ptr(), Ax.data_ptr(), s)
    proj.apply_adjoint_ptr(y.data_ptr(), Aty.data_ptr(), s)
    torch.cuda.synchronize()
    return proj, Ax, Aty


@pytest.mark.gpu
def test_reference_cuda_agreement(cuda, oracle):
    ref_cuda = _ref()
    import elsa_b200
    torch = cuda
    vol, views = (32, 32, 32), 24
    poses, det = oracle.circle_trajectory(vol, views, 360, 320, 80, [64, 64])
    rng = np.random.default_rng(5)
    x = _dev(torch, rng.uniform(0, 1, int(np.prod(vol))))
    y = _dev(torch, rng.uniform(0, 1, int(np.prod(det))))
    R = ref_cuda.RefProjectors(vol, det, poses)
    out = {}
    try:
        rAx = torch.empty(int(np.prod(det)), device="cuda")
        rAty = torch.empty(int(np.prod(vol)), device="cuda")
        # Siddon: the same operator
        _, Ax, Aty = _ours(torch, elsa_b200.PROJECTOR_SIDDON, vol, det, poses, x, y)
        R.siddon_forward(x.data_ptr(), rAx.data_ptr())
        R.siddon_adjoint(y.data_ptr(), rAty.data_ptr())
        torch.cuda.synchronize()
        out["siddon_fwd"] = rel_l2(rAx.cpu().numpy(), Ax.cpu().numpy())
        out["siddon_adj"] = rel_l2(rAty.cpu().numpy(), Aty.cpu().numpy())
        # Joseph: texture interpolation and the unmatched fast adjoint
        _, Ax, Aty = _ours(torch, elsa_b200.PROJECTOR_JOSEPH, vol, det, poses, x, y)
        R.joseph_forward(x.data_ptr(), rAx.data_ptr())
        R.joseph_adjoint_fast(y.data_ptr(), rAty.data_ptr())
        torch.cuda.synchronize()
        out["joseph_fwd"] = rel_l2(rAx.cpu().numpy(), Ax.cpu().numpy())
        a, b = rAty.cpu().numpy().astype(np.float64), Aty.cpu().numpy().astype(np.float64)
        out["joseph_fast_adj_corr"] = float(np.corrcoef(a, b)[0, 1])
        # this library's fast mode (JosephsMethodCUDA(..., fast = true)) against the reference's
        # fast kernel: the same float operations and texture reads
        Aty_fast = torch.empty(int(np.prod(vol)), device="cuda")
        fastp = elsa_b200.Projector(elsa_b200.PROJECTOR_JOSEPH, vol, det, poses, [1.0])
        fastp.apply_adjoint_ptr(y.data_ptr(), Aty_fast.data_ptr(),
                                torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        mine, theirs = Aty_fast.cpu().numpy(), rAty.cpu().numpy()
        out["joseph_fast_adj_vs_ours"] = rel_l2(mine, theirs)
        out["joseph_fast_adj_bits_differing"] = int(np.count_nonzero(
            mine.view(np.uint32) != theirs.view(np.uint32)))
        # blob voxel projector, absorption and phase contrast: the reference's CUDA kernels
        # against a restatement of their own formula, and against this library (which follows
        # the CPU path's footprint walk)
        xh, yh = x.cpu().numpy().astype(np.float64), y.cpu().numpy().astype(np.float64)
        for name, code, diff in (("blob", elsa_b200.PROJECTOR_BLOB, False),
                                 ("phase_blob", elsa_b200.PROJECTOR_PHASE_CONTRAST_BLOB, True)):
            lut, support, _ = oracle.voxel_lut(name, 3)
            R.set_lut(lut, support)
            _, Ax, Aty = _ours(torch, code, vol, det, poses, x, y)
            R.voxel_forward(x.data_ptr(), rAx.data_ptr(), diff)
            R.voxel_adjoint(y.data_ptr(), rAty.data_ptr(), diff)
            torch.cuda.synchronize()
            emu_fwd = _cuda_voxel_emulation(vol, det, poses, lut, support, diff, x=xh)
            emu_adj = _cuda_voxel_emulation(vol, det, poses, lut, support, diff, y=yh)
            out[name + "_fwd_vs_formula"] = rel_l2(rAx.cpu().numpy(), emu_fwd)
            out[name + "_adj_vs_formula"] = rel_l2(rAty.cpu().numpy(), emu_adj)
            out[name + "_fwd_vs_ours"] = rel_l2(rAx.cpu().numpy(), Ax.cpu().numpy())
            out[name + "_adj_vs_ours"] = rel_l2(rAty.cpu().numpy(), Aty.cpu().numpy())
    finally:
        R.close()
    print(json.dumps({"reference_cuda_agreement": out}))
    assert all(np.isfinite(v) for v in out.values()), out
    assert out["siddon_fwd"] <= 1e-3 and out["siddon_adj"] <= 1e-3, out
    assert out["joseph_fwd"] <= 5e-2 and out["joseph_fast_adj_corr"] >= 0.7, out
    assert out["joseph_fast_adj_vs_ours"] <= 1e-6, out
    for k in ("blob", "phase_blob"):
        # float32 footprint bounds and weights against the float64 restatement; the phase
        # contrast weights change sign across the footprint, so their sum cancels more
        assert out[k + "_fwd_vs_formula"] <= 5e-3 and out[k + "_adj_vs_formula"] <= 5e-3, out


@pytest.mark.gpu
def test_reference_cuda_fast_adjoint_2d(cuda, oracle):
    """The 2D fast adjoint (1D layered texture) against the reference's 2D kernel, with a volume
    edge that is not a multiple of 32 (the reference's remainder launch)."""
    ref_cuda = _ref()
    import elsa_b200
    torch = cuda
    vol, views = (100, 72), 90
    poses, det = oracle.circle_trajectory(vol, views, 360, 1000, 250, [150])
    rng = np.random.default_rng(6)
    y = _dev(torch, rng.uniform(0, 1, int(np.prod(det))))
    mine = torch.empty(int(np.prod(vol)), device="cuda")
    theirs = torch.empty(int(np.prod(vol)), device="cuda")
    p = elsa_b200.Projector(elsa_b200.PROJECTOR_JOSEPH, vol, det, poses, [1.0])
    p.apply_adjoint_ptr(y.data_ptr(), mine.data_ptr(), torch.cuda.current_stream().cuda_stream)
    R = ref_cuda.RefJoseph2D(vol, det, poses)
    try:
        R.joseph_adjoint_fast(y.data_ptr(), theirs.data_ptr())
        torch.cuda.synchronize()
    finally:
        R.close()
    a, b = mine.cpu().numpy(), theirs.cpu().numpy()
    err = rel_l2(a, b)
    print(json.dumps({"joseph2d_fast_adj_vs_ours": err, "bits_differing":
                      int(np.count_nonzero(a.view(np.uint32) != b.view(np.uint32)))}))
    assert err <= 1e-6


def _median_ms(torch, fn, reps=5, warm=2):
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    times = []
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        times.append(a.elapsed_time(b))
    return float(np.median(times))


@pytest.mark.gpu
def test_reference_cuda_timing(cuda, oracle, tmp_path):
    """Median device time (ms, CUDA events on the legacy default stream, where the reference
    kernels launch) of each operator, inputs resident on the device. The reference's operators
    upload their input into a texture and copy the pitched output back on every call; both its
    kernel alone ("kernel") and the whole call ("call") are timed."""
    ref_cuda = _ref()
    import elsa_b200
    torch = cuda
    s = torch.cuda.current_stream().cuda_stream
    result = {}
    for name, vol, views, det_size, s2c, c2d in (("cone256", (256, 256, 256), 360, 384, 2560, 640),
                                                 ("blob128", (128, 128, 128), 180, 192, 1280, 320)):
        poses, det = oracle.circle_trajectory(vol, views, 360, s2c, c2d, [det_size, det_size])
        rng = np.random.default_rng(1)
        x = _dev(torch, rng.uniform(0, 1, int(np.prod(vol))))
        y = _dev(torch, rng.uniform(0, 1, int(np.prod(det))))
        Ax = torch.empty(int(np.prod(det)), device="cuda")
        Aty = torch.empty(int(np.prod(vol)), device="cuda")
        R = ref_cuda.RefProjectors(vol, det, poses)
        rec = {}
        try:
            if name == "cone256":
                kinds = (("joseph", elsa_b200.PROJECTOR_JOSEPH), ("siddon", elsa_b200.PROJECTOR_SIDDON))
            else:
                kinds = (("blob", elsa_b200.PROJECTOR_BLOB),
                         ("phase_blob", elsa_b200.PROJECTOR_PHASE_CONTRAST_BLOB))
            for kname, code in kinds:
                proj = elsa_b200.Projector(code, vol, det, poses)
                rec[kname + "_ours_fwd"] = _median_ms(
                    torch, lambda: proj.apply_ptr(x.data_ptr(), Ax.data_ptr(), s))
                rec[kname + "_ours_adj"] = _median_ms(
                    torch, lambda: proj.apply_adjoint_ptr(y.data_ptr(), Aty.data_ptr(), s))
                del proj
                torch.cuda.synchronize()
            if name == "cone256":
                # the whole call first: it leaves the input in the texture the kernel reads
                rec["joseph_ref_fwd_call"] = _median_ms(
                    torch, lambda: R.joseph_forward(x.data_ptr(), Ax.data_ptr()))
                rec["joseph_ref_fwd_kernel"] = _median_ms(
                    torch, lambda: R.joseph_forward(x.data_ptr(), Ax.data_ptr(), True))
                rec["joseph_ref_fast_adj_call"] = _median_ms(
                    torch, lambda: R.joseph_adjoint_fast(y.data_ptr(), Aty.data_ptr()))
                rec["joseph_ref_fast_adj_kernel"] = _median_ms(
                    torch, lambda: R.joseph_adjoint_fast(y.data_ptr(), Aty.data_ptr(), True))
                fastp = elsa_b200.Projector(elsa_b200.PROJECTOR_JOSEPH, vol, det, poses, [1.0])
                rec["joseph_ours_fast_adj"] = _median_ms(
                    torch, lambda: fastp.apply_adjoint_ptr(y.data_ptr(), Aty.data_ptr(), s))
                del fastp
                rec["siddon_ref_fwd"] = _median_ms(
                    torch, lambda: R.siddon_forward(x.data_ptr(), Ax.data_ptr()), reps=3)
                rec["siddon_ref_adj"] = _median_ms(
                    torch, lambda: R.siddon_adjoint(y.data_ptr(), Aty.data_ptr()), reps=3)
            else:
                for kname, diff in (("blob", False), ("phase_blob", True)):
                    lut, support, _ = oracle.voxel_lut(kname, 3)
                    R.set_lut(lut, support)
                    rec[kname + "_ref_fwd"] = _median_ms(
                        torch, lambda: R.voxel_forward(x.data_ptr(), Ax.data_ptr(), diff), reps=3)
                    rec[kname + "_ref_adj"] = _median_ms(
                        torch, lambda: R.voxel_adjoint(y.data_ptr(), Aty.data_ptr(), diff), reps=3)
        finally:
            R.close()
        result[name] = {k: round(v, 3) for k, v in rec.items()}
        del x, y, Ax, Aty
        torch.cuda.empty_cache()
    result["device"] = torch.cuda.get_device_name(0)
    line = json.dumps({"reference_cuda_timing_ms": result})
    print(line)
    out_dir = os.environ.get("ELSA_TIMING_OUT")
    if out_dir:
        with open(os.path.join(out_dir, "reference_cuda_timing.json"), "w") as f:
            f.write(line + "\n")
    for rec in result.values():
        if isinstance(rec, dict):
            assert all(np.isfinite(v) and v > 0 for v in rec.values()), rec
