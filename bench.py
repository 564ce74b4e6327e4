#!/usr/bin/env python3
"""Benchmark of the elsa_b200 hot path: 3D cone-beam Joseph forward + matched adjoint inside CGNE
iterations at 256^3 (360 views, 384 x 384 detector, source-centre 2560, centre-detector 640).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl elsa_b200|reference]

One step is one CGNE iteration (solvers/CGNE.cpp:50-73 of elsa): a forward projection, the matched
adjoint and the fused float64 vector updates, enqueued through the C ABI (elsa_solver_iterate).
`value` counts the voxel-view updates of the forward + adjoint pass per second (GUPS = 2 * N_vox *
N_views per step). `e2e` is the same metric through the host-buffer entry points (the reference's
call pattern: volume in, sinogram out, sinogram in, volume out, every apply). Under torchrun the
one 256^3 problem is split by views over the ranks (strong scaling): every CGNE iteration applies
each rank's block of views and all-reduces one volume over NCCL; `value` is the whole problem's
rate, timed as the max over ranks.

`--impl reference` times the CPU restatement of elsa's own algorithm (oracle/, the reference
C++ library cannot be built here: Eigen 3.4 is absent) on the host cores, on a bounded subset of
views per step, and reports the same metric.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "3D cone-beam fwd+back GUPS and CG iters/s at 256^3; batched vs plain, 1 GPU"
WORKLOAD = dict(workload="cone-beam Joseph CGNE, 256^3 volume, 360 views, 384x384 detector",
                volume=[256, 256, 256], views=360, detector=[384, 384], source_to_center=2560,
                center_to_detector=640, phantom="modified Shepp-Logan 3D")
# kernels launched per CGNE iteration besides the projections: dot (partials + finish), step,
# finish-norm, direction (solvers.cu, cgneStep)
VECTOR_LAUNCHES_PER_STEP = 5


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.device_index = device_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device_index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names[1:], parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)),
                "reasons": sorted(reasons), "samples": len(sm)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_baseline_sample(views_in_sample, vol, poses, det, x):
    """Time the oracle (CPU restatement of elsa's Joseph path, all host threads) on a subset of
    the views: forward + adjoint. Returns (GUPS, seconds, threads)."""
    from oracle import oracle as O
    O.build()
    O.set_adjoint_atomic(True)  # time the reference's own scheme (omp atomic adds)
    idx = np.linspace(0, poses.shape[0] - 1, views_in_sample).round().astype(int)
    p = np.ascontiguousarray(poses[idx])
    d = np.array([det[0], det[1], len(idx)])
    t0 = time.perf_counter()
    y = O.joseph(x, vol, d, p)
    O.joseph_adjoint(y, vol, d, p)
    dt = time.perf_counter() - t0
    O.set_adjoint_atomic(False)
    return 2.0 * np.prod(vol) * len(idx) / dt / 1e9, dt, O.num_threads()


PARITY_VIEWS = (0, 45, 90, 135, 180, 225, 270, 315)


def parity_block(torch, proj, vol, poses, det, x_true):
    """Relative L2 of the benchmarked operator (the same projector handle, its kernels, view
    chunks and knobs) against the FP32 and FP64 oracle on a fixed subset of the views, outside the
    timed region. Forward: the rows of the subset's views of A x_true. Adjoint: A^T y with y
    seeded U(0,1) on the subset's views and zero on all others, which equals the oracle's adjoint
    over the subset's views alone."""
    from oracle import oracle as O
    O.build()
    idx = np.array(PARITY_VIEWS)
    view = int(det[0]) * int(det[1])
    sub = np.ascontiguousarray(poses[idx])
    dsub = np.array([det[0], det[1], len(idx)])
    s = torch.cuda.current_stream().cuda_stream
    xt = torch.from_numpy(np.ascontiguousarray(x_true).ravel()).cuda()
    Ax = torch.empty(proj.range_size, dtype=torch.float32, device="cuda")
    proj.apply_ptr(xt.data_ptr(), Ax.data_ptr(), s)
    ysub = np.random.default_rng(2).uniform(0, 1, len(idx) * view).astype(np.float32)
    yfull = np.zeros(proj.range_size, np.float32)
    for i, v in enumerate(idx):
        yfull[v * view:(v + 1) * view] = ysub[i * view:(i + 1) * view]
    yd = torch.from_numpy(yfull).cuda()
    Aty = torch.empty(proj.domain_size, dtype=torch.float32, device="cuda")
    proj.apply_adjoint_ptr(yd.data_ptr(), Aty.data_ptr(), s)
    torch.cuda.synchronize()
    fwd = Ax.cpu().numpy().reshape(-1, view)[idx].ravel()
    adj = Aty.cpu().numpy()
    del xt, Ax, yd, Aty

    def rel(a, b):
        a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    f32 = O.joseph(x_true, vol, dsub, sub)
    a32 = O.joseph_adjoint(ysub, vol, dsub, sub)
    f64 = O.joseph(x_true.astype(np.float64), vol, dsub, sub, dtype=np.float64)
    a64 = O.joseph_adjoint(ysub.astype(np.float64), vol, dsub, sub, dtype=np.float64)
    return {"views": [int(v) for v in idx], "bound": 1e-5,
            "forward_vs_f32": rel(fwd, f32), "forward_vs_f64": rel(fwd, f64),
            "adjoint_vs_f32": rel(adj, a32), "adjoint_vs_f64": rel(adj, a64),
            "oracle_f32_vs_f64": {"forward": rel(f32, f64), "adjoint": rel(a32, a64)},
            "how": "the benchmarked projector handle; oracle on the listed views; "
                   "x = modified Shepp-Logan, y = U(0,1) seed 2 on those views"}


def _traffic_from_profiles():
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "joseph_cone256_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return None


def _apply_size(args):
    """--size N scales the cone-beam problem (N^3 volume, 1.5 N detector, same ratios) for
    profiling small cases; the default is the 256^3 workload."""
    if args.size and args.size != 256:
        n = args.size
        WORKLOAD.update(volume=[n, n, n], detector=[3 * n // 2, 3 * n // 2],
                        source_to_center=10 * n, center_to_detector=5 * n // 2,
                        workload="cone-beam Joseph CGNE, %d^3 volume, 360 views, %dx%d detector"
                                 % (n, 3 * n // 2, 3 * n // 2))


def run_sharded(args):
    """N > 1: one 256^3 problem, its views split into N contiguous blocks, one per rank; every
    CGNE iteration applies each rank's block (native kernels) and all-reduces the volume
    A^T A c over NCCL on the solver stream (strong scaling: the total work is fixed)."""
    import ctypes
    import datetime

    import torch
    import torch.distributed as dist
    import elsa_b200
    from elsa_b200 import _capi, phantoms
    from elsa_b200.sharded import ShardedCGNE, native_split, view_block

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    if "MASTER_ADDR" not in os.environ:  # --sharded without torchrun: a group of one rank
        import socket
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(sk.getsockname()[1]),
                              RANK="0", WORLD_SIZE="1")
    os.environ.setdefault("NCCL_DEBUG", "INFO")  # NCCL's init log (transport, NVLS) on stderr
    os.environ.setdefault("NCCL_DEBUG_SUBSYS", "INIT")
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device("cuda", local))
    _apply_size(args)
    vol = tuple(WORKLOAD["volume"])
    poses, det = elsa_b200.circle_trajectory(vol, WORKLOAD["views"], 360,
                                             WORKLOAD["source_to_center"],
                                             WORKLOAD["center_to_detector"], WORKLOAD["detector"])
    split, proj, (lo, hi) = native_split(elsa_b200.PROJECTOR_JOSEPH, vol, poses, det, rank,
                                         world)
    x_true = phantoms.modified_shepp_logan(vol)
    stream = torch.cuda.current_stream().cuda_stream
    xt = torch.from_numpy(x_true.ravel()).cuda()
    b = torch.empty(proj.range_size, dtype=torch.float32, device="cuda")
    proj.apply_ptr(xt.data_ptr(), b.data_ptr(), stream)
    solver = ShardedCGNE(split, b)
    solver.begin()
    solver.iterate(args.warmup)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    dist.barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    hist = solver.iterate(args.steps)
    end.record()
    torch.cuda.synchronize()
    dist.barrier()
    ms = start.elapsed_time(end)
    clock_info = clocks.stop()
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    updates = 2.0 * np.prod(vol) * WORKLOAD["views"]  # the whole problem's fwd + adj per step
    value = updates * args.steps / (ms / 1e3) / 1e9

    # end to end: every rank's host-buffer forward + adjoint of its block (pinned buffers)
    xh = torch.from_numpy(x_true.ravel()).pin_memory().numpy()
    yh = torch.empty(proj.range_size, dtype=torch.float32).pin_memory().numpy()
    bh = torch.empty(proj.domain_size, dtype=torch.float32).pin_memory().numpy()

    def e2e_step():
        _capi.call("elsa_projector_apply_host", proj.handle, _capi.np_ptr(xh), _capi.np_ptr(yh))
        _capi.call("elsa_projector_apply_adjoint_host", proj.handle, _capi.np_ptr(yh),
                   _capi.np_ptr(bh))

    e2e_steps = max(2, min(args.steps, 5))
    e2e_step()
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    e2e_s = time.perf_counter() - t0
    t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_value = updates * e2e_steps / float(t.item()) / 1e9
    res = [float(v) for v in hist.cpu()]
    out = {
        "metric": METRIC, "value": round(value, 3), "unit": "GUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (modified Shepp-Logan 3D phantom, b = A x)",
        "config": dict(WORKLOAD, parallelism="views sharded over %d ranks, NCCL all-reduce of "
                                             "A^T A c per CGNE iteration" % world,
                       views_per_rank=[hi_ - lo_ for lo_, hi_ in
                                       (view_block(WORKLOAD["views"], r, world)
                                        for r in range(world))],
                       l2="working set > L2"),
        "cg_iters_per_s": round(1e3 * args.steps / ms, 3),
        "cg_residual_sq": [res[0], res[-1]] if res else [],
        "e2e": {"value": round(e2e_value, 3), "unit": "GUPS",
                "h2d_bytes_per_step": 4 * (proj.domain_size + proj.range_size),
                "d2h_bytes_per_step": 4 * (proj.range_size + proj.domain_size),
                "timing": "host wall clock, max over ranks, every rank its block"},
        "gpu_launches": (proj.info(6) + proj.info(7) + VECTOR_LAUNCHES_PER_STEP) * args.steps,
        "clocks": clock_info,
    }
    split.close()
    dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


def run_elsa(args):
    import torch
    import elsa_b200
    from elsa_b200 import phantoms

    world, rank, local = _dist()
    if world > 1 or args.sharded:
        run_sharded(args)
        return
    torch.cuda.set_device(local)
    dist = None

    _apply_size(args)
    vol = tuple(WORKLOAD["volume"])
    poses, det = elsa_b200.circle_trajectory(vol, WORKLOAD["views"], 360,
                                             WORKLOAD["source_to_center"],
                                             WORKLOAD["center_to_detector"], WORKLOAD["detector"])
    proj = elsa_b200.Projector(elsa_b200.PROJECTOR_JOSEPH, vol, det, poses)
    x_true = phantoms.modified_shepp_logan(vol)
    stream = torch.cuda.current_stream().cuda_stream
    xt = torch.from_numpy(x_true.ravel()).cuda()
    b = torch.empty(proj.range_size, dtype=torch.float32, device="cuda")
    proj.apply_ptr(xt.data_ptr(), b.data_ptr(), stream)
    x = torch.zeros(proj.domain_size, dtype=torch.float32, device="cuda")
    solver = elsa_b200.Solver(elsa_b200.SOLVER_CGNE, proj, b.data_ptr(), x.data_ptr(),
                              stream=stream)
    solver.iterate(args.warmup, stream)
    torch.cuda.synchronize()
    res0 = solver.squared_residual(stream)

    clocks = ClockSampler(local)
    clocks.start()
    solver.enable_timing(True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    solver.iterate(args.steps, stream)
    end.record()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = start.elapsed_time(end)
    clock_info = clocks.stop()
    fwd_ms, adj_ms, timed = solver.timing()
    res1 = solver.squared_residual(stream)
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    updates = 2.0 * np.prod(vol) * WORKLOAD["views"]  # forward + adjoint voxel-view updates
    ms_per_step = ms / args.steps
    value = updates * args.steps * world / (ms / 1e3) / 1e9

    # end to end through the host-buffer entry points (pinned host memory)
    xh = torch.from_numpy(x_true.ravel()).pin_memory().numpy()
    yh = torch.empty(proj.range_size, dtype=torch.float32).pin_memory().numpy()
    bh = torch.empty(proj.domain_size, dtype=torch.float32).pin_memory().numpy()
    import ctypes
    from elsa_b200 import _capi

    def e2e_step():
        _capi.call("elsa_projector_apply_host", proj.handle, _capi.np_ptr(xh), _capi.np_ptr(yh))
        _capi.call("elsa_projector_apply_adjoint_host", proj.handle, _capi.np_ptr(yh),
                   _capi.np_ptr(bh))

    e2e_steps = max(2, min(args.steps, 5))
    e2e_step()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = updates * e2e_steps * world / e2e_s / 1e9
    h2d = 4 * (proj.domain_size + proj.range_size)
    d2h = 4 * (proj.range_size + proj.domain_size)

    # roofline of the dominant kernel: algorithmic gather bytes 4 (N_vol + N_sino) + 16 S per pass
    samples = proj.info(2)
    bytes_per_pass = 4.0 * (proj.domain_size + proj.range_size) + 16.0 * samples
    fwd_avg, adj_avg = fwd_ms / max(timed, 1), adj_ms / max(timed, 1)
    dominant = "josephAdjointKernel" if adj_avg >= fwd_avg else "josephForwardKernel"
    dom_ms = max(fwd_avg, adj_avg)
    peak, peak_kind = _peaks()
    achieved = bytes_per_pass / (dom_ms / 1e3) / 1e9
    traffic = None
    prof = _traffic_from_profiles()
    if prof and (prof.get("kernel") != dominant or prof.get("workload") != WORKLOAD["workload"]):
        prof = None  # the committed capture is of another kernel or workload
    if prof:
        traffic = prof.get("dram_bytes_per_launch")
    compulsory = 4.0 * (proj.domain_size + proj.range_size)
    pair_achieved = 2.0 * bytes_per_pass / ((fwd_avg + adj_avg) / 1e3) / 1e9
    # issue-rate ceiling of the dominant kernel: its warp instructions per sample (ncu, on a
    # smaller case of the same geometry family) x samples / (148 SMs x 4 schedulers x clock)
    issue = None
    wips = prof.get("warp_inst_per_sample") if prof else None
    if wips:
        mhz = (clock_info or {}).get("sm_mhz") or 1965.0
        ceiling_ms = wips * samples / (148 * 4 * mhz * 1e6) * 1e3
        issue = {"warp_inst_per_sample": wips, "sm_mhz": mhz,
                 "ceiling_ms": round(ceiling_ms, 3),
                 "frac": round(ceiling_ms / dom_ms, 4),
                 "source": prof.get("warp_inst_source")}

    out = {
        "metric": METRIC, "value": round(value, 3), "unit": "GUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (modified Shepp-Logan 3D phantom, b = A x)",
        "config": dict(WORKLOAD, parallelism="replicas" if world > 1 else "single GPU",
                       l2="no flush; every pass streams the %d-ray table with its slab "
                          "checkpoints and the %.0f MB sinogram, together > L2 (126 MB)"
                          % (proj.range_size, 4e-6 * proj.range_size)),
        "cg_iters_per_s": round(1e3 / ms_per_step, 3),
        "forward_ms": round(fwd_avg, 4), "adjoint_ms": round(adj_avg, 4),
        "cg_residual_sq": [res0, res1],
        "e2e": {"value": round(e2e_value, 3), "unit": "GUPS", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "timing": "host wall clock, pinned buffers"},
        "roofline": {"bound": "hbm", "kernel": dominant, "achieved": round(achieved, 1),
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic,
                     "algorithmic_bytes_per_launch": bytes_per_pass,
                     "samples_per_launch": samples,
                     "compulsory_frac": round(compulsory / (dom_ms / 1e3) / 1e9 / peak, 5),
                     # forward + matched adjoint together: two passes of gather bytes over
                     # the sum of the two kernels' mean durations
                     "forward_back_achieved": round(pair_achieved, 1),
                     "forward_back_frac": round(pair_achieved / peak, 4),
                     # the kernels are bound by instruction issue, not by DRAM (traffic is a
                     # small fraction of the gather bytes): the issue-rate ceiling beside it
                     "issue": issue},
        "gpu_launches": (proj.info(6) + proj.info(7) + VECTOR_LAUNCHES_PER_STEP) * args.steps,
        "clocks": clock_info,
    }
    if rank == 0 and not args.no_parity:
        out["parity"] = parity_block(torch, proj, vol, poses, det, x_true)
    if rank == 0 and world == 1 and not args.no_batched:
        # the batched workload: 64 seeded instances, edges {64, 96, 128, 192, 256}, 60-360
        # views, detector 1.5 x edge, 50 CGNE iterations each (--batched-small: a reduced set)
        if args.batched_small:
            out["batched"] = batched_vs_plain(torch, elsa_b200, phantoms)
        else:
            out["batched"] = batched_vs_plain(torch, elsa_b200, phantoms, instances=64,
                                              iterations=50, edges=(64, 96, 128, 192, 256),
                                              views=(60, 360))
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        gups, dt, cores = cpu_baseline_sample(args.cpu_views, vol, poses, det, x_true)
        out["cpu_baseline"] = {"value": round(gups, 5), "unit": "GUPS", "cores": cores,
                               "kind": "port", "seconds": round(dt, 2),
                               "sample": "Joseph forward + adjoint over %d of the 360 views "
                                         "(256^3, 384^2 detector)" % args.cpu_views}
    if dist:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


def reference_form_cgne(torch, proj, b, iterations):
    """CGNE in the reference's per-instance form: solvers/CGNE.cpp:20-78 over the operator's
    apply / applyAdjoint, every operator application and vector operation its own call, and every
    scalar (c.Ac and |r|^2 of the recurrence, and |r|, |c| of the log line the reference formats
    each iteration) read back to the host before the next step, as DataContainer::dot and
    squaredL2Norm return host values. Device-resident data (no host copies per apply)."""
    import ctypes
    from elsa_b200 import _capi
    s = torch.cuda.current_stream().cuda_stream
    n = proj.domain_size
    x = torch.zeros(n, device="cuda")
    r = torch.empty(n, device="cuda")
    c = torch.empty(n, device="cuda")
    ac = torch.empty(n, device="cuda")
    atb = torch.empty(n, device="cuda")
    tmp = torch.empty(proj.range_size, device="cuda")
    res = torch.empty(1, dtype=torch.float64, device="cuda")

    def dot(u, v):
        _capi.call("elsa_dot", u.data_ptr(), v.data_ptr(), n, res.data_ptr(), s)
        return res.item()

    def sq(u):
        _capi.call("elsa_squared_l2_norm", u.data_ptr(), n, res.data_ptr(), s)
        return res.item()

    def lin(a, u, bb, v, out):
        _capi.call("elsa_lincomb", ctypes.c_float(a), u.data_ptr(), ctypes.c_float(bb),
                   v.data_ptr(), out.data_ptr(), n, s)

    def normal(u, out):  # (A^T A) u
        proj.apply_ptr(u.data_ptr(), tmp.data_ptr(), s)
        proj.apply_adjoint_ptr(tmp.data_ptr(), out.data_ptr(), s)

    proj.apply_adjoint_ptr(b.data_ptr(), atb.data_ptr(), s)  # A^T b
    normal(x, r)                                             # r = A^T b - A^T A x
    lin(-1.0, r, 1.0, atb, r)
    lin(1.0, r, 0.0, r, c)                                   # c = r
    kold = sq(r)
    for _ in range(iterations):
        normal(c, ac)
        alpha = kold / dot(c, ac)
        lin(1.0, x, alpha, c, x)
        lin(1.0, r, -alpha, ac, r)
        k = sq(r)
        beta = k / kold
        lin(1.0, r, beta, c, c)
        kold = k
        sq(r), sq(c)  # the norms of the per-iteration log line
    return x


def batched_vs_plain(torch, elsa_b200, phantoms, instances=12, iterations=10, streams=8,
                     seed=5, edges=(64, 96, 128), views=(60, 180), free_floor_gb=24.0):
    """Many independent reconstructions: one at a time (each solver's iterations enqueued on one
    stream, one problem after the other) against the batched solver elsa_batch_cgne (one CUDA
    graph for the whole batch; `batched_recon_per_s`), and against elsa_solve_batch (every
    solver's iterations as its own CUDA graph, problems spread over concurrent streams). Seeded instances with volume edges
    drawn from `edges`, views uniform in `views`, a detector of 1.5 x edge and a modified
    Shepp-Logan phantom. Instances are built in waves that leave `free_floor_gb` of device
    memory free; each wave is timed both ways and the times are summed. Projector and solver
    set-up is outside both timed regions."""
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(instances):
        n = int(rng.choice(list(edges)))
        nv = int(rng.integers(views[0], views[1] + 1))
        specs.append((n, nv))
    t_plain = t_batch = t_graphs = t_ref = 0.0
    waves = 0
    per_edge = {}  # plain form: seconds spent on the instances of each volume edge
    i = 0
    while i < len(specs):
        problems = []
        while i < len(specs):
            n, nv = specs[i]
            vol = (n, n, n)
            poses, det = elsa_b200.circle_trajectory(vol, nv, 360, 10.0 * n, 2.5 * n,
                                                     [int(1.5 * n), int(1.5 * n)])
            proj = elsa_b200.Projector(elsa_b200.PROJECTOR_JOSEPH, vol, det, poses)
            xt = torch.from_numpy(phantoms.modified_shepp_logan(vol).ravel()).cuda()
            b = torch.empty(proj.range_size, dtype=torch.float32, device="cuda")
            proj.apply_ptr(xt.data_ptr(), b.data_ptr(), torch.cuda.current_stream().cuda_stream)
            problems.append((proj, b))
            i += 1
            torch.cuda.synchronize()
            free, _ = torch.cuda.mem_get_info()
            # two solver workspaces per problem are still to come (4 volumes + 2 sinograms each)
            ws = 2 * 4 * (4 * proj.domain_size + 2 * proj.range_size)
            if free - ws < free_floor_gb * 1e9:
                break
        waves += 1

        def make():
            s = torch.cuda.current_stream().cuda_stream
            xs, sols = [], []
            for proj, b in problems:
                x = torch.zeros(proj.domain_size, dtype=torch.float32, device="cuda")
                sols.append(elsa_b200.Solver(elsa_b200.SOLVER_CGNE, proj, b.data_ptr(),
                                             x.data_ptr(), stream=s))
                xs.append(x)
            torch.cuda.synchronize()
            return xs, sols

        # the reference's per-instance form, one problem after the other
        reference_form_cgne(torch, problems[0][0], problems[0][1], 1)  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for proj, b in problems:
            reference_form_cgne(torch, proj, b, iterations)
        torch.cuda.synchronize()
        t_ref += time.perf_counter() - t0
        torch.cuda.empty_cache()
        xs, plain = make()
        s = torch.cuda.current_stream().cuda_stream
        for sol in plain:  # warm-up of every kernel shape
            sol.iterate(1, s)
        torch.cuda.synchronize()
        marks = [torch.cuda.Event(enable_timing=True) for _ in range(len(plain) + 1)]
        t0 = time.perf_counter()
        marks[0].record()
        for k, sol in enumerate(plain):
            sol.iterate(iterations, s)
            marks[k + 1].record()
        torch.cuda.synchronize()
        t_plain += time.perf_counter() - t0
        for k, (proj, _) in enumerate(problems):
            edge = int(proj.vol_dims[0])
            per_edge[edge] = per_edge.get(edge, 0.0) + marks[k].elapsed_time(marks[k + 1]) / 1e3
        for sol in plain:
            sol.close()
        del xs, plain
        xs2, batch = make()
        elsa_b200.solve_batch(batch, 1, streams)  # captures the one-iteration graphs (warm-up)
        t0 = time.perf_counter()
        elsa_b200.solve_batch(batch, iterations, streams)  # captures + runs the timed graphs
        t_graphs += time.perf_counter() - t0
        for sol in batch:
            sol.close()
        del xs2, batch
        # the batched solver: forwards side by side, all adjoints in one launch per axis grid,
        # batched vector updates, the whole iteration one CUDA graph
        st = torch.cuda.Stream()
        xs3 = [torch.zeros(p.domain_size, dtype=torch.float32, device="cuda")
               for p, _ in problems]
        with torch.cuda.stream(st):
            bc = elsa_b200.BatchCGNE([p for p, _ in problems], [b.data_ptr() for _, b in problems],
                                     [x.data_ptr() for x in xs3], st.cuda_stream)
            bc.iterate_graph(1, st.cuda_stream)  # warm-up of every kernel shape
        st.synchronize()
        t0 = time.perf_counter()
        with torch.cuda.stream(st):
            bc.iterate_graph(iterations, st.cuda_stream)  # captures + runs the timed graph
        st.synchronize()
        t_batch += time.perf_counter() - t0
        bc.close()
        for proj, _ in problems:
            proj.close()
        del xs3, problems
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    return {"instances": instances, "iterations": iterations, "streams": streams,
            "waves": waves,
            "workload": "seeded CGNE problems, edges {%s}, %d-%d views, detector 1.5 x edge, "
                        "Joseph" % (", ".join(str(e) for e in edges), views[0], views[1]),
            "plain_recon_per_s": round(instances / t_plain, 3),
            "batched_recon_per_s": round(instances / t_batch, 3),
            "speedup": round(t_plain / t_batch, 3),
            "plain_form": "this library's CGNE sessions one at a time: device-resident scalars, "
                          "every iteration enqueued without a host round trip",
            "reference_form_recon_per_s": round(instances / t_ref, 3),
            "speedup_vs_reference_form": round(t_ref / t_batch, 3),
            "reference_form": "CGNE.cpp's loop one problem at a time on this library's kernels: "
                              "one call per operator application and vector operation, four "
                              "scalars read back to the host per iteration",
            # the instances of edge <= 128 are the only ones that leave the GPU idle on their
            # own; if batching made them free the gain would still be bounded by their share
            "small_instance_share": round(sum(v for k, v in per_edge.items() if k <= 128)
                                          / max(sum(per_edge.values()), 1e-9), 4),
            "batched_form": "elsa_batch_cgne: forwards side by side, all adjoints in one launch "
                            "per axis grid over an instance table, batched vector updates, the "
                            "iterations one CUDA graph",
            "concurrent_graphs_recon_per_s": round(instances / t_graphs, 3),
            "plain_seconds_by_edge": {str(k): round(v, 3) for k, v in sorted(per_edge.items())},
            "instances_by_edge": {str(e): sum(1 for n, _ in specs if n == e)
                                  for e in sorted(set(n for n, _ in specs))},
            "timing": "host wall clock around synchronized device work, graph capture included"}


SECONDARY = {
    # name: (projector kind, volume, views, detector, params, source-centre, centre-detector)
    "siddon256": ("SIDDON", (256, 256, 256), 360, [384, 384], None, 2560, 640),
    "siddon128": ("SIDDON", (128, 128, 128), 360, [192, 192], None, 1280, 320),
    "blob128": ("BLOB", (128, 128, 128), 180, [192, 192], [2.0, 10.83, 2.0], 1280, 320),
    "bspline128": ("BSPLINE", (128, 128, 128), 180, [192, 192], [2.0], 1280, 320),
    "phase_blob128": ("PHASE_CONTRAST_BLOB", (128, 128, 128), 180, [192, 192],
                      [2.0, 10.83, 2.0], 1280, 320),
    "phase_bspline128": ("PHASE_CONTRAST_BSPLINE", (128, 128, 128), 180, [192, 192], [2.0],
                         1280, 320),
    "joseph2d128": ("JOSEPH", (128, 128), 180, [182], None, 1000, 250),
    "binary2d128": ("BINARY", (128, 128), 180, [182], None, 1000, 250),
    "rayblob64": ("RAY_BLOB", (64, 64, 64), 60, [96, 96], [2.0, 10.83, 2.0], 640, 160),
    # JosephsMethodCUDA(..., fast = true): the TMA forward and elsa's voxel-driven adjoint
    "joseph256fast": ("JOSEPH", (256, 256, 256), 360, [384, 384], [1.0], 2560, 640),
    "joseph2d512": ("JOSEPH", (512, 512), 720, [730], None, 5120, 1280),
}


def run_secondary(args):
    """Forward / adjoint times of the other projector workloads (CUDA events, mean of 5 calls
    after 3 warm-up calls, random inputs); one JSON line."""
    import torch
    import elsa_b200
    torch.cuda.set_device(0)
    names = list(SECONDARY) if args.secondary == "all" else args.secondary.split(",")
    s = torch.cuda.current_stream().cuda_stream
    out = {"secondary": {}}
    for name in names:
        kind, vol, views, det, params, s2c, c2d = SECONDARY[name]
        poses, dd = elsa_b200.circle_trajectory(vol, views, 360, s2c, c2d, det)
        p = elsa_b200.Projector(getattr(elsa_b200, "PROJECTOR_" + kind), vol, dd, poses, params)
        knobs = {}
        for kv in args.knob or []:  # e.g. exact_weights=1, adjoint_scatter=1
            k, v = kv.split("=")
            knob = elsa_b200._capi.KNOB_NAMES.index(k)
            if p.knob_candidates(knob):
                p.set_knob(knob, int(v))
                knobs[k] = int(v)
        x = torch.rand(p.domain_size, device="cuda")
        y = torch.rand(p.range_size, device="cuda")
        oy, ox = torch.empty_like(y), torch.empty_like(x)

        def timed(fn):
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(5):
                fn()
            b.record()
            torch.cuda.synchronize()
            return a.elapsed_time(b) / 5

        fwd = timed(lambda: p.apply_ptr(x.data_ptr(), oy.data_ptr(), s))
        adj = timed(lambda: p.apply_adjoint_ptr(y.data_ptr(), ox.data_ptr(), s))
        nvox = int(np.prod(vol))
        out["secondary"][name] = {
            "volume": [int(v) for v in vol], "views": int(views),
            "detector": [int(v) for v in dd[:-1]],
            "forward_ms": round(fwd, 3), "adjoint_ms": round(adj, 3), "knobs": knobs,
            "gups": round(2 * nvox * views / ((fwd + adj) / 1e3) / 1e9, 3)}
        p.close()
    print(json.dumps(out))


def run_reference(args):
    world, rank, local = _dist()
    if rank != 0:
        return
    from oracle import oracle as O
    from elsa_b200 import phantoms
    O.build()
    _apply_size(args)
    vol = tuple(WORKLOAD["volume"])
    poses, det = O.circle_trajectory(vol, WORKLOAD["views"], 360, WORKLOAD["source_to_center"],
                                     WORKLOAD["center_to_detector"], WORKLOAD["detector"])
    x = phantoms.modified_shepp_logan(vol)
    times = []
    for i in range(args.warmup + args.steps):
        gups, dt, cores = cpu_baseline_sample(args.cpu_views, vol, poses, det, x)
        if i >= args.warmup:
            times.append(dt)
    dt = float(np.mean(times))
    value = 2.0 * np.prod(vol) * args.cpu_views / dt / 1e9
    out = {
        "impl": "reference", "metric": METRIC, "value": round(value, 5), "unit": "GUPS",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(dt * 1e3, 2), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (modified Shepp-Logan 3D phantom)",
        "config": dict(WORKLOAD, parallelism="host cores"),
        "cpu_baseline": {"value": round(value, 5), "unit": "GUPS", "cores": O.num_threads(),
                         "kind": "port",
                         "sample": "per step: Joseph forward + adjoint over %d of the 360 views"
                                   % args.cpu_views},
        "e2e": {"value": round(value, 5), "unit": "GUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="elsa_b200", choices=["elsa_b200", "reference"])
    ap.add_argument("--cpu-views", type=int, default=None,
                    help="views per CPU baseline sample (default: 60 for the cpu_baseline of "
                         "this arm, about 10 s on 16 host threads; for --impl reference as many "
                         "as keep the whole run near 90 s, 4 to 60)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sharded", action="store_true",
                    help="run the view-sharded solver (the N > 1 path) also on one GPU")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the parity block (oracle check of the benchmarked operator)")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched-vs-plain small-problem measurement")
    ap.add_argument("--batched-small", action="store_true",
                    help="time the batched-vs-plain leg on a reduced set (12 instances of edges "
                         "64-128, 60-180 views, 10 iterations) instead of the 64-instance one")
    ap.add_argument("--secondary", default=None,
                    help="time other projector workloads instead ('all' or a comma list of: %s)"
                         % ", ".join(SECONDARY))
    ap.add_argument("--knob", action="append",
                    help="with --secondary: set a projector knob, name=value (names: %s); "
                         "repeatable, ignored where the projector lacks the knob"
                         % ", ".join(("forward_threads", "adjoint_chunks", "adjoint_threads",
                                      "adjoint_scatter", "exact_weights", "checkpoint_depth")))
    ap.add_argument("--size", type=int, default=256,
                    help="volume edge (profiling only; the benchmark workload is 256)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.secondary:
        run_secondary(args)
        return
    if args.impl == "reference":
        if args.cpu_views is None:
            # about 0.17 s per view (forward + adjoint) on 16 host threads
            args.cpu_views = max(4, min(60, int(90.0 / (args.steps + args.warmup) / 0.17)))
        run_reference(args)
    else:
        if args.cpu_views is None:
            args.cpu_views = 60
        run_elsa(args)


if __name__ == "__main__":
    main()
