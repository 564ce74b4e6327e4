"""elsa_dot_no_alloc: the inner product for callers that cannot allocate device memory.

cudaMalloc/cudaFree synchronize the device, so a caller inside a latency-bound loop, or a host
that routes all device memory through its own pool, cannot let the library allocate per call.
elsa_dot_no_alloc keeps its partial sums in a fixed device array instead. This file checks it
against elsa_dot through the C ABI and against numpy's float64 sum, on two calls in a row (the
shared array keeps the previous call's contents, which must not leak into the next result), that
sizes beyond the array's limit are refused, and that its translation unit references no
allocation routine. The file name sorts last so that a run stopping at the first failure has run
every other test before it.
"""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

# Both entry points sum float products in float64, in different orders; the tolerance is the one
# the vector-op tests use against a float64 numpy reference (1e-13 of sum |x_i y_i|).
REL = 1e-13


def _dot(torch, name, x, y, n, offset=0):
    from elsa_b200 import _capi
    res = torch.full((1,), np.nan, dtype=torch.float64, device="cuda")
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    xp = ctypes.c_void_p(x.data_ptr() + 4 * offset if x.numel() else 0)
    yp = ctypes.c_void_p(y.data_ptr() + 4 * offset if y.numel() else 0)
    _capi.call(name, xp, yp, int(n), ctypes.c_void_p(res.data_ptr()), s)
    torch.cuda.synchronize()
    return float(res.cpu().numpy()[0])


@pytest.mark.gpu
@pytest.mark.parametrize("n, offset", [(0, 0), (1, 0), (4097, 1), ((1 << 20) + 3, 0),
                                       (16777216, 0)])
def test_no_alloc_matches_dot_twice(cuda, n, offset):
    torch = cuda
    for call in range(2):  # two calls in a row with different data
        rng = np.random.default_rng(1000 * call + n)
        xs = rng.standard_normal(n + offset).astype(np.float32)
        ys = rng.standard_normal(n + offset).astype(np.float32)
        x = torch.from_numpy(xs).cuda()
        y = torch.from_numpy(ys).cuda()
        ref = _dot(torch, "elsa_dot", x, y, n, offset)
        got = _dot(torch, "elsa_dot_no_alloc", x, y, n, offset)
        x64, y64 = xs[offset:].astype(np.float64), ys[offset:].astype(np.float64)
        scale = max(1.0, float(np.dot(np.abs(x64), np.abs(y64))))
        assert abs(got - ref) <= REL * scale, (call, got, ref)
        assert abs(got - float(np.dot(x64, y64))) <= REL * scale, (call, got)


@pytest.mark.gpu
def test_no_alloc_refuses_oversize(cuda):
    import elsa_b200
    from elsa_b200 import _capi
    torch = cuda
    x = torch.zeros(4, dtype=torch.float32, device="cuda")
    res = torch.zeros(1, dtype=torch.float64, device="cuda")
    too_big = 67108864 + 1
    with pytest.raises(elsa_b200.InvalidArgumentError, match="exceeds the maximum"):
        # refused before any launch, so the short buffers are never read
        _capi.call("elsa_dot_no_alloc", ctypes.c_void_p(x.data_ptr()),
                   ctypes.c_void_p(x.data_ptr()), too_big, ctypes.c_void_p(res.data_ptr()),
                   ctypes.c_void_p(0))


def test_no_alloc_unit_references_no_allocator():
    """The translation unit of elsa_dot_no_alloc names no allocating CUDA runtime routine, so no
    code path of the entry point can allocate (its C ABI wrapper only forwards to it)."""
    from elsa_b200 import build
    build.build()
    nm = shutil.which("nm")
    if nm is None:
        pytest.skip("nm is not installed")
    obj = os.path.join(build.BUILD, "noalloc.cu.o")
    out = subprocess.run([nm, "-u", "-C", obj], capture_output=True, text=True, check=True).stdout
    undefined = [line.split()[-1] for line in out.splitlines() if line.strip()]
    allocators = ("cudaMalloc", "cudaFree", "cudaMallocAsync", "cudaFreeAsync", "cudaMallocManaged",
                  "cudaMallocHost", "cudaHostAlloc", "cuMemAlloc", "cuMemCreate")
    bad = [u for u in undefined if any(u == a or u.startswith(a + "_") or u.startswith(a + "(")
                                       for a in allocators)]
    assert not bad, bad
    assert any("cudaGetSymbolAddress" in u for u in undefined)
