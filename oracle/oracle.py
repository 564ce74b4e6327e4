"""ctypes bindings of the oracle (oracle/oracle.cpp), the CPU restatement of elsa's reference
algorithms for the projector + solver hot path.

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use it
as the checker. The product (the elsa_b200 package) never imports it.

Geometry is exchanged as pose records of 40 float32 (P at 0, Pinv at 12, C at 24, ext at 27,
sdd at 39; row-major, dim x dim+1 / dim+1 x dim), the same layout as the product's C ABI.
Volumes are float arrays with x fastest (numpy shape (nz, ny, nx) in C order); sinograms have u
fastest and the pose last (numpy shape (P, V, U)).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
POSE_FLOATS = 40

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")


def build(force=False):
    """Compile oracle.cpp and voxel_oracle.cpp into liboracle.so (g++, OpenMP, no FP
    contraction)."""
    srcs = [os.path.join(_HERE, "oracle.cpp"), os.path.join(_HERE, "voxel_oracle.cpp")]
    if (not force and os.path.exists(_LIB_PATH)
            and all(os.path.getmtime(_LIB_PATH) >= os.path.getmtime(f) for f in srcs)):
        return _LIB_PATH
    cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared",
           "-o", _LIB_PATH] + srcs
    subprocess.check_call(cmd)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        c_int, c_i64, c_f = ctypes.c_int, ctypes.c_int64, ctypes.c_float
        L.oracle_num_threads.restype = c_int
        L.oracle_set_num_threads.argtypes = [c_int]
        L.oracle_set_adjoint_atomic.argtypes = [c_int]
        L.oracle_geometry2d.argtypes = [c_f, c_f, c_f, _f32p, _f32p, _f32p, _f32p, c_f, _f32p,
                                        _f32p]
        L.oracle_geometry3d.argtypes = [c_f, c_f, _f32p, _f32p, _f32p, _f32p, c_f, c_f, c_f,
                                        _f32p, _f32p, _f32p]
        L.oracle_circle_trajectory.argtypes = [c_int, _i64p, _f32p, c_i64, c_f, c_f, c_f,
                                               ctypes.c_void_p, ctypes.c_void_p, _f32p, _i64p]
        L.oracle_ray.argtypes = [c_int, _i64p, _f32p, c_i64, _f32p, _f32p]
        L.oracle_dd_setup.argtypes = [c_int, _i64p, _f32p, _f32p, _f32p, _f32p,
                                      ctypes.POINTER(c_f), ctypes.POINTER(c_int),
                                      ctypes.POINTER(c_i64)]
        _vp = ctypes.c_void_p  # optional curved-detector coordinates (None: flat detector)
        for name, fp in (("f32", _f32p), ("f64", _f64p)):
            fn = getattr(L, "oracle_joseph_" + name)
            fn.argtypes = [c_int, c_int, _i64p, _i64p, _f32p, fp, fp, c_int, _vp]
            fn = getattr(L, "oracle_siddon_" + name)
            fn.argtypes = [c_int, c_int, _i64p, _i64p, _f32p, fp, fp, _vp]
            fn = getattr(L, "oracle_binary_" + name)
            fn.argtypes = [c_int, c_int, _i64p, _i64p, _f32p, fp, fp, _vp]
        L.oracle_curved_coords.argtypes = [c_int, c_i64, c_i64, c_f, c_f, _f32p]
        for name, fp in (("f32", _f32p), ("f64", _f64p)):
            getattr(L, "oracle_lut_" + name).argtypes = [c_int, c_int, _i64p, _i64p, _f32p,
                                                         _f32p, c_i64, c_f, c_int, fp, fp]
        L.oracle_joseph_sample_count.argtypes = [c_int, _i64p, _i64p, _f32p]
        L.oracle_joseph_sample_count.restype = c_i64
        L.oracle_siddon_visit_count.argtypes = [c_int, _i64p, _i64p, _f32p]
        L.oracle_siddon_visit_count.restype = c_i64
        L.oracle_bessel.argtypes = [c_int, ctypes.c_double]
        L.oracle_bessel.restype = ctypes.c_double
        L.oracle_blob_projected.argtypes = [c_f, c_f, c_f, c_int, c_int]
        L.oracle_blob_projected.restype = c_f
        L.oracle_bspline1d.argtypes = [c_f, c_int]
        L.oracle_bspline1d.restype = c_f
        L.oracle_blob_lut.argtypes = [c_f, c_f, c_int, c_int, c_i64, _f32p]
        L.oracle_bspline_lut.argtypes = [c_int, c_int, c_int, c_i64, _f32p]
        L.oracle_lut_lerp.argtypes = [_f32p, c_i64, c_f, c_f]
        L.oracle_lut_lerp.restype = c_f
        for name, fp in (("f32", _f32p), ("f64", _f64p)):
            fn = getattr(L, "oracle_voxel_" + name)
            fn.argtypes = [c_int, c_int, _i64p, _i64p, _f32p, _f32p, c_i64, c_f, c_int, c_int,
                           fp, fp]
        L.oracle_dot_f32.argtypes = [_f32p, _f32p, c_i64]
        L.oracle_dot_f32.restype = ctypes.c_double
        L.oracle_dot_f64.argtypes = [_f64p, _f64p, c_i64]
        L.oracle_dot_f64.restype = ctypes.c_double
        _lib = L
    return _lib


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def set_num_threads(n):
    lib().oracle_set_num_threads(int(n))


def set_adjoint_atomic(on):
    """True: the adjoints add with `omp atomic` as the reference does (its speed, a run-dependent
    order; for CPU-baseline timing only). False (the default): the fixed, deterministic order."""
    lib().oracle_set_adjoint_atomic(1 if on else 0)


def num_threads():
    return lib().oracle_num_threads()


def geometry2d(s2c, c2d, angle_rad, vol_spacing, vol_origin, sino_spacing, sino_origin,
               pp_offset=0.0, cor_offset=(0.0, 0.0)):
    """One 2D pose (core/Geometry.cpp:12-51) as a 40-float record."""
    out = np.zeros(POSE_FLOATS, np.float32)
    lib().oracle_geometry2d(s2c, c2d, angle_rad, _f32(vol_spacing), _f32(vol_origin),
                            _f32(sino_spacing), _f32(sino_origin), pp_offset, _f32(cor_offset),
                            out)
    return out


def geometry3d(s2c, c2d, vol_spacing, vol_origin, sino_spacing, sino_origin, gamma, beta=0.0,
               alpha=0.0, pp_offset=(0.0, 0.0), cor_offset=(0.0, 0.0, 0.0)):
    """One 3D pose (core/Geometry.cpp:53-109) as a 40-float record."""
    out = np.zeros(POSE_FLOATS, np.float32)
    lib().oracle_geometry3d(s2c, c2d, _f32(vol_spacing), _f32(vol_origin), _f32(sino_spacing),
                            _f32(sino_origin), gamma, beta, alpha, _f32(pp_offset),
                            _f32(cor_offset), out)
    return out


def circle_trajectory(vol_dims, num_poses, arc_degrees, s2c, c2d, det_size=None,
                      vol_spacing=None, det_spacing=None):
    """CircleTrajectoryGenerator::createTrajectory: returns (poses[P,40], det_dims)."""
    dim = len(vol_dims)
    vd = np.asarray(vol_dims, np.int64)
    vs = _f32(vol_spacing if vol_spacing is not None else np.ones(dim))
    poses = np.zeros((num_poses, POSE_FLOATS), np.float32)
    det_dims = np.zeros(dim, np.int64)
    ds = np.asarray(det_size, np.int64) if det_size is not None else None
    dsp = _f32(det_spacing) if det_spacing is not None else None
    lib().oracle_circle_trajectory(
        dim, vd, vs, num_poses, float(arc_degrees), float(s2c), float(c2d),
        ds.ctypes.data if ds is not None else None,
        dsp.ctypes.data if dsp is not None else None, poses, det_dims)
    return poses, det_dims


def ray(det_dims, poses, ir):
    dim = len(det_dims)
    o = np.zeros(dim, np.float32)
    d = np.zeros(dim, np.float32)
    lib().oracle_ray(dim, np.asarray(det_dims, np.int64), _f32(poses), ir, o, d)
    return o, d


def dd_setup(vol_dims, origin, direction):
    dim = len(vol_dims)
    pos = np.zeros(dim, np.float32)
    step = np.zeros(dim, np.float32)
    length = ctypes.c_float()
    drv = ctypes.c_int()
    n = ctypes.c_int64()
    lib().oracle_dd_setup(dim, np.asarray(vol_dims, np.int64), _f32(origin), _f32(direction),
                          pos, step, ctypes.byref(length), ctypes.byref(drv), ctypes.byref(n))
    return pos, step, length.value, drv.value, n.value


def _det_count(det_dims):
    return int(np.prod(det_dims))


def _vol_count(vol_dims):
    return int(np.prod(vol_dims))


def _call_projector(name, adjoint, vol_dims, det_dims, poses, data, dtype, extra=(),
                    coords=None):
    dim = len(vol_dims)
    vd = np.asarray(vol_dims, np.int64)
    dd = np.asarray(det_dims, np.int64)
    inp = np.ascontiguousarray(data, dtype=dtype).reshape(-1)
    n_out = _vol_count(vol_dims) if adjoint else _det_count(det_dims)
    out = np.zeros(n_out, dtype)
    suffix = "f32" if dtype == np.float32 else "f64"
    cc = None if coords is None else np.ascontiguousarray(coords, np.float32).reshape(-1)
    if cc is not None and cc.size != 2 * int(np.prod(dd[:-1])):
        raise ValueError("curved detector coordinates: 2 floats per detector pixel")
    getattr(lib(), "oracle_%s_%s" % (name, suffix))(
        int(adjoint), dim, vd, dd, _f32(poses), inp, out, *extra,
        cc.ctypes.data_as(ctypes.c_void_p) if cc is not None else None)
    return out


def curved_coords(dim, nu, nv, angle, s2d):
    """CurvedDetectorDescriptor::getPlanarCoords (core/Descriptors/CurvedDetectorDescriptor.cpp:
    33-91): planar (u', v') of every pixel centre, shape (nv, nu, 2) (nv = 1 in 2D)."""
    h = nv if dim == 3 else 1
    out = np.zeros(2 * nu * h, np.float32)
    lib().oracle_curved_coords(int(dim), int(nu), int(h), float(angle), float(s2d), out)
    return out.reshape(h, nu, 2)


def joseph(x, vol_dims, det_dims, poses, dtype=np.float32, mode=0, coords=None):
    """Joseph forward projection (projectors/JosephsMethod.cpp:140-198). mode 0 accumulates the
    sample position like the reference; mode 1 evaluates it as fma(j, step, pos0). coords: a
    curved detector's planar pixel coordinates (curved_coords)."""
    return _call_projector("joseph", False, vol_dims, det_dims, poses, x, dtype, (mode,), coords)


def joseph_adjoint(y, vol_dims, det_dims, poses, dtype=np.float32, mode=0, coords=None):
    return _call_projector("joseph", True, vol_dims, det_dims, poses, y, dtype, (mode,), coords)


def siddon(x, vol_dims, det_dims, poses, dtype=np.float32, coords=None):
    """Siddon forward projection (projectors/SiddonsMethod.cpp:76-100)."""
    return _call_projector("siddon", False, vol_dims, det_dims, poses, x, dtype, coords=coords)


def siddon_adjoint(y, vol_dims, det_dims, poses, dtype=np.float32, coords=None):
    return _call_projector("siddon", True, vol_dims, det_dims, poses, y, dtype, coords=coords)


def binary(x, vol_dims, det_dims, poses, dtype=np.float32, coords=None):
    """BinaryMethod forward projection (projectors/BinaryMethod.cpp:66-111): the sum of the voxels
    that TraverseAABB visits."""
    return _call_projector("binary", False, vol_dims, det_dims, poses, x, dtype, coords=coords)


def binary_adjoint(y, vol_dims, det_dims, poses, dtype=np.float32, coords=None):
    return _call_projector("binary", True, vol_dims, det_dims, poses, y, dtype, coords=coords)


def lut_project(adjoint, data, vol_dims, det_dims, poses, lut, radius, support,
                dtype=np.float32):
    """Ray-driven blob / B-spline projector (projectors/LutProjector.h:85-163): the slice walk of
    SliceTraversal and lut(distance to the ray) for the voxels within `support` in each slice.
    The backward walks the box grown by `support`, the forward the volume box, as the
    reference does."""
    dim = len(vol_dims)
    n_out = int(np.prod(vol_dims)) if adjoint else int(np.prod(det_dims))
    data = np.ascontiguousarray(data, dtype).ravel()
    out = np.empty(n_out, dtype)
    lut = _f32(lut)
    fn = lib().oracle_lut_f64 if dtype == np.float64 else lib().oracle_lut_f32
    fn(int(adjoint), dim, np.asarray(vol_dims, np.int64), np.asarray(det_dims, np.int64),
       _f32(poses), lut, lut.size, float(radius), int(support), data, out)
    return out


def joseph_sample_count(vol_dims, det_dims, poses):
    return int(lib().oracle_joseph_sample_count(len(vol_dims), np.asarray(vol_dims, np.int64),
                                                np.asarray(det_dims, np.int64), _f32(poses)))


def siddon_visit_count(vol_dims, det_dims, poses):
    return int(lib().oracle_siddon_visit_count(len(vol_dims), np.asarray(vol_dims, np.int64),
                                               np.asarray(det_dims, np.int64), _f32(poses)))


def dot(a, b):
    a = np.ascontiguousarray(a).reshape(-1)
    b = np.ascontiguousarray(b).reshape(-1)
    if a.dtype == np.float64:
        return lib().oracle_dot_f64(a, np.ascontiguousarray(b, np.float64), a.size)
    return lib().oracle_dot_f32(_f32(a), _f32(b), a.size)


# ---- voxel (blob / B-spline) projectors: oracle/voxel_oracle.cpp --------------------------------
LUT_SIZE = 100  # DEFAULT_PROJECTOR_LUT_SIZE, projectors/Luts.hpp:8
WEIGHT_CLASSIC = 0
WEIGHT_DIFFERENTIAL = 1


def bessel(m, x):
    return lib().oracle_bessel(int(m), float(x))


def blob_projected(s, a, alpha, m, which=0):
    """which: 0 value, 1 derivative, 2 normalized gradient (projectors/Blobs.h:67-210)."""
    return lib().oracle_blob_projected(s, a, alpha, int(m), int(which))


def bspline1d(x, m):
    return lib().oracle_bspline1d(x, int(m))


def blob_lut(radius=2.0, alpha=10.83, order=2, which=0, n=LUT_SIZE):
    out = np.empty(n, np.float32)
    lib().oracle_blob_lut(radius, alpha, int(order), int(which), int(n), out)
    return out


def bspline_lut(dim, order=2, which=0, n=LUT_SIZE):
    out = np.empty(n, np.float32)
    lib().oracle_bspline_lut(int(dim), int(order), int(which), int(n), out)
    return out


def bspline_support(order):
    return float(np.float32((order + 1) * 0.5))


def lut_lerp(lut, support, distance):
    lut = _f32(lut)
    return lib().oracle_lut_lerp(lut, lut.size, support, distance)


def voxel_lut(kind, dim, radius=2.0, alpha=10.83, order=2):
    """(lut, support, weight kind) of a voxel projector: kind one of 'blob', 'bspline',
    'phase_blob', 'phase_bspline' (VoxelProjector.cpp, PhaseContrastProjector.cpp)."""
    phase = kind.startswith("phase")
    which = 0 if not phase else (1 if dim == 2 else 2)
    if kind.endswith("blob"):
        return blob_lut(radius, alpha, order, which), float(np.float32(radius)), int(phase)
    return bspline_lut(dim, order, which), bspline_support(order), int(phase)


def voxel_project(adjoint, data, vol_dims, det_dims, poses, lut, support, weight_kind,
                  loop_mode=1, dtype=np.float32):
    """Blob / B-spline voxel projector (projectors/VoxelComputation.h:116-184). loop_mode 1 visits
    the footprint rectangle; 0 follows the reference CPU loop as written."""
    dim = len(vol_dims)
    n_out = int(np.prod(vol_dims)) if adjoint else int(np.prod(det_dims))
    data = np.ascontiguousarray(data, dtype).ravel()
    out = np.empty(n_out, dtype)
    fn = lib().oracle_voxel_f64 if dtype == np.float64 else lib().oracle_voxel_f32
    lut = _f32(lut)
    fn(int(adjoint), dim, np.asarray(vol_dims, np.int64), np.asarray(det_dims, np.int64),
       _f32(poses), lut, lut.size, float(support), int(weight_kind), int(loop_mode), data, out)
    return out
