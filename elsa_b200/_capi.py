"""ctypes binding of the elsa_b200 C ABI (include/elsa_b200.h).

Loading fails loudly when libelsa_b200.so has not been built: there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libelsa_b200.so")
POSE_FLOATS = 40

SUCCESS = 0
STATUS_NAMES = {
    0: "ELSA_SUCCESS",
    1: "ELSA_ERROR_INVALID_ARGUMENT",
    2: "ELSA_ERROR_LOGIC",
    3: "ELSA_ERROR_BAD_ALLOC",
    4: "ELSA_ERROR_CUDA",
    5: "ELSA_ERROR_NOT_SUPPORTED",
}

PROJECTOR_JOSEPH = 0
PROJECTOR_SIDDON = 1
PROJECTOR_BLOB = 2
PROJECTOR_BSPLINE = 3
PROJECTOR_PHASE_CONTRAST_BLOB = 4
PROJECTOR_PHASE_CONTRAST_BSPLINE = 5
PROJECTOR_BINARY = 6
PROJECTOR_RAY_BLOB = 7
PROJECTOR_RAY_BSPLINE = 8
FOOTPRINT_REFERENCE = 0
FOOTPRINT_RECTANGLE = 1
SOLVER_CGNE = 0
SOLVER_CGLS = 1
SOLVER_LANDWEBER = 2
SOLVER_APGD = 3
SOLVER_SIRT = 4
SOLVER_FGM = 5
SOLVER_OGM = 6
SOLVER_SQS = 7
SUBSET_ROUND_ROBIN = 0
SUBSET_ROTATIONAL_CLUSTERING = 1
PROX_IDENTITY = 0
PROX_BOX = 1
PROX_L1 = 2
KNOB_FORWARD_THREADS = 0
KNOB_ADJOINT_CHUNKS = 1
KNOB_ADJOINT_THREADS = 2
KNOB_ADJOINT_SCATTER = 3
KNOB_EXACT_WEIGHTS = 4
KNOB_CHECKPOINT_DEPTH = 5
KNOB_COUNT = 6
KNOB_NAMES = ("forward_threads", "adjoint_chunks", "adjoint_threads", "adjoint_scatter",
              "exact_weights", "checkpoint_depth")

IO_MAX_DIMS = 8
IO_TYPES = ("int8", "uint8", "int16", "uint16", "int32", "uint32", "float32", "float64")


class ImageInfo(ctypes.Structure):
    """elsa_image_info"""
    _fields_ = [("ndim", ctypes.c_int32), ("data_type", ctypes.c_int32),
                ("dims", ctypes.c_int64 * IO_MAX_DIMS), ("spacing", ctypes.c_float * IO_MAX_DIMS)]


# Every function the header declares: name -> (restype, argtypes)
_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_f32 = ctypes.c_float
_st = ctypes.c_int
SIGNATURES = {
    "elsa_last_error": (ctypes.c_char_p, []),
    "elsa_abi_version": (_i32, []),
    "elsa_pose_2d": (_st, [_f32, _f32, _f32, _vp, _vp, _vp, _vp, _f32, _vp, _vp]),
    "elsa_pose_3d": (_st, [_f32, _f32, _vp, _vp, _vp, _vp, _f32, _f32, _f32, _vp, _vp, _vp]),
    "elsa_circle_trajectory": (_st, [_i32, _vp, _vp, _i64, _f32, _f32, _f32, _vp, _vp, _vp,
                                     _vp]),
    "elsa_projector_create": (_st, [_i32, _i32, _vp, _vp, _vp, _vp, _i32,
                                    ctypes.POINTER(_vp)]),
    "elsa_projector_create_curved": (_st, [_i32, _i32, _vp, _vp, _vp, _vp, _i32, _f32, _f32,
                                           ctypes.POINTER(_vp)]),
    "elsa_curved_detector_coords": (_st, [_i32, _i32, _i32, _f32, _f32, _vp]),
    "elsa_projector_destroy": (_st, [_vp]),
    "elsa_projector_sizes": (_st, [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
    "elsa_projector_info": (_st, [_vp, _i32, ctypes.POINTER(_i64)]),
    "elsa_projector_wait_test": (_st, [_vp, _i64, _i32]),
    "elsa_projector_apply_batch": (_st, [_vp, _vp, _i64, _vp, _i64, _i32, _vp]),
    "elsa_batch_cgne_create": (_st, [_vp, _vp, _vp, _i32, _vp, ctypes.POINTER(_vp)]),
    "elsa_batch_cgne_iterate": (_st, [_vp, _i32, _vp]),
    "elsa_batch_cgne_iterate_graph": (_st, [_vp, _i32, _vp]),
    "elsa_batch_cgne_residuals": (_st, [_vp, _vp, _vp]),
    "elsa_batch_cgne_destroy": (_st, [_vp]),
    "elsa_cgne_split_create": (_st, [_vp, _vp, ctypes.POINTER(_vp)]),
    "elsa_cgne_split_backproject": (_st, [_vp, _vp, _vp, _vp]),
    "elsa_cgne_split_begin": (_st, [_vp, _vp, _vp]),
    "elsa_cgne_split_normal": (_st, [_vp, _vp, _vp]),
    "elsa_cgne_split_update": (_st, [_vp, _vp, _vp]),
    "elsa_cgne_split_residual": (_st, [_vp, _vp, _vp]),
    "elsa_cgne_split_destroy": (_st, [_vp]),
    "elsa_projector_apply_adjoint_batch": (_st, [_vp, _vp, _i64, _vp, _i64, _i32, _vp]),
    "elsa_projector_get_knob": (_st, [_vp, _i32, ctypes.POINTER(_i32)]),
    "elsa_projector_knob_candidates": (_st, [_vp, _i32, _vp, _i32, ctypes.POINTER(_i32)]),
    "elsa_projector_set_knob": (_st, [_vp, _i32, _i32]),
    "elsa_projector_autotune": (_st, [_vp, _vp, _i32, _vp, ctypes.POINTER(_i32)]),
    "elsa_tune_cache_size": (_st, [ctypes.POINTER(_i64)]),
    "elsa_tune_cache_clear": (_st, []),
    "elsa_tune_cache_save": (_st, [ctypes.c_char_p]),
    "elsa_tune_cache_load": (_st, [ctypes.c_char_p]),
    "elsa_tune_cache_put": (_st, [ctypes.c_char_p, _vp]),
    "elsa_tune_cache_get": (_st, [ctypes.c_char_p, _vp, ctypes.POINTER(_i32)]),
    "elsa_projector_apply": (_st, [_vp, _vp, _vp, _vp]),
    "elsa_projector_apply_adjoint": (_st, [_vp, _vp, _vp, _vp]),
    "elsa_projector_apply_host": (_st, [_vp, _vp, _vp]),
    "elsa_projector_apply_adjoint_host": (_st, [_vp, _vp, _vp]),
    "elsa_dot": (_st, [_vp, _vp, _i64, _vp, _vp]),
    "elsa_dot_no_alloc": (_st, [_vp, _vp, _i64, _vp, _vp]),
    "elsa_voxel_lut": (_st, [_i32, _i32, _vp, _i32, _i32, _vp, _vp]),
    "elsa_squared_l2_norm": (_st, [_vp, _i64, _vp, _vp]),
    "elsa_lincomb": (_st, [_f32, _vp, _f32, _vp, _vp, _i64, _vp]),
    "elsa_cgne_solve": (_st, [_vp, _vp, _vp, _i32, _i32, _vp]),
    "elsa_solver_create": (_st, [_i32, _vp, _vp, _vp, _i32, ctypes.POINTER(ctypes.c_double),
                                 _i32, _vp, ctypes.POINTER(_vp)]),
    "elsa_solver_step_size": (_st, [_vp, ctypes.POINTER(ctypes.c_double)]),
    "elsa_sqs_create": (_st, [_vp, _vp, _vp, _vp, _i32, _vp, _i32, _i32, ctypes.c_double, _vp,
                              _vp, ctypes.POINTER(_vp)]),
    "elsa_subset_split": (_st, [_i32, _vp, _i32, _i32, _i32, _vp, _vp]),
    "elsa_edf_info": (_st, [ctypes.c_char_p, ctypes.POINTER(ImageInfo)]),
    "elsa_edf_read": (_st, [ctypes.c_char_p, _vp, _i64]),
    "elsa_edf_write": (_st, [ctypes.c_char_p, _vp, _i32, _vp, _vp]),
    "elsa_mhd_info": (_st, [ctypes.c_char_p, ctypes.POINTER(ImageInfo)]),
    "elsa_mhd_read": (_st, [ctypes.c_char_p, _vp, _i64]),
    "elsa_mhd_write": (_st, [ctypes.c_char_p, ctypes.c_char_p, _vp, _i32, _vp, _vp]),
    "elsa_pgm_write": (_st, [ctypes.c_char_p, _vp, _i32, _vp]),
    "elsa_gather_views": (_st, [_vp, _i64, _vp, _i32, _i32, _vp, _vp]),
    "elsa_power_iterations": (_st, [_vp, _i32, _vp, ctypes.POINTER(ctypes.c_double)]),
    "elsa_solver_iterate": (_st, [_vp, _i32, _vp]),
    "elsa_solver_iterate_graph": (_st, [_vp, _i32, _vp]),
    "elsa_solve_batch": (_st, [ctypes.POINTER(_vp), _i32, _i32, _i32]),
    "elsa_solver_squared_residual": (_st, [_vp, _vp, ctypes.POINTER(ctypes.c_double)]),
    "elsa_solver_enable_timing": (_st, [_vp, _i32]),
    "elsa_solver_timing": (_st, [_vp, ctypes.POINTER(ctypes.c_double),
                                 ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_i64)]),
    "elsa_solver_destroy": (_st, [_vp]),
}


class ElsaError(RuntimeError):
    """A failed C ABI call; .status is the elsa_status code."""

    def __init__(self, status, message):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), message))
        self.status = status


class InvalidArgumentError(ElsaError, ValueError):
    pass


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("elsa_b200 native library not built (%s); run "
                              "`python -m elsa_b200.build`" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status):
    if status != SUCCESS:
        msg = lib().elsa_last_error().decode()
        if status == 1:
            raise InvalidArgumentError(status, msg)
        raise ElsaError(status, msg)


def call(name, *args):
    check(getattr(lib(), name)(*args))


def np_ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def circle_trajectory(vol_dims, num_poses, arc_degrees, s2c, c2d, det_size=None,
                      vol_spacing=None, det_spacing=None):
    """Poses (P x 40 float32) and detector dims of a circular trajectory."""
    dim = len(vol_dims)
    vd = np.asarray(vol_dims, np.int64)
    vs = np.ascontiguousarray(vol_spacing if vol_spacing is not None else np.ones(dim),
                              np.float32)
    poses = np.zeros((num_poses, POSE_FLOATS), np.float32)
    det_dims = np.zeros(dim, np.int64)
    ds = np.asarray(det_size, np.int64) if det_size is not None else None
    dsp = np.ascontiguousarray(det_spacing, np.float32) if det_spacing is not None else None
    call("elsa_circle_trajectory", dim, np_ptr(vd), np_ptr(vs), int(num_poses),
         float(arc_degrees), float(s2c), float(c2d), np_ptr(ds) if ds is not None else None,
         np_ptr(dsp) if dsp is not None else None, np_ptr(poses), np_ptr(det_dims))
    return poses, det_dims


def pose_2d(s2c, c2d, angle_rad, vol_spacing, vol_origin, sino_spacing, sino_origin,
            pp_offset=0.0, cor_offset=(0.0, 0.0)):
    out = np.zeros(POSE_FLOATS, np.float32)
    arrs = [np.ascontiguousarray(a, np.float32) for a in
            (vol_spacing, vol_origin, sino_spacing, sino_origin, cor_offset)]
    call("elsa_pose_2d", float(s2c), float(c2d), float(angle_rad), np_ptr(arrs[0]),
         np_ptr(arrs[1]), np_ptr(arrs[2]), np_ptr(arrs[3]), float(pp_offset), np_ptr(arrs[4]),
         np_ptr(out))
    return out


def pose_3d(s2c, c2d, vol_spacing, vol_origin, sino_spacing, sino_origin, gamma, beta=0.0,
            alpha=0.0, pp_offset=(0.0, 0.0), cor_offset=(0.0, 0.0, 0.0)):
    out = np.zeros(POSE_FLOATS, np.float32)
    arrs = [np.ascontiguousarray(a, np.float32) for a in
            (vol_spacing, vol_origin, sino_spacing, sino_origin, pp_offset, cor_offset)]
    call("elsa_pose_3d", float(s2c), float(c2d), np_ptr(arrs[0]), np_ptr(arrs[1]),
         np_ptr(arrs[2]), np_ptr(arrs[3]), float(gamma), float(beta), float(alpha),
         np_ptr(arrs[4]), np_ptr(arrs[5]), np_ptr(out))
    return out


class Projector:
    """Owning handle of an elsa_projector (device-side operator)."""

    def __init__(self, kind, vol_dims, det_dims, poses, params=None, curved=None):
        """curved: (opening angle in radian, source-to-detector distance) of a curved detector,
        None for a flat one."""
        self.dim = len(vol_dims)
        self.vol_dims = tuple(int(v) for v in vol_dims)
        self.det_dims = tuple(int(v) for v in det_dims)
        vd = np.asarray(vol_dims, np.int64)
        dd = np.asarray(det_dims, np.int64)
        ps = np.ascontiguousarray(poses, np.float32)
        if ps.size != POSE_FLOATS * self.det_dims[-1]:
            raise InvalidArgumentError(1, "pose array does not match the number of poses")
        prm = np.ascontiguousarray(params if params is not None else [], np.float32)
        # False for JosephsMethodCUDA's `fast` adjoint (Joseph parameter 1), which is not the
        # transpose of the forward
        self.matched = not (int(kind) == PROJECTOR_JOSEPH and prm.size > 0 and prm[0] != 0)
        h = ctypes.c_void_p()
        self.curved = None if curved is None else (float(curved[0]), float(curved[1]))
        if self.curved is None:
            call("elsa_projector_create", int(kind), self.dim, np_ptr(vd), np_ptr(dd),
                 np_ptr(ps), np_ptr(prm) if prm.size else None, int(prm.size), ctypes.byref(h))
        else:
            call("elsa_projector_create_curved", int(kind), self.dim, np_ptr(vd), np_ptr(dd),
                 np_ptr(ps), np_ptr(prm) if prm.size else None, int(prm.size),
                 self.curved[0], self.curved[1], ctypes.byref(h))
        self._h = h
        d = ctypes.c_int64()
        r = ctypes.c_int64()
        call("elsa_projector_sizes", self._h, ctypes.byref(d), ctypes.byref(r))
        self.domain_size = d.value
        self.range_size = r.value

    @property
    def handle(self):
        return self._h

    def info(self, key):
        v = ctypes.c_int64()
        call("elsa_projector_info", self._h, int(key), ctypes.byref(v))
        return v.value

    def wait_test(self, wait_cycles, withhold_copies):
        """Test hook of the bounded device waits (elsa_projector_wait_test)."""
        call("elsa_projector_wait_test", self._h, int(wait_cycles), int(bool(withhold_copies)))

    def knob(self, knob):
        """Current value of a launch knob (KNOB_*), -1 when this projector does not use it."""
        v = ctypes.c_int32()
        call("elsa_projector_get_knob", self._h, int(knob), ctypes.byref(v))
        return v.value

    def knob_candidates(self, knob):
        """Values the autotuner may try for `knob` on this geometry ([] when fixed)."""
        n = ctypes.c_int32()
        call("elsa_projector_knob_candidates", self._h, int(knob), None, 0, ctypes.byref(n))
        out = np.zeros(max(1, n.value), np.int32)
        call("elsa_projector_knob_candidates", self._h, int(knob), np_ptr(out), int(out.size),
             ctypes.byref(n))
        return [int(v) for v in out[:n.value]]

    def set_knob(self, knob, value):
        call("elsa_projector_set_knob", self._h, int(knob), int(value))

    def autotune(self, stream=None, force=False):
        """Time the candidates of every knob and keep the fastest (or take the tuning cache's
        entry for this shape). Returns ({knob name: value}, from_cache)."""
        vals = np.full(KNOB_COUNT, -1, np.int32)
        hit = ctypes.c_int32()
        call("elsa_projector_autotune", self._h, ctypes.c_void_p(stream or 0), int(bool(force)),
             np_ptr(vals), ctypes.byref(hit))
        return {KNOB_NAMES[k]: int(vals[k]) for k in range(KNOB_COUNT)}, bool(hit.value)

    def apply_ptr(self, x_ptr, y_ptr, stream=None):
        call("elsa_projector_apply", self._h, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr),
             ctypes.c_void_p(stream or 0))

    def apply_adjoint_ptr(self, y_ptr, x_ptr, stream=None):
        call("elsa_projector_apply_adjoint", self._h, ctypes.c_void_p(y_ptr),
             ctypes.c_void_p(x_ptr), ctypes.c_void_p(stream or 0))

    def apply_batch_ptr(self, x_ptr, x_stride, y_ptr, y_stride, batch, stream=None):
        """y + b y_stride = A (x + b x_stride) for b < batch (strides in floats)."""
        call("elsa_projector_apply_batch", self._h, ctypes.c_void_p(x_ptr), int(x_stride),
             ctypes.c_void_p(y_ptr), int(y_stride), int(batch), ctypes.c_void_p(stream or 0))

    def apply_adjoint_batch_ptr(self, y_ptr, y_stride, x_ptr, x_stride, batch, stream=None):
        """x + b x_stride = A^T (y + b y_stride) for b < batch (strides in floats)."""
        call("elsa_projector_apply_adjoint_batch", self._h, ctypes.c_void_p(y_ptr),
             int(y_stride), ctypes.c_void_p(x_ptr), int(x_stride), int(batch),
             ctypes.c_void_p(stream or 0))

    def apply_host(self, x):
        x = np.ascontiguousarray(x, np.float32).reshape(-1)
        if x.size != self.domain_size:
            raise InvalidArgumentError(1, "input size does not match the domain")
        y = np.empty(self.range_size, np.float32)
        call("elsa_projector_apply_host", self._h, np_ptr(x), np_ptr(y))
        return y

    def apply_adjoint_host(self, y):
        y = np.ascontiguousarray(y, np.float32).reshape(-1)
        if y.size != self.range_size:
            raise InvalidArgumentError(1, "input size does not match the range")
        x = np.empty(self.domain_size, np.float32)
        call("elsa_projector_apply_adjoint_host", self._h, np_ptr(y), np_ptr(x))
        return x

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().elsa_projector_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def curved_detector_coords(dim, nu, nv, angle, s2d):
    """Planar (u', v') of every pixel centre of a curved detector, shape (nv, nu, 2)."""
    h = int(nv) if dim == 3 else 1
    out = np.zeros(2 * int(nu) * h, np.float32)
    call("elsa_curved_detector_coords", int(dim), int(nu), h, float(angle), float(s2d),
         np_ptr(out))
    return out.reshape(h, int(nu), 2)


def subset_split(dim, poses, num_subsets, strategy=SUBSET_ROUND_ROBIN):
    """Ordered-subset partition of the poses (SubsetSampler): a list of num_subsets lists of
    pose indices."""
    ps = np.ascontiguousarray(poses, np.float32).reshape(-1)
    n = ps.size // POSE_FLOATS
    order = np.zeros(max(1, n), np.int32)
    sizes = np.zeros(max(1, int(num_subsets)), np.int32)
    call("elsa_subset_split", int(dim), np_ptr(ps), int(n), int(num_subsets), int(strategy),
         np_ptr(order), np_ptr(sizes))
    out, k = [], 0
    for c in sizes[:int(num_subsets)]:
        out.append([int(v) for v in order[k:k + int(c)]])
        k += int(c)
    return out


def gather_views(sino_ptr, view_size, views, total_views, out_ptr, stream=None):
    """Device copy of the sinogram views `views` (in that order) to out (elsa_gather_views)."""
    idx = np.ascontiguousarray(views, np.int32)
    call("elsa_gather_views", ctypes.c_void_p(sino_ptr), int(view_size),
         np_ptr(idx) if idx.size else None, int(idx.size), int(total_views),
         ctypes.c_void_p(out_ptr), ctypes.c_void_p(stream or 0))


def _image_read(fmt, path):
    info = ImageInfo()
    call("elsa_%s_info" % fmt, os.fsencode(path), ctypes.byref(info))
    dims = [int(info.dims[i]) for i in range(info.ndim)]
    spacing = [float(info.spacing[i]) for i in range(info.ndim)]
    data = np.empty(int(np.prod(dims)), np.float32)
    call("elsa_%s_read" % fmt, os.fsencode(path), np_ptr(data), int(data.size))
    return data, dims, spacing, IO_TYPES[info.data_type]


def edf_read(path):
    """(flat float32 data x fastest, dims, spacing, stored type) of an EDF file."""
    return _image_read("edf", path)


def mhd_read(meta_path):
    """(flat float32 data x fastest, dims, spacing, stored type) of an MHD meta + raw file."""
    return _image_read("mhd", meta_path)


def _shape_args(data, dims, spacing):
    d = np.ascontiguousarray(dims, np.int64)
    buf = np.ascontiguousarray(data, np.float32).reshape(-1)
    if buf.size != int(np.prod(d)):
        raise InvalidArgumentError(1, "image data does not match its dimensions")
    sp = None if spacing is None else np.ascontiguousarray(spacing, np.float32)
    if sp is not None and sp.size != d.size:
        raise InvalidArgumentError(1, "one spacing per dimension")
    return buf, d, sp


def edf_write(path, data, dims, spacing=None):
    buf, d, sp = _shape_args(data, dims, spacing)
    call("elsa_edf_write", os.fsencode(path), np_ptr(buf), int(d.size), np_ptr(d),
         np_ptr(sp) if sp is not None else None)


def mhd_write(meta_path, raw_path, data, dims, spacing=None):
    buf, d, sp = _shape_args(data, dims, spacing)
    call("elsa_mhd_write", os.fsencode(meta_path), os.fsencode(raw_path), np_ptr(buf),
         int(d.size), np_ptr(d), np_ptr(sp) if sp is not None else None)


def pgm_write(path, data, dims):
    buf, d, _ = _shape_args(data, dims, None)
    call("elsa_pgm_write", os.fsencode(path), np_ptr(buf), int(d.size), np_ptr(d))


def tune_cache_size():
    n = ctypes.c_int64()
    call("elsa_tune_cache_size", ctypes.byref(n))
    return n.value


def tune_cache_clear():
    call("elsa_tune_cache_clear")


def tune_cache_save(path):
    """Write the process-wide tuning cache to a text file (one line per projector shape)."""
    call("elsa_tune_cache_save", os.fsencode(path))


def tune_cache_load(path):
    """Add the entries of a file written by tune_cache_save to the tuning cache."""
    call("elsa_tune_cache_load", os.fsencode(path))


def tune_cache_put(key, values):
    v = np.ascontiguousarray(values, np.int32)
    if v.size != KNOB_COUNT:
        raise InvalidArgumentError(1, "tune_cache_put: need %d knob values" % KNOB_COUNT)
    call("elsa_tune_cache_put", key.encode(), np_ptr(v))


def tune_cache_get(key):
    """Knob values cached under `key` ("kind:dim:nx,ny,nz:nu,nv,np"), or None."""
    v = np.zeros(KNOB_COUNT, np.int32)
    found = ctypes.c_int32()
    call("elsa_tune_cache_get", key.encode(), np_ptr(v), ctypes.byref(found))
    return [int(a) for a in v] if found.value else None


def voxel_lut(kind, dim, params=(), samples=100):
    """(table, support) of a voxel projector kind (ProjectedBlob / ProjectedBSpline LUTs)."""
    import numpy as _np
    params = _np.ascontiguousarray(params, _np.float32)
    out = _np.empty(int(samples), _np.float32)
    sup = ctypes.c_float()
    call("elsa_voxel_lut", int(kind), int(dim),
         ctypes.c_void_p(params.ctypes.data if params.size else 0), int(params.size),
         int(samples), ctypes.c_void_p(out.ctypes.data), ctypes.byref(sup))
    return out, sup.value


def solve_batch(solvers, iterations, streams=8):
    """Run `iterations` iterations of every Solver concurrently, each as a CUDA graph, over
    `streams` streams; returns when all are done."""
    arr = (ctypes.c_void_p * max(1, len(solvers)))(*[s._h.value for s in solvers])
    call("elsa_solve_batch", arr, len(solvers), int(iterations), int(streams))


def power_iterations(projector, iterations=5, stream=None):
    """Largest eigenvalue of A^T A (powerIterations(adjoint(A) * A), PowerIterations.cpp:10-27)."""
    v = ctypes.c_double()
    call("elsa_power_iterations", projector.handle, int(iterations), ctypes.c_void_p(stream or 0),
         ctypes.byref(v))
    return v.value


class BatchCGNE:
    """Owning handle of an elsa_batch_cgne: CGNE on many 3D Joseph operators advanced together
    (x0 = 0); b_ptrs / x_ptrs are device buffers that must outlive the batch."""

    def __init__(self, projectors, b_ptrs, x_ptrs, stream=None):
        n = len(projectors)
        self._keep = list(projectors)
        ops = (ctypes.c_void_p * n)(*[p.handle.value for p in projectors])
        bs = (ctypes.c_void_p * n)(*[int(v) for v in b_ptrs])
        xs = (ctypes.c_void_p * n)(*[int(v) for v in x_ptrs])
        h = ctypes.c_void_p()
        call("elsa_batch_cgne_create", ops, bs, xs, n, ctypes.c_void_p(stream or 0),
             ctypes.byref(h))
        self._h = h
        self.size = n

    def iterate(self, iterations, stream=None):
        call("elsa_batch_cgne_iterate", self._h, int(iterations), ctypes.c_void_p(stream or 0))

    def iterate_graph(self, iterations, stream):
        call("elsa_batch_cgne_iterate_graph", self._h, int(iterations), ctypes.c_void_p(stream))

    def squared_residuals(self, stream=None):
        out = np.zeros(self.size, np.float64)
        call("elsa_batch_cgne_residuals", self._h, np_ptr(out), ctypes.c_void_p(stream or 0))
        return out

    def close(self):
        if self._h:
            call("elsa_batch_cgne_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Solver:
    """Owning handle of an elsa_solver: a device-resident iterative solve on device buffers
    (b: range, x: domain; both must outlive the solver)."""

    def __init__(self, kind, projector, b_ptr, x_ptr, use_x0=False, stream=None, params=()):
        """params: the solver's constructor arguments in the C ABI's order (elsa_b200.h):
        CGLS (eps, tol), Landweber (step,), APGD (mu, epsilon, prox, lower, upper, sigma)."""
        self._proj = projector  # keep the operator alive
        h = ctypes.c_void_p()
        params = [float(v) for v in params]
        arr = (ctypes.c_double * max(1, len(params)))(*params)
        call("elsa_solver_create", int(kind), projector.handle, ctypes.c_void_p(b_ptr),
             ctypes.c_void_p(x_ptr), int(bool(use_x0)), arr, len(params),
             ctypes.c_void_p(stream or 0), ctypes.byref(h))
        self._h = h

    @classmethod
    def sqs(cls, projector, b_ptr, x_ptr, subsets=(), use_x0=False, momentum=True,
            epsilon=1.1920928955078125e-07, preconditioner_ptr=None, stream=None):
        """SQS on LeastSquares(projector, b) (elsa_sqs_create). subsets: (Projector, b_ptr)
        pairs of an ordered-subset split (none: the full problem)."""
        self = cls.__new__(cls)
        self._proj = projector
        self._subsets = list(subsets)  # keep the subset operators alive
        n = len(self._subsets)
        projs = (ctypes.c_void_p * max(1, n))(*[p.handle.value for p, _ in self._subsets])
        bs = (ctypes.c_void_p * max(1, n))(*[int(bp) for _, bp in self._subsets])
        h = ctypes.c_void_p()
        call("elsa_sqs_create", projector.handle, ctypes.c_void_p(b_ptr), projs, bs, n,
             ctypes.c_void_p(x_ptr), int(bool(use_x0)), int(bool(momentum)), float(epsilon),
             ctypes.c_void_p(preconditioner_ptr or 0), ctypes.c_void_p(stream or 0),
             ctypes.byref(h))
        self._h = h
        return self

    def iterate_graph(self, iterations, stream):
        call("elsa_solver_iterate_graph", self._h, int(iterations), ctypes.c_void_p(stream))

    def step_size(self):
        v = ctypes.c_double()
        call("elsa_solver_step_size", self._h, ctypes.byref(v))
        return v.value

    def iterate(self, iterations, stream=None):
        call("elsa_solver_iterate", self._h, int(iterations), ctypes.c_void_p(stream or 0))

    def squared_residual(self, stream=None):
        v = ctypes.c_double()
        call("elsa_solver_squared_residual", self._h, ctypes.c_void_p(stream or 0),
             ctypes.byref(v))
        return v.value

    def enable_timing(self, on=True):
        call("elsa_solver_enable_timing", self._h, int(bool(on)))

    def timing(self):
        f, a, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
        call("elsa_solver_timing", self._h, ctypes.byref(f), ctypes.byref(a), ctypes.byref(n))
        return f.value, a.value, n.value

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().elsa_solver_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
